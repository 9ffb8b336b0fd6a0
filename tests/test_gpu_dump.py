"""Every intermediate of a proof against the oracle (lg_dump_intermediates).

The GPU prover hands over each intermediate of src/prover.rs:15-199 as it
produces it: the RS tables, encoded matrices and Merkle trees of every
commitment, the folded polynomial, each opening's queries and rows, the
induced bases and enforced sums, every sumcheck triple, each fold round's
f and summed basis, the glue challenges and yr.  Each is recomputed here
by the oracle's own building blocks from the oracle's inputs (its
transcript trace supplies the challenges) and compared bit for bit; the
proof bytes equal the oracle's proof.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def u32(b):
    return np.frombuffer(b, dtype=np.uint32)


def pis(ref, log_m):
    m = 1 << log_m
    sk = ref.eval_sk_at_vks(m)
    out = np.zeros(m, dtype=np.uint32)
    ref.lib().lgref_compute_pis(32, m, sk.ctypes.data, out.ctypes.data)
    return out


def gf_scale(ref, v, c):
    return np.array([ref.gf_mul(int(x), c) for x in v], dtype=np.uint32)


@pytest.mark.parametrize("name", ["small_L12", "small_L14_two_steps", "cfg16_seed16"])
def test_intermediates_match_oracle(lg, ref, ctx, golden, name):
    case = golden["cases"][name]
    steps, m0, n0, k0, lms, lns, ks = case["config"]
    pc = lg.ProverConfig(steps, (1 << m0, 1 << n0), [(1 << m, 1 << n) for m, n in zip(lms, lns)], k0, list(ks))
    rc = ref.config(steps, m0, n0, lms, lns)
    poly = lg.splitmix_coeffs(case["seed"], pc.poly_len)

    proof, d = lg.dump_intermediates(pc, lg.to_device(poly), ctx)
    want = ref.prove(rc, poly, nthreads=8)
    assert proof.to_bytes() == want
    tr = ref.last_trace()
    ch = list(tr.challenges[: tr.n_challenges])

    # commitments: level 0 is the polynomial, level i+1 the f committed in step i
    log_m = [m0] + lms
    cols = [1 << n0] + [1 << n for n in lns]
    # the folded polynomial (partial_eval by the initial_k challenges)
    assert list(u32(d[("fold_challenges", 0)])) == ch[:k0]
    f = ref.partial_eval(poly, ch[:k0], nthreads=8)
    assert np.array_equal(u32(d[("folded", 0)]), f)

    msgs = {0: poly, 1: f}
    mats = {}
    for lv in range(steps + 1):
        lm = log_m[lv]
        assert np.array_equal(u32(d[("twiddles", lv)]), ref.twiddles(lm + 2)), lv
        assert np.array_equal(u32(d[("pis", lv)]), pis(ref, lm)), lv
        # the committed message of levels >= 2 is f after step lv-2's rounds
        if lv in msgs:
            flat, tree = ref.ligero_commit(msgs[lv], lm, cols[lv], nthreads=8)
            assert np.array_equal(u32(d[("encoded", lv)]), flat), lv
            assert np.frombuffer(d[("tree", lv)], dtype=np.uint8).tobytes() == tree.tobytes(), lv
            assert bytes(tr.roots[lv]) == tree.tobytes()[-32:], lv
            mats[lv] = flat.reshape(cols[lv], 4 << lm)

        if lv == steps:
            break
        # opening of commitment lv and the basis it induces
        q = np.frombuffer(d[("queries", lv)], dtype=np.uint64)
        assert list(q) == sorted(set(int(x) for x in q)) and len(q) == 148
        rows = mats[lv][:, q.astype(np.int64)].T.copy()
        assert np.array_equal(u32(d[("opened_rows", lv)]).reshape(148, cols[lv]), rows), lv
        alpha = int(u32(d[("alpha", lv)])[0])
        if lv == 0:
            vch = ch[:k0]
            n = m0 + n0 - k0
            assert alpha == ch[k0]
        else:
            vch = step_rounds[lv - 1]
            n = int(np.log2(fcur.size))
        basis, es = ref.induce(n, rows, vch, [int(x) for x in q], alpha, nthreads=8)
        assert np.array_equal(u32(d[("basis", lv)]), basis), lv
        assert int(u32(d[("enforced_sum", lv)])[0]) == es == tr.enforced_sums[lv], lv
        if lv == 0:
            fcur, Bcur = f, basis
            step_rounds = []
            rnd = 0
            tri = 0
        else:
            beta = int(u32(d[("beta", lv)])[0])
            Bcur = Bcur ^ gf_scale(ref, basis, beta)
            assert np.array_equal(u32(d[("basis_sum", lv)]), Bcur), lv
        s3 = ref.eval_013(fcur, basis)
        assert tuple(int(x) for x in u32(d[("triple", tri)])) == s3
        tri += 1
        # the step's fold rounds
        rs = []
        for _ in range(ks[lv]):
            r = int(u32(d[("round_challenge", rnd)])[0])
            rs.append(r)
            fcur = ref.partial_eval(fcur, [r])
            Bcur = ref.partial_eval(Bcur, [r])
            assert np.array_equal(u32(d[("round_f", rnd)]), fcur), rnd
            assert np.array_equal(u32(d[("round_basis", rnd)]), Bcur), rnd
            assert tuple(int(x) for x in u32(d[("triple", tri)])) == ref.eval_013(fcur, Bcur)
            rnd += 1
            tri += 1
        step_rounds.append(rs)
        msgs[lv + 2] = fcur
    # the last step ends at yr, opened on the last commitment
    assert np.array_equal(u32(d[("yr", steps)]), fcur)
    q = np.frombuffer(d[("queries", steps)], dtype=np.uint64)
    assert len(q) == 148 and list(q) == sorted(set(int(x) for x in q))
    # the challenges in transcript order are the oracle's
    got = list(u32(d[("fold_challenges", 0)]))
    for lv in range(steps):
        got.append(int(u32(d[("alpha", lv)])[0]))
        if lv > 0:
            got.append(int(u32(d[("beta", lv)])[0]))
        got += step_rounds[lv]
    assert got == ch


def test_dump_hook_is_cleared_and_checks_arguments(lg, ctx, golden):
    # a dump leaves the context as it was: the next plain proof gives the
    # same bytes and calls no callback; a missing callback is refused
    case = golden["cases"]["small_L12"]
    steps, m0, n0, k0, lms, lns, ks = case["config"]
    pc = lg.ProverConfig(steps, (1 << m0, 1 << n0), [(1 << m, 1 << n) for m, n in zip(lms, lns)], k0, list(ks))
    poly = lg.to_device(lg.splitmix_coeffs(case["seed"], pc.poly_len))
    dumped, d = lg.dump_intermediates(pc, poly, ctx)
    assert len(d) > 10
    assert lg.prover(pc, poly, ctx).to_bytes() == dumped.to_bytes()
    import ctypes

    h = ctypes.c_void_p()
    st = lg.lib.lg_dump_intermediates(ctx.handle, ctypes.byref(pc.to_c()), lg._dev_ptr(poly), poly.numel(), 1,
                                      ctypes.cast(None, lg._DUMP_CB), None, ctypes.byref(h))
    assert lg.STATUS[st] == "invalid argument"
