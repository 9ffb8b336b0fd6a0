"""Kernel-level parity on the GPU, through the C ABI, against the oracle.
All results must be bit-identical (GF(2^32) and BLAKE3 are exact)."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
rng = np.random.default_rng(7)


def rand_u32(n):
    return rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("log_n,batch", [(1, 3), (2, 5), (3, 1), (5, 7), (6, 3), (7, 2), (10, 4), (12, 3),
                                         (13, 2), (16, 2), (8, 100), (10, 130), (4, 70)])
def test_fft_ifft_match_oracle(lg, ref, ctx, log_n, batch):
    # fft / ifft, src/binary_fft.rs:4-28, every vector of a batch
    v = rand_u32(batch << log_n).reshape(batch, -1)
    d = lg.to_device(v.ravel())
    lg.fft(d, log_n, ctx)
    got = lg.to_host(d).reshape(batch, -1)
    tw = ref.twiddles(log_n)
    for i in range(batch):
        assert (got[i] == ref.fft(v[i], tw=tw)).all()
    lg.ifft(d, log_n, ctx)
    assert (lg.to_host(d).reshape(batch, -1) == v).all()
    inv = np.stack([ref.ifft(v[i], tw=tw) for i in range(batch)])
    d2 = lg.to_device(v.ravel())
    lg.ifft(d2, log_n, ctx)
    assert (lg.to_host(d2).reshape(batch, -1) == inv).all()


def test_fft_zero_and_constant_vectors(lg, ref, ctx):
    for v in (np.zeros(1 << 9, np.uint32), np.full(1 << 9, 0xFFFFFFFF, np.uint32)):
        d = lg.to_device(v)
        lg.fft(d, 9, ctx)
        assert (lg.to_host(d) == ref.fft(v)).all()


@pytest.mark.parametrize("log_n,batch", [(16, 1024), (20, 64), (22, 16)])
def test_fft_microbench_sizes_roundtrip(lg, ref, ctx, golden_large, log_n, batch):
    # the 256 MiB batched transforms of the fft/ifft microbench: ifft(fft(v))
    # == v everywhere, one vector checked against the oracle, and the
    # transform is linear (fft(a ^ b) == fft(a) ^ fft(b)) on a sample
    import torch

    d = lg.splitmix_coeffs_device(1, batch << log_n, ctx)
    keep = d.clone()
    lg.fft(d, log_n, ctx)
    if log_n <= 20:
        col = lg.to_host(keep[:1 << log_n])
        assert (lg.to_host(d[:1 << log_n]) == ref.fft(col)).all()
    else:  # the oracle's transform of the first vector, committed as a digest
        k = golden_large["kernels"]
        assert hashlib.sha256(lg.to_host(d[:1 << log_n]).tobytes()).hexdigest() == k["fft22_seed1_first_sha256"]
        first = keep[:1 << log_n].clone()
        lg.ifft(first, log_n, ctx)
        assert hashlib.sha256(lg.to_host(first).tobytes()).hexdigest() == k["ifft22_seed1_first_sha256"]
    a, b = keep[: 2 << log_n].clone(), lg.splitmix_coeffs_device(9, 2 << log_n, ctx)
    ab = torch.bitwise_xor(a, b)
    for t in (a, b, ab):
        lg.fft(t, log_n, ctx)
    assert torch.equal(torch.bitwise_xor(a, b), ab)
    lg.ifft(d, log_n, ctx)
    assert torch.equal(d, keep)


@pytest.mark.parametrize("log_m,n", [(6, 1), (6, 4), (6, 16), (8, 64), (10, 16), (11, 3), (12, 64), (14, 16), (7, 40), (9, 100)])
def test_encode_and_commit_match_oracle(lg, ref, ctx, log_m, n):
    # encode_cols + extract_leaves + build_merkle_tree (src/ligero.rs:11-95)
    poly = rand_u32(n << log_m)
    enc = lg.encode_cols(lg.to_device(poly), log_m, n, ctx)
    flat, tree = ref.ligero_commit(poly, log_m, n, nthreads=8)
    assert (lg.to_host(enc) == flat).all()
    enc2, tree2, root = lg.ligero_commit(lg.to_device(poly), log_m, n, ctx)
    assert (lg.to_host(enc2) == flat).all()
    assert (lg.to_host(tree2).view(np.uint8) == tree).all()
    assert root == bytes(tree[-32:])


def test_commit_golden(lg, ctx, golden):
    k = golden["kernels"]
    poly = lg.splitmix_coeffs(4, 64 * 64)
    enc, tree, root = lg.ligero_commit(lg.to_device(poly), 6, 64, ctx)
    assert root.hex() == k["commit_m64_n64_seed4_root"]
    assert hashlib.sha256(lg.to_host(enc).tobytes()).hexdigest() == k["commit_m64_n64_seed4_flat_sha256"]
    d = lg.to_device(lg.splitmix_coeffs(3, 256))
    lg.fft(d, 8, ctx)
    assert hashlib.sha256(lg.to_host(d).tobytes()).hexdigest() == k["fft256_seed3_sha256"]


def test_commit_full_size_rows_open_consistently(lg, ref, ctx):
    # 2^18 x 64 first-round matrix of config 24: spot rows against the
    # oracle's RS encoding of the same column (column-independent), and the
    # root is reproducible
    import torch

    log_m, n = 18, 64
    poly = lg.splitmix_coeffs_device(1, n << log_m, ctx)
    enc, tree, root = lg.ligero_commit(poly, log_m, n, ctx)
    enc_b, tree_b, root_b = lg.ligero_commit(poly, log_m, n, ctx)
    assert root == root_b and torch.equal(tree, tree_b)
    col = lg.to_host(poly[: 1 << log_m])
    v = np.zeros(4 << log_m, np.uint32)
    v[: 1 << log_m] = col
    assert ref.lib().lgref_rs_encode_non_systematic(32, v.ctypes.data, 1 << log_m, 4 << log_m, 8) == 0
    assert (lg.to_host(enc[: 4 << log_m]) == v).all()


@pytest.mark.parametrize("log_len,k", [(14, 6), (10, 1), (12, 4), (16, 9), (8, 8), (20, 6), (6, 1)])
def test_partial_eval_matches_oracle(lg, ref, ctx, log_len, k):
    # MultiLinearPoly::partial_eval (src/multilinear_poly.rs:66-87)
    e, rs = rand_u32(1 << log_len), rand_u32(k)
    got = lg.to_host(lg.partial_eval(lg.to_device(e), rs, ctx))
    assert (got == ref.partial_eval(e, rs, nthreads=8)).all()


@pytest.mark.parametrize("log_len", [1, 2, 5, 12, 18])
def test_eval013_matches_oracle(lg, ref, ctx, log_len):
    # eval_013_product (src/multilinear_poly.rs:90-131)
    f, g = rand_u32(1 << log_len), rand_u32(1 << log_len)
    assert lg.eval_013_product(lg.to_device(f), lg.to_device(g), ctx) == ref.eval_013(f, g)


@pytest.mark.parametrize("n,nch", [(10, 6), (14, 4), (6, 2), (18, 6), (8, 4), (12, 1)])
def test_induce_matches_oracle(lg, ref, ctx, n, nch):
    # induce_sumcheck_poly_parallel (src/sumcheck_polys.rs:74-160)
    rows = rand_u32(148 << nch).reshape(148, -1)
    q = np.sort(rng.choice(4 << n, size=148, replace=False)).astype(np.uint64)
    ch = rand_u32(nch)
    alpha = int(rng.integers(0, 2**32))
    b, es = lg.induce_sumcheck_poly(n, rows, ch, q, alpha, ctx)
    b2, es2 = ref.induce(n, rows, ch, q, alpha, nthreads=8)
    assert es == es2
    assert (lg.to_host(b) == b2).all()


def test_induce_edge_queries(lg, ref, ctx):
    # query 0 and the largest row index, alpha 0 and 1
    n, nch = 8, 2
    rows = rand_u32(148 << nch).reshape(148, -1)
    q = np.arange(4 << n, dtype=np.uint64)[-148:]
    q[0] = 0
    q = np.sort(q)
    for alpha in (0, 1):
        b, es = lg.induce_sumcheck_poly(n, rows, rand_u32(nch) * 0 + 5, q, alpha, ctx)
        b2, es2 = ref.induce(n, rows, np.full(nch, 5, np.uint32), q, alpha)
        assert es == es2 and (lg.to_host(b) == b2).all()


def test_device_splitmix_matches_host(lg, ctx):
    assert (lg.to_host(lg.splitmix_coeffs_device(77, 100003, ctx)) == lg.splitmix_coeffs(77, 100003)).all()


def test_bad_arguments_return_status(lg, ctx):
    import ctypes

    with pytest.raises(lg.LigeritoError):
        lg.fft(lg.to_device(np.zeros(8, np.uint32)), 0, ctx)
    assert lg.lib.lg_fft(ctx.handle, None, 4, 1) == 1
    assert lg.lib.lg_partial_eval(ctx.handle, None, 4, None, 1, None) == 1


def test_gf128_mul_matches_oracle(lg, ref, ctx):
    # BinaryElem128 (src/binary_field.rs:182-189): device products against
    # the oracle's on random pairs, edge values and a ragged count
    import ctypes

    import torch

    n = 4099
    r = np.random.default_rng(128)
    a = r.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)
    b = r.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)
    top = np.iinfo(np.uint64).max
    edges = [(0, 0), (1, 0), (top, top), (0, 1 << 63), (1 << 63, 0), (0, 1), (0x87, 0), (2, 0)]
    for i, e in enumerate(edges):
        for j, f in enumerate(edges):
            a[i * len(edges) + j] = e
            b[i * len(edges) + j] = f
    dev = lambda x: torch.from_numpy(x.view(np.int64)).cuda()  # noqa: E731
    got = lg.gf128_mul(dev(a), dev(b), ctx).cpu().numpy().view(np.uint64)
    A, B, O = (ctypes.c_uint64 * 2)(), (ctypes.c_uint64 * 2)(), (ctypes.c_uint64 * 2)()
    for i in range(n):
        A[0], A[1], B[0], B[1] = int(a[i, 0]), int(a[i, 1]), int(b[i, 0]), int(b[i, 1])
        ref.lib().lgref_gf128_mul(A, B, O)
        assert (int(got[i, 0]), int(got[i, 1])) == (O[0], O[1]), i
    # no elements; misaligned arrays are refused
    z = torch.zeros((0, 2), dtype=torch.int64, device="cuda")
    assert lg.gf128_mul(z, z, ctx).shape == (0, 2)
    t = torch.zeros(9, dtype=torch.int64, device="cuda")
    assert lg.lib.lg_gf128_mul(ctx.handle, t.data_ptr() + 8, t.data_ptr(), t.data_ptr(), 1) == 1
