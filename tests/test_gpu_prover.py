"""End-to-end parity on the GPU: proofs from liblgpu are byte-identical to
the oracle's for the same config and coefficients, both verifiers accept
them, and both reject / panic on the same corrupted proofs."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfgs(lg, ref, case):
    c = case["config"]
    pc = lg.ProverConfig(c[0], (1 << c[1], 1 << c[2]), [(1 << m, 1 << n) for m, n in zip(c[4], c[5])], c[3],
                         list(c[6]))
    return pc, ref.config(c[0], c[1], c[2], c[4], c[5])


@pytest.mark.parametrize("name", ["small_L12", "small_L14_two_steps", "cfg16_seed16", "cfg20_seed0"])
def test_proof_matches_golden_and_oracle(lg, ref, ctx, golden, name):
    case = golden["cases"][name]
    pc, rc = _cfgs(lg, ref, case)
    poly = lg.splitmix_coeffs(case["seed"], pc.poly_len)
    proof = lg.prover(pc, lg.to_device(poly), ctx)
    b = proof.to_bytes()
    assert len(b) == case["proof_len"]
    assert hashlib.sha256(b).hexdigest() == case["proof_sha256"]
    f = proof.fields()
    assert [f.initial_root.hex()] + [r.hex() for r in f.recursive_roots] == case["roots"]
    assert ref.verify(rc, b, nthreads=8) == (ref.OK, True)
    assert lg.verifier(pc, proof, ctx) is True
    if pc.poly_len <= 1 << 16:
        assert b == ref.prove(rc, poly, nthreads=8)


def test_config20_host_input_equals_device_input(lg, ctx, golden):
    # the reference's own workload (src/main.rs:22-53) through the host path
    cfg = lg.hardcoded_config_20()
    poly = lg.splitmix_coeffs(0, 1 << 20)
    a = lg.prover(cfg, poly, ctx).to_bytes()
    b = lg.prover(cfg, lg.to_device(poly), ctx).to_bytes()
    assert a == b
    assert hashlib.sha256(a).hexdigest() == golden["cases"]["cfg20_seed0"]["proof_sha256"]
    assert lg.verifier(lg.hardcoded_config_20_verifier(), a, ctx)


@pytest.mark.parametrize("k", [2, 4, 5, 7])
def test_host_input_column_groups_match_oracle(lg, ref, ctx, k):
    # The host-input commitment copies and encodes 16-column groups and
    # hashes them in pairs: 4 columns (one partial group and BLAKE3 block),
    # 16 (one group), 32 (one pair), 128 (four pairs).
    pc = lg.ProverConfig(1, (1 << 10, 1 << k), [(1 << 6, 1 << 4)], k, [4])
    rc = ref.config(1, 10, k, [6], [4])
    poly = lg.splitmix_coeffs(100 + k, pc.poly_len)
    a = lg.prover(pc, poly, ctx).to_bytes()
    b = lg.prover(pc, lg.to_device(poly), ctx).to_bytes()
    assert a == b == ref.prove(rc, poly, nthreads=8)


def test_large_last_commitment_matches_oracle(lg, ref, ctx):
    # The last opening normally reads host copies of the last commitment,
    # fetched during the last rounds; this one (2^16 rows x 16 columns, 8 MB
    # with its tree) is over that limit and is gathered on the device.
    import os

    pc = lg.ProverConfig(1, (1 << 18, 1 << 2), [(1 << 14, 1 << 4)], 2, [4])
    rc = ref.config(1, 18, 2, [14], [4])
    poly = lg.splitmix_coeffs(7, pc.poly_len)
    got = lg.prover(pc, lg.to_device(poly), ctx).to_bytes()
    assert got == ref.prove(rc, poly, nthreads=os.cpu_count() or 8)
    assert lg.verifier(pc, got, ctx)


def test_pinned_and_pageable_host_inputs_give_the_same_proof(lg, ctx):
    # the host paths overlap the input copy with the first commitment
    import torch

    cfg = lg.hardcoded_config_24()
    poly = lg.splitmix_coeffs(1, 1 << 24)
    pinned = torch.empty(1 << 24, dtype=torch.int32, pin_memory=True)
    pinned.copy_(torch.from_numpy(poly.view(np.int32)))
    a = lg.prover(cfg, pinned.numpy().view(np.uint32), ctx).to_bytes()
    b = lg.prover(cfg, poly, ctx).to_bytes()
    c = lg.prover(cfg, lg.to_device(poly), ctx).to_bytes()
    assert a == b == c


def test_config24_matches_oracle(lg, ref, ctx):
    # config 24 (src/config.rs:69-134), seed 1: byte-identical to the oracle
    import os

    cfg = lg.hardcoded_config_24()
    poly = lg.splitmix_coeffs(1, 1 << 24)
    got = lg.prover(cfg, lg.to_device(poly), ctx).to_bytes()
    want = ref.prove(ref.config_make(24), poly, nthreads=os.cpu_count() or 8)
    assert got == want
    assert ref.verify(ref.config_make(24), got, nthreads=os.cpu_count() or 8) == (ref.OK, True)
    assert lg.verifier(cfg, got, ctx)


@pytest.mark.parametrize("L", [17, 18, 19, 21, 22])
def test_generated_configs_match_oracle(lg, ref, ctx, golden_large, L):
    # generated configs (the config.rs pattern extended): byte-identical to
    # the oracle's proof -- re-proved here up to 2^19, against the oracle's
    # committed digest (tests/golden/make_golden_large.py) above
    cfg = lg.config_for_size(L)
    poly = lg.splitmix_coeffs_device(L, cfg.poly_len, ctx)
    proof = lg.prover(cfg, poly, ctx)
    assert lg.verifier(cfg, proof, ctx)
    b = proof.to_bytes()
    assert ref.verify(ref.config_make(L), b, nthreads=8) == (ref.OK, True)
    if L <= 19:
        assert b == ref.prove(ref.config_make(L), lg.to_host(poly), nthreads=8)
    else:
        case = golden_large["cases"][f"cfg{L}_seed{L}"]
        assert len(b) == case["proof_len"]
        assert hashlib.sha256(b).hexdigest() == case["proof_sha256"]
        f = proof.fields()
        assert [f.initial_root.hex()] + [r.hex() for r in f.recursive_roots] == case["roots"]


def test_config24_matches_golden_digest(lg, ctx, golden_large):
    cfg = lg.hardcoded_config_24()
    b = lg.prover(cfg, lg.splitmix_coeffs_device(1, 1 << 24, ctx), ctx).to_bytes()
    assert hashlib.sha256(b).hexdigest() == golden_large["cases"]["cfg24_seed1"]["proof_sha256"]


def test_config28_matches_oracle_digest(lg, ref, ctx, golden_large):
    # 2^28 coefficients (1 GiB input, 4 GiB first encoded matrix, seed 2,
    # the generated config): byte-identical to the oracle's proof (its
    # digest, roots and challenges, committed), accepted by both verifiers
    import os

    case = golden_large["cases"]["cfg28_seed2"]
    cfg = lg.config_for_size(28)
    poly = lg.splitmix_coeffs_device(2, cfg.poly_len, ctx)
    proof = lg.prover(cfg, poly, ctx)
    del poly
    b = proof.to_bytes()
    f = proof.fields()
    assert [f.initial_root.hex()] + [r.hex() for r in f.recursive_roots] == case["roots"]
    assert len(b) == case["proof_len"]
    assert hashlib.sha256(b).hexdigest() == case["proof_sha256"]
    assert lg.verifier(cfg, proof, ctx)
    assert ref.verify(ref.config_make(28), b, nthreads=os.cpu_count() or 8) == (ref.OK, True)


def test_proving_is_deterministic(lg, ctx):
    cfg = lg.config_for_size(18)
    poly = lg.splitmix_coeffs_device(5, cfg.poly_len, ctx)
    assert lg.prover(cfg, poly, ctx).to_bytes() == lg.prover(cfg, poly, ctx).to_bytes()


def test_edge_coefficients(lg, ref, ctx):
    # all-zero and all-ones polynomials at a small config
    pc = lg.ProverConfig(1, (256, 16), [(64, 4)], 4, [2])
    rc = ref.config(1, 8, 4, [6], [2])
    for poly in (np.zeros(1 << 12, np.uint32), np.full(1 << 12, 0xFFFFFFFF, np.uint32)):
        b = lg.prover(pc, lg.to_device(poly), ctx).to_bytes()
        assert b == ref.prove(rc, poly)
        assert lg.verifier(pc, b, ctx)


def _both_verify(lg, ref, pc, rc, b, ctx):
    st, ok = ref.verify(rc, b)
    try:
        mine = ("ok", lg.verifier(pc, b, ctx))
    except lg.LigeritoPanic:
        mine = ("panic", False)
    except lg.LigeritoError as e:
        mine = ("malformed" if e.status == 8 else "error", False)
    theirs = {ref.OK: "ok", ref.PANIC: "panic", ref.BAD_ARG: "malformed"}[st], ok
    return mine, theirs


def test_verifiers_agree_on_corrupted_proofs(lg, ref, ctx):
    pc = lg.ProverConfig(1, (256, 16), [(64, 4)], 4, [2])
    rc = ref.config(1, 8, 4, [6], [2])
    poly = lg.splitmix_coeffs(12, 1 << 12)
    b = lg.prover(pc, lg.to_device(poly), ctx).to_bytes()
    rng = np.random.default_rng(3)
    positions = [16, 40, 60, 100, len(b) // 2, len(b) - 200, len(b) - 20, len(b) - 5, len(b) - 1]
    positions += [int(x) for x in rng.integers(12, len(b), size=20)]
    for pos in positions:
        bad = bytearray(b)
        bad[pos] ^= 1 << int(rng.integers(0, 8))
        mine, theirs = _both_verify(lg, ref, pc, rc, bytes(bad), ctx)
        assert mine == theirs, (pos, mine, theirs)
        assert mine[1] is False
    # a transcript-consistent dishonest proof is rejected without a panic
    forged = ref.prove_tampered(rc, poly)
    assert _both_verify(lg, ref, pc, rc, forged, ctx) == (("ok", False), ("ok", False))
    # truncated
    assert _both_verify(lg, ref, pc, rc, b[:-7], ctx)[0][0] == "malformed"


def test_wrong_config_is_reported(lg, ctx):
    cfg = lg.hardcoded_config_20()
    with pytest.raises(lg.LigeritoError) as e:
        lg.prover(cfg, lg.splitmix_coeffs(0, 1 << 16), ctx)
    assert e.value.status == 2


def test_hbm_budget_reports_oom_and_context_survives(lg, ctx):
    small = lg.Context(0, hbm_budget_bytes=1 << 20)
    cfg = lg.config_for_size(18)
    poly = lg.splitmix_coeffs(1, cfg.poly_len)
    with pytest.raises(lg.LigeritoError) as e:
        lg.prover(cfg, poly, small)
    assert e.value.status == 3
    assert small.device_bytes_in_use == 0
    small.close()
    # the shared context still proves afterwards
    assert lg.verifier(cfg, lg.prover(cfg, poly, ctx), ctx)


def test_launch_count_and_timing(lg, ctx):
    cfg = lg.config_for_size(16)
    poly = lg.splitmix_coeffs_device(2, cfg.poly_len, ctx)
    before = ctx.launch_count
    ctx.set_kernel_timing(True)
    ctx.reset_kernel_stats()
    lg.prover(cfg, poly, ctx)
    stats = ctx.kernel_stats()
    ctx.set_kernel_timing(False)
    assert ctx.launch_count - before == sum(n for n, _ in stats.values())
    assert {"leaf_hash", "fold_round", "induce_main", "fs_queries"} <= set(stats)
    assert any(k.startswith("merkle_") for k in stats)
    assert any(k.startswith("fft_pass_L") for k in stats)


# Witnesses of 512 and 1024 rows opened by the device transcript: 148
# distinct queries among 512 rows take the most squeezes and sometimes a
# second batch (the batch is sized by the repeats expected).
SMALL_ROWS = {
    "initial512": (1, 7, 2, [6], [1]),
    "step512": (2, 9, 2, [7, 6], [2, 1]),
    "steps1024_512": (3, 9, 1, [8, 7, 6], [1, 1, 1]),
}


@pytest.mark.parametrize("name", list(SMALL_ROWS))
def test_small_row_openings_match_oracle(lg, ref, ctx, name):
    steps, lm0, ln0, lm, ln = SMALL_ROWS[name]
    pc = lg.ProverConfig(steps, (1 << lm0, 1 << ln0), [(1 << m, 1 << n) for m, n in zip(lm, ln)], ln0, list(ln))
    rc = ref.config(steps, lm0, ln0, lm, ln)
    for seed in range(6):
        poly = lg.splitmix_coeffs(700 + seed, pc.poly_len)
        assert lg.prover(pc, lg.to_device(poly), ctx).to_bytes() == ref.prove(rc, poly, nthreads=4), seed
