"""Lockstep batches (lg_prove_lockstep): B proofs of one config through the
same kernel launches, each proof in its own slice of every buffer.  Every
proof must be byte-identical to the one the single-proof path gives for the
same coefficients (which the golden and oracle tests pin), for every input
form, group split and config shape (one and two recursive steps)."""
import hashlib

import pytest

pytestmark = pytest.mark.gpu


def _golden_cfg(lg, golden, name):
    c = golden["cases"][name]["config"]
    return lg.ProverConfig(c[0], (1 << c[1], 1 << c[2]), [(1 << m, 1 << n) for m, n in zip(c[4], c[5])], c[3],
                           list(c[6]))


def _stack(lg, ctx, cfg, seeds):
    import torch

    rows = [lg.splitmix_coeffs_device(s, cfg.poly_len, ctx) for s in seeds]
    return torch.stack(rows), rows


def _single(lg, ctx, cfg, rows):
    return [lg.prover(cfg, r, ctx).to_bytes() for r in rows]


@pytest.mark.parametrize("which,B", [("small_L12", 3), ("small_L14_two_steps", 4), (16, 5), (20, 3), (24, 2)])
def test_lockstep_equals_single_proofs(lg, ctx, golden, which, B):
    cfg = _golden_cfg(lg, golden, which) if isinstance(which, str) else lg.config_for_size(which)
    seeds = [1000 + 17 * i for i in range(B)]
    mat, rows = _stack(lg, ctx, cfg, seeds)
    got = [p.to_bytes() for p in lg.prove_lockstep(cfg, mat, ctx)]
    assert got == _single(lg, ctx, cfg, rows)
    assert all(lg.verifier(cfg, b, ctx) for b in got[:2])


def test_lockstep_golden_digest(lg, ctx, golden):
    # the golden config-20 proof (seed 0) as member 1 of a batch of 3
    cfg = lg.hardcoded_config_20()
    mat, _ = _stack(lg, ctx, cfg, [7, 0, 9])
    b = lg.prove_lockstep(cfg, mat, ctx)[1].to_bytes()
    assert hashlib.sha256(b).hexdigest() == golden["cases"]["cfg20_seed0"]["proof_sha256"]


def test_lockstep_input_forms(lg, ctx, golden):
    # contiguous device rows (read in place), separate device tensors
    # (gathered first) and host arrays give the same proofs
    cfg = _golden_cfg(lg, golden, "small_L12")
    seeds = [5, 6, 7, 8]
    mat, rows = _stack(lg, ctx, cfg, seeds)
    a = [p.to_bytes() for p in lg.prove_lockstep(cfg, mat, ctx)]
    b = [p.to_bytes() for p in lg.prove_lockstep(cfg, rows[::-1], ctx)][::-1]
    c = [p.to_bytes() for p in lg.prove_lockstep(cfg, [lg.to_host(r) for r in rows], ctx)]
    assert a == b == c == _single(lg, ctx, cfg, rows)


def test_lockstep_groups_of_64(lg, ctx, golden):
    # 70 proofs: a full group of 64 (the launch limit) and a group of 6
    cfg = _golden_cfg(lg, golden, "small_L12")
    seeds = [3 * i + 1 for i in range(70)]
    mat, rows = _stack(lg, ctx, cfg, seeds)
    got = [p.to_bytes() for p in lg.prove_lockstep(cfg, mat, ctx)]
    want = _single(lg, ctx, cfg, [rows[i] for i in (0, 31, 63, 64, 69)])
    assert [got[i] for i in (0, 31, 63, 64, 69)] == want
    assert len(set(got)) == 70


def test_lockstep_reports_like_single_prover(lg, ctx):
    # a last commitment of 64 rows cannot give 148 distinct queries (the
    # reference would loop in get_distinct_queries): both paths refuse the
    # config with the same status before any work
    cfg = lg.ProverConfig(1, (1 << 8, 1 << 4), [(1 << 4, 1 << 4)], 4, [4])
    mat, rows = _stack(lg, ctx, cfg, [1, 2])
    with pytest.raises(lg.LigeritoError) as e1:
        lg.prover(cfg, rows[0], ctx)
    with pytest.raises(lg.LigeritoError) as e2:
        lg.prove_lockstep(cfg, mat, ctx)
    assert e1.value.status == e2.value.status == 2
    # a wrong length is refused too
    good = lg.config_for_size(16)
    with pytest.raises(lg.LigeritoError):
        lg.prove_lockstep(good, mat, ctx)
    # the context still proves afterwards
    m2, r2 = _stack(lg, ctx, good, [11, 12])
    assert [p.to_bytes() for p in lg.prove_lockstep(good, m2, ctx)] == _single(lg, ctx, good, r2)


def test_lockstep_64_large_group(lg, ctx):
    # 64 proofs at 2^20: the openings outgrow the context's pinned arena
    # (about 9 MiB for the first opening alone), so the call spills to
    # extra pinned blocks; members still equal their single proofs
    cfg = lg.config_for_size(20)
    mat, rows = _stack(lg, ctx, cfg, [5000 + i for i in range(64)])
    got = lg.prove_lockstep(cfg, mat, ctx)
    pick = (0, 17, 63)
    assert [got[i].to_bytes() for i in pick] == _single(lg, ctx, cfg, [rows[i] for i in pick])
    # and again: the next call starts with an arena of the size this one used
    got2 = lg.prove_lockstep(cfg, mat, ctx)
    assert [got2[i].to_bytes() for i in pick] == [got[i].to_bytes() for i in pick]
