"""Generate tests/golden/golden.json from the CPU oracle.

The reference crate (Rust) cannot be built in this environment, so the
fixtures are produced by the oracle after it has replayed every
known-answer test of the reference (twiddles, Merkle root / multi-proofs)
and cross-checked SHA-256 / BLAKE3 against Python's hashlib / blake3.
They pin the oracle against regressions and give the GPU tests full-proof
digests without re-running the oracle at the larger sizes.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "oracle"))
import lgref  # noqa: E402

# name -> (config constructor args, coefficient seed)
CASES = {
    "small_L12": ("custom", (1, 8, 4, [6], [2]), 12),
    "small_L14_two_steps": ("custom", (2, 10, 4, [8, 6], [2, 2]), 14),
    "cfg16_seed16": ("make", 16, 16),
    "cfg20_seed0": ("make", 20, 0),
}


def make_cfg(kind, arg):
    if kind == "make":
        return lgref.config_make(arg)
    return lgref.config(*arg)


def case_record(kind, arg, seed):
    cfg = make_cfg(kind, arg)
    n = 1 << (cfg.initial_log_m + cfg.initial_log_n)
    poly = lgref.splitmix(seed, n)
    proof = lgref.prove(cfg, poly, nthreads=8)
    tr = lgref.last_trace()
    st, ok = lgref.verify(cfg, proof, nthreads=8)
    assert st == 0 and ok
    return {
        "config": list(cfg.as_tuple()[:4]) + [list(x) for x in cfg.as_tuple()[4:]],
        "seed": seed,
        "poly_sha256": hashlib.sha256(poly.tobytes()).hexdigest(),
        "proof_len": len(proof),
        "proof_sha256": hashlib.sha256(proof).hexdigest(),
        "roots": [bytes(tr.roots[i]).hex() for i in range(tr.n_roots)],
        "challenges": [int(tr.challenges[i]) for i in range(tr.n_challenges)],
        "enforced_sums": [int(tr.enforced_sums[i]) for i in range(tr.n_sums)],
        "proof_head_hex": proof[:64].hex(),
    }


def kernel_vectors():
    out = {}
    # 2^8-point GF(2^32) FFT of splitmix(3) and its twiddles (prefix)
    v = lgref.splitmix(3, 256)
    out["fft256_seed3_sha256"] = hashlib.sha256(lgref.fft(v).tobytes()).hexdigest()
    out["twiddles32_log8_head"] = [int(x) for x in lgref.twiddles(8)[:16]]
    flat, tree = lgref.ligero_commit(lgref.splitmix(4, 64 * 64), 6, 64)
    out["commit_m64_n64_seed4_root"] = bytes(tree[-32:]).hex()
    out["commit_m64_n64_seed4_flat_sha256"] = hashlib.sha256(flat.tobytes()).hexdigest()
    return out


def main():
    data = {"cases": {}, "kernels": kernel_vectors()}
    for name, (kind, arg, seed) in CASES.items():
        data["cases"][name] = case_record(kind, arg, seed)
    (HERE / "golden.json").write_text(json.dumps(data, indent=1) + "\n")
    print("wrote", HERE / "golden.json")


if __name__ == "__main__":
    main()
