"""Generate tests/golden/golden_large.json from the CPU oracle.

Full-proof digests for the generated configs too large to re-prove with the
oracle inside a GPU test run: 2^21 and 2^22 (seeds 21, 22, the seeds the
GPU tests use for those sizes), 2^24 (config_24, seed 1) and 2^28 (the
generated config, seed 2; about ten minutes on eight host cores and ~8 GB
of host memory), plus the oracle's FFT of the first 2^22-point vector of
SplitMix64 seed 1 (the 256 MiB microbench batch).  The oracle is pinned to
the reference's known-answer tests before this runs (tests/test_oracle_kats.py).

    python tests/golden/make_golden_large.py [--skip28]
"""
from __future__ import annotations

import hashlib
import json
import os
import pathlib
import sys
import time

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1] / "oracle"))
import lgref  # noqa: E402

# name -> (log size of the generated config, coefficient seed)
CASES = {"cfg21_seed21": (21, 21), "cfg22_seed22": (22, 22), "cfg24_seed1": (24, 1), "cfg28_seed2": (28, 2)}


def case_record(L, seed, threads):
    cfg = lgref.config_make(L)
    poly = lgref.splitmix(seed, 1 << L)
    t0 = time.perf_counter()
    proof = lgref.prove(cfg, poly, nthreads=threads)
    t_prove = time.perf_counter() - t0
    tr = lgref.last_trace()
    del poly
    st, ok = lgref.verify(cfg, proof, nthreads=threads)
    assert st == 0 and ok
    return {
        "log_size": L,
        "seed": seed,
        "proof_len": len(proof),
        "proof_sha256": hashlib.sha256(proof).hexdigest(),
        "roots": [bytes(tr.roots[i]).hex() for i in range(tr.n_roots)],
        "challenges": [int(tr.challenges[i]) for i in range(tr.n_challenges)],
        "enforced_sums": [int(tr.enforced_sums[i]) for i in range(tr.n_sums)],
        "oracle_prove_s": round(t_prove, 1),
        "oracle_threads": threads,
    }


def main():
    threads = os.cpu_count() or 8
    out = HERE / "golden_large.json"
    data = json.loads(out.read_text()) if out.exists() else {"cases": {}, "kernels": {}}
    v = lgref.splitmix(1, 1 << 22)
    data["kernels"]["fft22_seed1_first_sha256"] = hashlib.sha256(lgref.fft(v, nthreads=threads).tobytes()).hexdigest()
    data["kernels"]["ifft22_seed1_first_sha256"] = hashlib.sha256(lgref.ifft(v).tobytes()).hexdigest()
    for name, (L, seed) in CASES.items():
        if L == 28 and "--skip28" in sys.argv:
            continue
        data["cases"][name] = case_record(L, seed, threads)
        out.write_text(json.dumps(data, indent=1) + "\n")
        print(name, data["cases"][name]["oracle_prove_s"], "s", flush=True)
    print("wrote", out)


if __name__ == "__main__":
    main()
