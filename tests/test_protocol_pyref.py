"""The oracle's protocol composition against an independent restatement.

tests/pyref_protocol.py restates src/prover.rs and src/verifier.rs in plain
Python (Python-integer GF(2^32), hashlib SHA-256, the blake3 module) without
sharing code with the C oracle.  Here both prove the same small inputs and
must agree on every root, challenge, opening, sumcheck triple, yr and the
proof bytes; each verifier accepts the other's proof, and both reject or
panic on the same tampered proofs.  CPU only.
"""
import hashlib

import numpy as np
import pytest

import pyref_protocol as py

# (steps, initial_log_m, initial_log_n, initial_k, log_m, log_n, ks), seed
# (every opened witness has at least 148 rows, as get_distinct_queries needs)
CASES = {
    "L11_one_step": ((1, 7, 4, 4, [6], [1], [1]), 11),
    "L12_one_step": ((1, 8, 4, 4, [6], [2], [2]), 12),
    "L12_two_steps": ((2, 9, 3, 3, [8, 6], [1, 2], [1, 2]), 13),
}


def _both(ref, spec, seed):
    steps, lm0, ln0, k0, lm, ln, ks = spec
    rcfg = ref.config(steps, lm0, ln0, lm, ln)
    poly = ref.splitmix(seed, 1 << (lm0 + ln0))
    want = ref.prove(rcfg, poly)
    trace = ref.last_trace()
    pcfg = py.Config(steps, lm0, ln0, k0, lm, ln, ks)
    P = py.prove(pcfg, [int(x) for x in poly])
    return rcfg, pcfg, poly, want, trace, P


@pytest.mark.parametrize("name", list(CASES))
def test_python_restatement_matches_oracle(ref, name):
    spec, seed = CASES[name]
    rcfg, pcfg, poly, want, trace, P = _both(ref, spec, seed)
    roots = [bytes(trace.roots[i]) for i in range(trace.n_roots)]
    assert [P["initial_root"]] + P["recursive_roots"] == roots
    assert P["challenges"] == [int(trace.challenges[i]) for i in range(trace.n_challenges)]
    got = py.serialize(P)
    assert len(got) == len(want)
    assert hashlib.sha256(got).hexdigest() == hashlib.sha256(want).hexdigest()
    # each verifier accepts the other's proof
    assert py.verify(pcfg, P) is True
    assert ref.verify(rcfg, got) == (ref.OK, True)


def _py_outcome(pcfg, P):
    try:
        return "ok", py.verify(pcfg, P)
    except (AssertionError, IndexError):
        return "panic", False


def test_tampered_proofs_same_outcome(ref):
    spec, seed = CASES["L11_one_step"]
    rcfg, pcfg, poly, want, trace, P = _both(ref, spec, seed)
    rng = np.random.default_rng(11)
    cases = []
    # a flipped opened word, Merkle sibling, yr word and each triple word
    for what in ("initial_row", "initial_sibling", "final_row", "yr", "triple0", "triple_last"):
        Q = {k: (list(v) if isinstance(v, list) else v) for k, v in P.items()}
        if what == "initial_row":
            rows, mp = P["initial"]
            rows = [list(r) for r in rows]
            rows[int(rng.integers(len(rows)))][0] ^= 1
            Q["initial"] = (rows, mp)
        elif what == "initial_sibling":
            rows, mp = P["initial"]
            mp = list(mp)
            k = int(rng.integers(len(mp)))
            mp[k] = bytes([mp[k][0] ^ 1]) + mp[k][1:]
            Q["initial"] = (rows, mp)
        elif what == "final_row":
            rows, mp = P["final"]
            rows = [list(r) for r in rows]
            rows[-1][-1] ^= 1 << 7
            Q["final"] = (rows, mp)
        elif what == "yr":
            Q["yr"] = list(P["yr"])
            Q["yr"][3] ^= 1
        else:
            tr = [tuple(t) for t in P["transcript"]]
            k = 0 if what == "triple0" else len(tr) - 1
            tr[k] = (tr[k][0], tr[k][1], tr[k][2] ^ 1)
            Q["transcript"] = tr
        cases.append((what, Q))
    # the oracle's transcript-consistent forged proof
    forged = ref.prove_tampered(rcfg, poly)
    for what, Q in cases:
        st, ok = ref.verify(rcfg, py.serialize(Q))
        theirs = ({ref.OK: "ok", ref.PANIC: "panic"}[st], ok)
        assert _py_outcome(pcfg, Q) == theirs, what
        assert theirs[1] is False, what
    assert ref.verify(rcfg, forged) == (ref.OK, False)
