"""ctypes wrapper of the CPU oracle (oracle/_build/liblgref.so).

TEST INFRASTRUCTURE ONLY: used by tests/, by the smoke check of
__graft_entry__ and by bench.py's CPU-baseline leg.  The shipped library
never calls it.  See lgref.h for the reference file:line of every routine.
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liblgref.so"

OK, PANIC, BAD_ARG, OOM = 0, 1, 2, 3
HASH_BLAKE3, HASH_SHA256 = 0, 1
MAX_STEPS = 8


class Config(ctypes.Structure):
    _fields_ = [
        ("recursive_steps", ctypes.c_uint32),
        ("initial_log_m", ctypes.c_uint32),
        ("initial_log_n", ctypes.c_uint32),
        ("initial_k", ctypes.c_uint32),
        ("log_m", ctypes.c_uint32 * MAX_STEPS),
        ("log_n", ctypes.c_uint32 * MAX_STEPS),
        ("ks", ctypes.c_uint32 * MAX_STEPS),
    ]

    def as_tuple(self):
        s = self.recursive_steps
        return (s, self.initial_log_m, self.initial_log_n, self.initial_k,
                tuple(self.log_m[:s]), tuple(self.log_n[:s]), tuple(self.ks[:s]))


class Trace(ctypes.Structure):
    _fields_ = [
        ("roots", (ctypes.c_uint8 * 32) * (MAX_STEPS + 1)),
        ("n_roots", ctypes.c_uint32),
        ("challenges", ctypes.c_uint32 * 256),
        ("n_challenges", ctypes.c_uint32),
        ("enforced_sums", ctypes.c_uint32 * (MAX_STEPS + 1)),
        ("n_sums", ctypes.c_uint32),
    ]


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        build()
    L = ctypes.CDLL(str(LIB_PATH))
    P, u32, u64, sz, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
    sig = {
        "lgref_gf_mul": (u32, [i32, u32, u32]),
        "lgref_gf_pow": (u32, [i32, u32, u64]),
        "lgref_gf_inv": (i32, [i32, u32, P]),
        "lgref_gf128_mul": (None, [P, P, P]),
        "lgref_gf128_inv": (i32, [P, P]),
        "lgref_compute_twiddles": (None, [i32, i32, P]),
        "lgref_fft": (None, [i32, P, sz, P, i32]),
        "lgref_ifft": (None, [i32, P, sz, P]),
        "lgref_eval_sk_at_vks": (None, [i32, sz, P]),
        "lgref_evaluate_basis": (None, [i32, sz, P, u32, P]),
        "lgref_compute_pis": (None, [i32, sz, P, P]),
        "lgref_short_from_long_tw": (None, [P, i32, i32, P]),
        "lgref_rs_encode": (i32, [i32, P, sz, sz, P]),
        "lgref_rs_encode_non_systematic": (i32, [i32, P, sz, sz, i32]),
        "lgref_sha256": (None, [P, sz, P]),
        "lgref_blake3": (None, [P, sz, P]),
        "lgref_merkle_build": (i32, [i32, P, P, sz, P]),
        "lgref_merkle_prove": (i32, [P, sz, P, sz, P, sz, P]),
        "lgref_merkle_verify": (i32, [i32, P, P, sz, sz, P, P, P, sz, P]),
        "lgref_ligero_commit": (i32, [P, sz, sz, P, P, i32]),
        "lgref_ligero_verify": (i32, [P, P, sz, sz, P, sz, P, sz]),
        "lgref_lagrange_basis": (None, [P, sz, P]),
        "lgref_partial_eval": (i32, [P, sz, P, sz, P, i32]),
        "lgref_eval_013_product": (None, [P, P, sz, P]),
        "lgref_induce_sumcheck_poly": (i32, [sz, P, P, sz, sz, P, sz, P, u32, P, P, i32]),
        "lgref_quadratic_from_evals": (None, [u32, u32, u32, P]),
        "lgref_fs_new": (P, [u32]),
        "lgref_fs_free": (None, [P]),
        "lgref_fs_absorb": (None, [P, P, sz]),
        "lgref_fs_squeeze": (None, [P, P]),
        "lgref_fs_get_field32": (u32, [P]),
        "lgref_fs_get_query": (u64, [P, u64]),
        "lgref_fs_get_distinct_queries": (i32, [P, u64, sz, P]),
        "lgref_config_make": (i32, [u32, P]),
        "lgref_prove": (i32, [P, P, sz, i32, P, P]),
        "lgref_free": (None, [P]),
        "lgref_verify": (i32, [P, P, sz, i32, P]),
        "lgref_last_trace": (None, [P]),
        "lgref_set_tamper": (None, [i32]),
        "lgref_splitmix_coeffs": (None, [u64, P, sz]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


_L = None


def lib() -> ctypes.CDLL:
    global _L
    if _L is None:
        _L = load()
    return _L


def u32arr(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


# ------------------------------------------------------------ conveniences
def gf_mul(a: int, b: int, bits: int = 32) -> int:
    return int(lib().lgref_gf_mul(bits, a, b))


def config_make(log_size: int) -> Config:
    c = Config()
    assert lib().lgref_config_make(log_size, ctypes.byref(c)) == OK
    return c


def config(steps, initial_log_m, initial_log_n, log_m, log_n) -> Config:
    c = Config()
    c.recursive_steps = steps
    c.initial_log_m, c.initial_log_n, c.initial_k = initial_log_m, initial_log_n, initial_log_n
    for i in range(steps):
        c.log_m[i], c.log_n[i], c.ks[i] = log_m[i], log_n[i], log_n[i]
    return c


def splitmix(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    lib().lgref_splitmix_coeffs(seed, out.ctypes.data, n)
    return out


def twiddles(log_n: int, bits: int = 32) -> np.ndarray:
    out = np.zeros((1 << log_n) - 1, dtype=np.uint32)
    lib().lgref_compute_twiddles(bits, log_n, out.ctypes.data)
    return out


def fft(v, bits: int = 32, tw=None, nthreads: int = 1) -> np.ndarray:
    v = u32arr(v).copy()
    n = v.size
    tw = twiddles(n.bit_length() - 1, bits) if tw is None else u32arr(tw)
    lib().lgref_fft(bits, v.ctypes.data, n, tw.ctypes.data, nthreads)
    return v


def ifft(v, bits: int = 32, tw=None) -> np.ndarray:
    v = u32arr(v).copy()
    n = v.size
    tw = twiddles(n.bit_length() - 1, bits) if tw is None else u32arr(tw)
    lib().lgref_ifft(bits, v.ctypes.data, n, tw.ctypes.data)
    return v


def ligero_commit(poly, log_m: int, n: int, nthreads: int = 1):
    poly = u32arr(poly)
    rows = 4 << log_m
    flat = np.zeros(rows * n, dtype=np.uint32)
    tree = np.zeros(32 * (2 * rows - 1), dtype=np.uint8)
    st = lib().lgref_ligero_commit(poly.ctypes.data, 1 << log_m, n, flat.ctypes.data, tree.ctypes.data, nthreads)
    assert st == OK, st
    return flat, tree


def blake3(b: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().lgref_blake3(b, len(b), out)
    return out.raw


def sha256(b: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().lgref_sha256(b, len(b), out)
    return out.raw


def partial_eval(evals, rs, nthreads: int = 1) -> np.ndarray:
    e = u32arr(evals)
    r = u32arr(rs)
    out = np.zeros(e.size >> r.size, dtype=np.uint32)
    assert lib().lgref_partial_eval(e.ctypes.data, e.size, r.ctypes.data, r.size, out.ctypes.data, nthreads) == OK
    return out


def eval_013(f, g):
    f, g = u32arr(f), u32arr(g)
    out = np.zeros(3, dtype=np.uint32)
    lib().lgref_eval_013_product(f.ctypes.data, g.ctypes.data, f.size, out.ctypes.data)
    return tuple(int(x) for x in out)


def eval_sk_at_vks(n: int) -> np.ndarray:
    out = np.zeros(n.bit_length(), dtype=np.uint32)
    lib().lgref_eval_sk_at_vks(32, n, out.ctypes.data)
    return out


def induce(n: int, rows, v_ch, queries, alpha: int, nthreads: int = 1):
    rows = u32arr(rows).reshape(len(queries), -1)
    ch = u32arr(v_ch)
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.uint64))
    sk = eval_sk_at_vks(1 << n)
    out = np.zeros(1 << n, dtype=np.uint32)
    es = ctypes.c_uint32()
    st = lib().lgref_induce_sumcheck_poly(n, sk.ctypes.data, rows.ctypes.data, rows.shape[0], rows.shape[1],
                                          ch.ctypes.data, ch.size, q.ctypes.data, alpha, out.ctypes.data,
                                          ctypes.byref(es), nthreads)
    assert st == OK, st
    return out, int(es.value)


def prove(cfg: Config, poly, nthreads: int = 1) -> bytes:
    poly = u32arr(poly)
    p = ctypes.POINTER(ctypes.c_uint8)()
    n = ctypes.c_size_t()
    st = lib().lgref_prove(ctypes.byref(cfg), poly.ctypes.data, poly.size, nthreads, ctypes.byref(p), ctypes.byref(n))
    if st != OK:
        raise RuntimeError(f"lgref_prove status {st}")
    try:
        return ctypes.string_at(p, n.value)
    finally:
        lib().lgref_free(p)


def prove_tampered(cfg: Config, poly, flags: int = 1, nthreads: int = 1) -> bytes:
    """A dishonest proof for negative tests (see lgref_set_tamper)."""
    lib().lgref_set_tamper(flags)
    try:
        return prove(cfg, poly, nthreads)
    finally:
        lib().lgref_set_tamper(0)


def verify(cfg: Config, proof: bytes, nthreads: int = 1):
    """-> (status, accepted): status PANIC where the reference panics."""
    acc = ctypes.c_int()
    st = lib().lgref_verify(ctypes.byref(cfg), proof, len(proof), nthreads, ctypes.byref(acc))
    return int(st), bool(acc.value)


def last_trace() -> Trace:
    t = Trace()
    lib().lgref_last_trace(ctypes.byref(t))
    return t
