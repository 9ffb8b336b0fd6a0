"""Host-side mirror of the Ligerito prover/verifier API of
ashutosh1206/ligerito-rust over liblgpu.so (CUDA, sm_100a).

Names and argument meanings follow the reference crate:

* ``hardcoded_config_20`` / ``hardcoded_config_24`` (+ ``_verifier``)
  -- src/config.rs:6-134
* ``prover(config, poly)`` -- src/prover.rs:15
* ``verifier(config, proof)`` -- src/verifier.rs:10; returns the reference's
  bool and raises :class:`LigeritoPanic` where the reference panics.
* kernel-level functions (``fft``, ``ifft``, ``compute_twiddles``,
  ``encode_cols``, ``ligero_commit``, ``partial_eval``,
  ``eval_013_product``, ``induce_sumcheck_poly``) -- src/binary_fft.rs,
  src/reed_solomon.rs, src/ligero.rs, src/multilinear_poly.rs,
  src/sumcheck_polys.rs.

Field elements are GF(2^32) values held as ``uint32`` (numpy on the host,
``torch.int32`` tensors on the device, same bits).  Every device call goes
through the C ABI in ``include/ligerito_b200.h``; there is no CPU fallback:
importing this package fails when liblgpu.so has not been built.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "_build" / "liblgpu.so"

LG_MAX_STEPS = 8
NUM_QUERIES = 148
FS_SEED = 1234

STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "invalid config",
    3: "out of memory",
    4: "CUDA error",
    5: "verifier panic",
    6: "prover assertion failed",
    7: "no CUDA device",
    8: "malformed proof",
    9: "sizes exceed the fixed scratch of an allocation-free call",
    10: "timed out",
}


class LigeritoError(RuntimeError):
    """A liblgpu call returned a non-OK status."""

    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}{': ' + msg if msg else ''}")


class LigeritoPanic(LigeritoError, AssertionError):
    """The reference implementation would have panicked here (assert / index)."""


class LgConfig(ctypes.Structure):
    _fields_ = [
        ("recursive_steps", ctypes.c_uint32),
        ("initial_log_m", ctypes.c_uint32),
        ("initial_log_n", ctypes.c_uint32),
        ("initial_k", ctypes.c_uint32),
        ("log_m", ctypes.c_uint32 * LG_MAX_STEPS),
        ("log_n", ctypes.c_uint32 * LG_MAX_STEPS),
        ("ks", ctypes.c_uint32 * LG_MAX_STEPS),
    ]


# lg_dump_cb: (user, name, level, data, bytes)
_DUMP_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_void_p,
                            ctypes.c_uint64)


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it first (python -c 'import __graft_entry__ as g; g.build()')"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.c_void_p
    u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    sigs = {
        "lg_status_string": (ctypes.c_char_p, [i32]),
        "lg_abi_version": (u32, []),
        "lg_hardcoded_config_20": (i32, [P]),
        "lg_hardcoded_config_24": (i32, [P]),
        "lg_config_make": (i32, [u32, P]),
        "lg_config_validate": (i32, [P, u64]),
        "lg_ctx_create": (i32, [i32, u64, P]),
        "lg_ctx_destroy": (None, [P]),
        "lg_ctx_last_error": (ctypes.c_char_p, [P]),
        "lg_ctx_stream": (P, [P]),
        "lg_ctx_synchronize": (i32, [P]),
        "lg_ctx_launch_count": (u64, [P]),
        "lg_ctx_set_kernel_timing": (i32, [P, i32]),
        "lg_ctx_kernel_stats": (i32, [P, u32, ctypes.c_char_p, ctypes.c_size_t, P, P]),
        "lg_ctx_reset_kernel_stats": (i32, [P]),
        "lg_ctx_kernel_work": (i32, [P, u32, P, P, P]),
        "lg_ctx_set_autotune": (i32, [P, i32]),
        "lg_tuned_choices": (i32, [P, P]),
        "lg_measure_pipe_peaks": (i32, [i32, P, u32]),
        "lg_ctx_device_bytes_in_use": (u64, [P]),
        "lg_ctx_device_bytes_cached": (u64, [P]),
        "lg_device_table_bytes": (u64, [i32]),
        "lg_server_warm": (i32, [P, P, u32]),
        "lg_prove": (i32, [P, P, P, u64, i32, P]),
        "lg_dump_intermediates": (i32, [P, P, P, u64, i32, _DUMP_CB, P, P]),
        "lg_verify": (i32, [P, P, P, P]),
        "lg_verify_bytes": (i32, [P, P, ctypes.c_char_p, u64, P]),
        "lg_proof_serialize": (i32, [P, P, P]),
        "lg_proof_deserialize": (i32, [P, u64, P]),
        "lg_proof_free": (None, [P]),
        "lg_proof_size": (i32, [P, P]),
        "lg_compute_twiddles": (i32, [u32, P]),
        "lg_fft": (i32, [P, P, u32, u64]),
        "lg_config_parse": (i32, [ctypes.c_char_p, P]),
        "lg_config_format": (i32, [P, P, P]),
        "lg_gf128_mul": (i32, [P, P, P, P, u64]),
        "lg_ifft": (i32, [P, P, u32, u64]),
        "lg_rs_encode_cols": (i32, [P, P, u32, u32, P]),
        "lg_ligero_commit": (i32, [P, P, u32, u32, P, P, P]),
        "lg_partial_eval": (i32, [P, P, u32, P, u32, P]),
        "lg_eval_013_product": (i32, [P, P, P, u32, P]),
        "lg_induce_sumcheck_poly": (i32, [P, u32, P, u32, P, u32, P, u32, P, P]),
        "lg_fill_splitmix": (i32, [P, u64, P, u64]),
        "lg_transcript_new": (i32, [u32, P]),
        "lg_transcript_free": (None, [P]),
        "lg_transcript_absorb": (i32, [P, P, u64]),
        "lg_transcript_squeeze": (i32, [P, P]),
        "lg_transcript_get_field": (i32, [P, P]),
        "lg_transcript_get_query": (i32, [P, u64, P]),
        "lg_transcript_get_distinct_queries": (i32, [P, u64, u64, P]),
        "lg_merkle_verify": (i32, [P, P, u64, u64, P, P, P, u64, P]),
        "lg_fill_splitmix_host": (None, [u64, P, u64]),
        "lg_induce_sumcheck_poly_noalloc": (i32, [P, u32, P, u32, P, u32, P, u32, P, P]),
        "lg_server_create": (i32, [i32, u64, u32, P]),
        "lg_server_set_max_batch": (i32, [P, u32]),
        "lg_server_submit": (i32, [P, P, P, u64, i32, i32, P]),
        "lg_server_wait": (i32, [P, u64, ctypes.c_int64, P, P, P]),
        "lg_server_stats": (i32, [P, P, P, P]),
        "lg_server_destroy": (None, [P]),
        "lg_prove_batch": (i32, [i32, u32, P, P, P, i32, u32, P]),
        "lg_prove_lockstep": (i32, [P, P, P, u64, u32, i32, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _check(status: int, ctx: Optional["Context"] = None) -> None:
    if status == 0:
        return
    msg = ""
    if ctx is not None and ctx.handle:
        msg = (lib.lg_ctx_last_error(ctx.handle) or b"").decode()
    if status == 5:
        raise LigeritoPanic(status, msg)
    raise LigeritoError(status, msg)


# ------------------------------------------------------------------ configs
@dataclass
class ProverConfig:
    """ProverConfig (src/data_structures.rs:9-22) minus the RS tables, which
    the device context builds and caches per message length."""

    recursive_steps: int
    initial_dims: tuple  # (m, n)
    dims: list           # [(m_i, n_i)]
    initial_k: int
    ks: list

    def to_c(self) -> LgConfig:
        c = LgConfig()
        c.recursive_steps = self.recursive_steps
        c.initial_log_m = _log2(self.initial_dims[0])
        c.initial_log_n = _log2(self.initial_dims[1])
        c.initial_k = self.initial_k
        for i, (m, n) in enumerate(self.dims):
            c.log_m[i] = _log2(m)
            c.log_n[i] = _log2(n)
            c.ks[i] = self.ks[i]
        return c

    @property
    def poly_len(self) -> int:
        return self.initial_dims[0] * self.initial_dims[1]


@dataclass
class VerifierConfig:
    """VerifierConfig (src/data_structures.rs:24-30)."""

    recursive_steps: int
    initial_dim: int
    log_dims: list
    initial_k: int
    ks: list

    def to_c(self) -> LgConfig:
        c = LgConfig()
        c.recursive_steps = self.recursive_steps
        c.initial_log_m = self.initial_dim
        c.initial_log_n = self.initial_k
        c.initial_k = self.initial_k
        for i, d in enumerate(self.log_dims):
            c.log_m[i] = d
            c.log_n[i] = self.ks[i]
            c.ks[i] = self.ks[i]
        return c


def _log2(x: int) -> int:
    if x <= 0 or x & (x - 1):
        raise LigeritoError(2, f"{x} is not a power of two")
    return x.bit_length() - 1


def _from_c(c: LgConfig) -> ProverConfig:
    s = c.recursive_steps
    return ProverConfig(
        recursive_steps=s,
        initial_dims=(1 << c.initial_log_m, 1 << c.initial_log_n),
        dims=[(1 << c.log_m[i], 1 << c.log_n[i]) for i in range(s)],
        initial_k=c.initial_k,
        ks=[c.ks[i] for i in range(s)],
    )


def _to_verifier(p: ProverConfig) -> VerifierConfig:
    return VerifierConfig(
        recursive_steps=p.recursive_steps,
        initial_dim=_log2(p.initial_dims[0]),
        log_dims=[_log2(m) for m, _ in p.dims],
        initial_k=p.initial_k,
        ks=list(p.ks),
    )


def hardcoded_config_20() -> ProverConfig:
    c = LgConfig()
    _check(lib.lg_hardcoded_config_20(ctypes.byref(c)))
    return _from_c(c)


def hardcoded_config_24() -> ProverConfig:
    c = LgConfig()
    _check(lib.lg_hardcoded_config_24(ctypes.byref(c)))
    return _from_c(c)


def config_from_text(text: str) -> ProverConfig:
    """A ProverConfig from its text form (lg_config_parse): lines
    "key = values" for recursive_steps, initial_dims, initial_k, dims and ks."""
    c = LgConfig()
    _check(lib.lg_config_parse(text.encode(), ctypes.byref(c)))
    return _from_c(c)


def config_to_text(cfg: ProverConfig) -> str:
    """The text form lg_config_parse reads back."""
    c = cfg.to_c()
    n = ctypes.c_uint64()
    _check(lib.lg_config_format(ctypes.byref(c), None, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value)
    _check(lib.lg_config_format(ctypes.byref(c), buf, ctypes.byref(n)))
    return buf.value.decode()


def hardcoded_config_20_verifier() -> VerifierConfig:
    return _to_verifier(hardcoded_config_20())


def hardcoded_config_24_verifier() -> VerifierConfig:
    return _to_verifier(hardcoded_config_24())


def config_for_size(log_size: int) -> ProverConfig:
    """Config for 2^log_size coefficients (16..30); equals config.rs at 20/24."""
    c = LgConfig()
    _check(lib.lg_config_make(log_size, ctypes.byref(c)))
    return _from_c(c)


def verifier_config_for(p: ProverConfig) -> VerifierConfig:
    return _to_verifier(p)


def validate_config(p: ProverConfig, poly_len: Optional[int] = None) -> None:
    c = p.to_c()
    _check(lib.lg_config_validate(ctypes.byref(c), p.poly_len if poly_len is None else poly_len))


# --------------------------------------------------------------- transcript
class FS:
    """Fiat-Shamir transcript, emulated_fs.rs:6-76 (host side of liblgpu)."""

    def __init__(self, seed: int):
        self.handle = ctypes.c_void_p()
        _check(lib.lg_transcript_new(seed, ctypes.byref(self.handle)))

    def __del__(self):
        try:
            if self.handle:
                lib.lg_transcript_free(self.handle)
        except Exception:
            pass

    def absorb(self, b: bytes) -> None:
        _check(lib.lg_transcript_absorb(self.handle, bytes(b), len(b)))

    def squeeze(self) -> int:
        out = (ctypes.c_uint64 * 2)()
        _check(lib.lg_transcript_squeeze(self.handle, out))
        return out[0] | (out[1] << 64)

    def get_field(self) -> int:
        v = ctypes.c_uint32()
        _check(lib.lg_transcript_get_field(self.handle, ctypes.byref(v)))
        return int(v.value)

    def get_query(self, n: int) -> int:
        v = ctypes.c_uint64()
        _check(lib.lg_transcript_get_query(self.handle, n, ctypes.byref(v)))
        return int(v.value)

    def get_distinct_queries(self, n: int, s: int) -> list:
        out = (ctypes.c_uint64 * max(s, 1))()
        _check(lib.lg_transcript_get_distinct_queries(self.handle, n, s, out))
        return [int(x) for x in out[:s]]


def merkle_verify(root: bytes, proof: Sequence[bytes], depth: int, leaves: Sequence[bytes],
                  leaf_indices: Sequence[int]) -> bool:
    """merkle_tree::verify (src/merkle_tree.rs:164-188), BLAKE3."""
    buf = b"".join(leaves)
    off = np.cumsum([0] + [len(x) for x in leaves]).astype(np.uint64)
    q = np.asarray(leaf_indices, dtype=np.uint64)
    sib = b"".join(proof) or b"\0"
    ok = ctypes.c_int()
    _check(lib.lg_merkle_verify(root, sib, len(proof), depth, buf or b"\0", off.ctypes.data, q.ctypes.data,
                                len(q), ctypes.byref(ok)))
    return bool(ok.value)


# ------------------------------------------------------------------ context
class Context:
    """One device, one CUDA stream, cached twiddle/pis tables (lg_ctx)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.handle = ctypes.c_void_p()
        _check(lib.lg_ctx_create(device, hbm_budget_bytes, ctypes.byref(self.handle)))
        self.device = device

    def close(self) -> None:
        if self.handle:
            lib.lg_ctx_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self) -> int:
        return lib.lg_ctx_stream(self.handle) or 0

    def synchronize(self) -> None:
        _check(lib.lg_ctx_synchronize(self.handle), self)

    @property
    def launch_count(self) -> int:
        return int(lib.lg_ctx_launch_count(self.handle))

    def set_kernel_timing(self, enabled: bool) -> None:
        _check(lib.lg_ctx_set_kernel_timing(self.handle, 1 if enabled else 0), self)

    def kernel_stats(self) -> dict:
        out, i = {}, 0
        name = ctypes.create_string_buffer(128)
        n, ms = ctypes.c_uint64(), ctypes.c_double()
        while lib.lg_ctx_kernel_stats(self.handle, i, name, 128, ctypes.byref(n), ctypes.byref(ms)) == 0:
            out[name.value.decode()] = (int(n.value), float(ms.value))
            i += 1
        return out

    def kernel_work(self) -> dict:
        """name -> (compulsory HBM bytes, GF(2^32) multiplications, BLAKE3
        compressions) of the timed launches, the same keys as kernel_stats."""
        out, i = {}, 0
        names = list(self.kernel_stats())
        b, m, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        while i < len(names) and lib.lg_ctx_kernel_work(self.handle, i, ctypes.byref(b), ctypes.byref(m),
                                                        ctypes.byref(c)) == 0:
            out[names[i]] = (float(b.value), float(m.value), float(c.value))
            i += 1
        return out

    def set_autotune(self, enabled: bool) -> None:
        _check(lib.lg_ctx_set_autotune(self.handle, 1 if enabled else 0), self)

    def reset_kernel_stats(self) -> None:
        _check(lib.lg_ctx_reset_kernel_stats(self.handle), self)

    @property
    def device_bytes_in_use(self) -> int:
        return int(lib.lg_ctx_device_bytes_in_use(self.handle))


def tuned_choices() -> list:
    """The autotuner's choices so far (lg_tuned_choices), one string each."""
    n = ctypes.c_uint64()
    _check(lib.lg_tuned_choices(None, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value)
    _check(lib.lg_tuned_choices(buf, ctypes.byref(n)))
    return [x for x in buf.value.decode().splitlines() if x]


PIPES = ("lop3", "iadd", "prmt", "shf", "imad", "imad_hi", "lop3_imad", "lds")


def measure_pipe_peaks(device: int = 0) -> dict:
    """Peak instruction rates of the device's integer pipes and of
    conflict-free shared-memory loads (lg_measure_pipe_peaks), per second
    over the whole device."""
    rates = (ctypes.c_double * len(PIPES))()
    _check(lib.lg_measure_pipe_peaks(device, rates, len(PIPES)))
    return {k: float(v) for k, v in zip(PIPES, rates)}


_default_ctx: dict = {}


def default_context(device: int = 0) -> Context:
    ctx = _default_ctx.get(device)
    if ctx is None:
        ctx = _default_ctx[device] = Context(device)
    return ctx


# -------------------------------------------------------------------- proofs
@dataclass
class Opening:
    opened_rows: list = field(default_factory=list)   # list of np.uint32 arrays
    merkle_proof: list = field(default_factory=list)  # list of bytes


@dataclass
class ProofFields:
    """Decoded FinalizedLigeritoProof (src/data_structures.rs:91-103)."""

    initial_root: bytes
    recursive_roots: list
    initial_ligero_proof: Opening
    recursive_proofs: list
    yr: np.ndarray
    final_ligero_proof: Opening
    sumcheck_transcript: list


def decode_proof(b: bytes) -> ProofFields:
    """Decode the canonical encoding (magic 'LGRP', version 1, field bytes 4)."""
    at = 0

    def u32():
        nonlocal at
        v = int.from_bytes(b[at:at + 4], "little")
        at += 4
        return v

    def raw(n):
        nonlocal at
        v = b[at:at + n]
        at += n
        return v

    def opening():
        o = Opening()
        for _ in range(u32()):
            n = u32()
            o.opened_rows.append(np.frombuffer(raw(4 * n), dtype="<u4").copy())
        for _ in range(u32()):
            o.merkle_proof.append(raw(u32()))
        return o

    if raw(4) != b"LGRP" or u32() != 1 or u32() != 4:
        raise LigeritoError(8, "bad magic/version")
    root0 = raw(u32())
    rr = [raw(u32()) for _ in range(u32())]
    init = opening()
    rec = [opening() for _ in range(u32())]
    n = u32()
    yr = np.frombuffer(raw(4 * n), dtype="<u4").copy()
    fin = opening()
    tr = [(u32(), u32(), u32()) for _ in range(u32())]
    if at != len(b):
        raise LigeritoError(8, "trailing bytes")
    return ProofFields(root0, rr, init, rec, yr, fin, tr)


class FinalizedLigeritoProof:
    """Opaque proof handle (lg_proof) with the canonical byte encoding."""

    def __init__(self, handle: ctypes.c_void_p):
        self.handle = handle

    def __del__(self):
        try:
            if self.handle:
                lib.lg_proof_free(self.handle)
        except Exception:
            pass

    def to_bytes(self) -> bytes:
        n = ctypes.c_uint64()
        _check(lib.lg_proof_serialize(self.handle, None, ctypes.byref(n)))
        out = bytearray(n.value)
        _check(lib.lg_proof_serialize(self.handle, (ctypes.c_char * len(out)).from_buffer(out), ctypes.byref(n)))
        return bytes(out)

    @classmethod
    def from_bytes(cls, b: bytes) -> "FinalizedLigeritoProof":
        h = ctypes.c_void_p()
        _check(lib.lg_proof_deserialize(b, len(b), ctypes.byref(h)))
        return cls(h)

    def proof_size(self) -> int:
        """ProofSize::proof_size (src/data_structures.rs:165-194)."""
        n = ctypes.c_uint64()
        _check(lib.lg_proof_size(self.handle, ctypes.byref(n)))
        return int(n.value)

    def fields(self) -> ProofFields:
        return decode_proof(self.to_bytes())


# ---------------------------------------------------------- device buffers
def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _dev_ptr(t) -> int:
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise LigeritoError(1, "expected a CUDA tensor")
    if t.element_size() != 4 or not t.is_contiguous():
        raise LigeritoError(1, "expected a contiguous 32-bit CUDA tensor")
    return t.data_ptr()


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _empty_dev(n: int, device: int):
    import torch

    return torch.empty(n, dtype=torch.int32, device=f"cuda:{device}")


def to_device(a, device: int = 0):
    import torch

    return torch.from_numpy(_u32(a).view(np.int32)).to(f"cuda:{device}")


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint32)


# ---------------------------------------------------------------- protocol
def prover(config: ProverConfig, poly, ctx: Optional[Context] = None) -> FinalizedLigeritoProof:
    """prover::<BinaryElem32>(config, poly) (src/prover.rs:15).  ``poly`` is a
    host uint32 array or a CUDA tensor of 32-bit words."""
    ctx = ctx or default_context()
    c = config.to_c()
    h = ctypes.c_void_p()
    if _is_torch(poly):
        st = lib.lg_prove(ctx.handle, ctypes.byref(c), _dev_ptr(poly), poly.numel(), 1, ctypes.byref(h))
    else:
        a = _u32(poly)
        st = lib.lg_prove(ctx.handle, ctypes.byref(c), a.ctypes.data, a.size, 0, ctypes.byref(h))
    _check(st, ctx)
    return FinalizedLigeritoProof(h)


def dump_intermediates(config: ProverConfig, poly, ctx: Optional[Context] = None):
    """lg_dump_intermediates: the proof ``prover`` gives, plus a dict
    {(name, level): bytes} of every intermediate the device produced on the
    way (encoded matrices, Merkle trees, folded vectors, queries, opened
    rows, induced bases, sumcheck triples, fold rounds, yr; the names and
    levels are listed in include/ligerito_b200.h).  Synchronises at every
    intermediate: a parity and debugging aid, not a fast path."""
    ctx = ctx or default_context()
    c = config.to_c()
    got = {}

    def cb(_user, name, level, data, nbytes):
        got[(name.decode(), int(level))] = ctypes.string_at(data, nbytes)

    fn = _DUMP_CB(cb)
    h = ctypes.c_void_p()
    if _is_torch(poly):
        st = lib.lg_dump_intermediates(ctx.handle, ctypes.byref(c), _dev_ptr(poly), poly.numel(), 1, fn, None,
                                       ctypes.byref(h))
    else:
        a = _u32(poly)
        st = lib.lg_dump_intermediates(ctx.handle, ctypes.byref(c), a.ctypes.data, a.size, 0, fn, None,
                                       ctypes.byref(h))
    _check(st, ctx)
    return FinalizedLigeritoProof(h), got


def prove_lockstep(config: ProverConfig, polys, ctx: Optional[Context] = None) -> list:
    """Many polynomials of one config proved in lockstep on one context
    (lg_prove_lockstep): every kernel launch covers up to 64 proofs.
    ``polys``: a 2-D CUDA tensor or host array (one polynomial per row), or
    a sequence of 1-D ones (all CUDA tensors or all host arrays).  Returns
    one proof per polynomial, each the bytes ``prover`` gives alone."""
    ctx = ctx or default_context()
    c = config.to_c()
    rows = [polys[i] for i in range(len(polys))]
    n = len(rows)
    if n == 0:
        return []
    on_dev = 1 if _is_torch(rows[0]) else 0
    keep = []
    ptrs = (ctypes.c_void_p * n)()
    length = None
    for i, r in enumerate(rows):
        if on_dev:
            if not r.is_contiguous():
                raise ValueError("polynomial rows must be contiguous")
            ptrs[i], ln = _dev_ptr(r), r.numel()
        else:
            a = _u32(r)
            keep.append(a)
            ptrs[i], ln = a.ctypes.data, a.size
        if length is None:
            length = ln
        elif ln != length:
            raise ValueError("lockstep polynomials must all have the config's length")
    out = (ctypes.c_void_p * n)()
    st = lib.lg_prove_lockstep(ctx.handle, ctypes.byref(c), ptrs, length, n, on_dev, out)
    proofs = [FinalizedLigeritoProof(ctypes.c_void_p(out[i])) if out[i] else None for i in range(n)]
    _check(st, ctx)
    return proofs


def verifier(config, proof, ctx: Optional[Context] = None) -> bool:
    """verifier::<BinaryElem32>(config, proof) (src/verifier.rs:10): the
    reference's bool, or LigeritoPanic where the reference panics."""
    ctx = ctx or default_context()
    if isinstance(config, ProverConfig):
        config = _to_verifier(config)
    c = config.to_c()
    acc = ctypes.c_int()
    if isinstance(proof, (bytes, bytearray)):
        b = bytes(proof)
        _check(lib.lg_verify_bytes(ctx.handle, ctypes.byref(c), b, len(b), ctypes.byref(acc)), ctx)
        return bool(acc.value)
    _check(lib.lg_verify(ctx.handle, ctypes.byref(c), proof.handle, ctypes.byref(acc)), ctx)
    return bool(acc.value)


# ------------------------------------------------------------ kernel level
def compute_twiddles(log_n: int) -> np.ndarray:
    """compute_twiddles::<BinaryElem32>(log_n, None) (src/binary_fft.rs:30)."""
    out = np.zeros((1 << log_n) - 1, dtype=np.uint32)
    _check(lib.lg_compute_twiddles(log_n, out.ctypes.data))
    return out


def fft(data, log_n: int, ctx: Optional[Context] = None) -> None:
    """In-place fft (src/binary_fft.rs:4) of each contiguous 2^log_n slice of
    the CUDA tensor ``data``."""
    ctx = ctx or default_context()
    batch = data.numel() >> log_n
    _check(lib.lg_fft(ctx.handle, _dev_ptr(data), log_n, batch), ctx)


def ifft(data, log_n: int, ctx: Optional[Context] = None) -> None:
    """In-place ifft (src/binary_fft.rs:19) of each 2^log_n slice."""
    ctx = ctx or default_context()
    batch = data.numel() >> log_n
    _check(lib.lg_ifft(ctx.handle, _dev_ptr(data), log_n, batch), ctx)


def encode_cols(poly, log_m: int, n: int, ctx: Optional[Context] = None):
    """poly2flatmat + encode_cols (src/ligero.rs:11-38): column-major n x 4m."""
    ctx = ctx or default_context()
    out = _empty_dev(n << (log_m + 2), ctx.device)
    _check(lib.lg_rs_encode_cols(ctx.handle, _dev_ptr(poly), log_m, n, _dev_ptr(out)), ctx)
    return out


def ligero_commit(poly, log_m: int, n: int, ctx: Optional[Context] = None):
    """ligero_commit (src/ligero.rs:70-95) -> (encoded, tree, root)."""
    import torch

    ctx = ctx or default_context()
    rows = 4 << log_m
    enc = _empty_dev(n * rows, ctx.device)
    tree = torch.empty((2 * rows - 1) * 8, dtype=torch.int32, device=f"cuda:{ctx.device}")
    root = ctypes.create_string_buffer(32)
    _check(lib.lg_ligero_commit(ctx.handle, _dev_ptr(poly), log_m, n, _dev_ptr(enc), _dev_ptr(tree), root), ctx)
    return enc, tree, root.raw


def partial_eval(evals, rs: Sequence[int], ctx: Optional[Context] = None):
    """MultiLinearPoly::partial_eval (src/multilinear_poly.rs:66-87)."""
    ctx = ctx or default_context()
    log_len = _log2(evals.numel())
    r = _u32(rs)
    out = _empty_dev(evals.numel() >> len(r), ctx.device)
    _check(lib.lg_partial_eval(ctx.handle, _dev_ptr(evals), log_len, r.ctypes.data, len(r), _dev_ptr(out)), ctx)
    return out


def eval_013_product(f, g, ctx: Optional[Context] = None) -> tuple:
    """eval_013_product (src/multilinear_poly.rs:90-131)."""
    ctx = ctx or default_context()
    out = np.zeros(3, dtype=np.uint32)
    _check(lib.lg_eval_013_product(ctx.handle, _dev_ptr(f), _dev_ptr(g), _log2(f.numel()), out.ctypes.data), ctx)
    return tuple(int(x) for x in out)


def induce_sumcheck_poly(n: int, opened_rows, v_challenges: Sequence[int], sorted_queries: Sequence[int],
                         alpha: int, ctx: Optional[Context] = None):
    """induce_sumcheck_poly_parallel (src/sumcheck_polys.rs:74-160) ->
    (basis_poly CUDA tensor of 2^n, enforced_sum)."""
    ctx = ctx or default_context()
    rows = _u32(opened_rows).reshape(len(sorted_queries), -1)
    ch = _u32(v_challenges)
    q = np.ascontiguousarray(np.asarray(sorted_queries, dtype=np.uint64))
    out = _empty_dev(1 << n, ctx.device)
    es = ctypes.c_uint32()
    _check(lib.lg_induce_sumcheck_poly(ctx.handle, n, rows.ctypes.data, rows.shape[0], ch.ctypes.data, len(ch),
                                       q.ctypes.data, alpha, _dev_ptr(out), ctypes.byref(es)), ctx)
    return out, int(es.value)


def splitmix_coeffs(seed: int, n: int) -> np.ndarray:
    """Seeded coefficients: SplitMix64, coefficient i = low 32 bits of output i."""
    out = np.empty(n, dtype=np.uint32)
    lib.lg_fill_splitmix_host(seed, out.ctypes.data, n)
    return out


def gf128_mul(a, b, ctx: Optional[Context] = None):
    """BinaryElem128 products a[i] * b[i] (src/binary_field.rs:182-189) of
    two CUDA int64 tensors of shape (n, 2): each row is an element's low and
    high 64 bits.  Returns a new tensor of the same shape."""
    import torch

    ctx = ctx or default_context()
    if a.shape != b.shape or a.dim() != 2 or a.shape[1] != 2 or a.dtype != torch.int64 or b.dtype != torch.int64:
        raise ValueError("gf128_mul wants two int64 tensors of shape (n, 2)")
    if not (a.is_cuda and b.is_cuda):
        raise LigeritoError(1, "expected CUDA tensors")
    a, b = a.contiguous(), b.contiguous()
    out = torch.empty_like(a)
    _check(lib.lg_gf128_mul(ctx.handle, a.data_ptr(), b.data_ptr(), out.data_ptr(), a.shape[0]), ctx)
    return out


def splitmix_coeffs_device(seed: int, n: int, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    out = _empty_dev(n, ctx.device)
    _check(lib.lg_fill_splitmix(ctx.handle, seed, _dev_ptr(out), n), ctx)
    return out


# ------------------------------------------------------- batched / serving
class Server:
    """Continuous-batching proof server (lg_server_*): `workers` concurrent
    contexts on one GPU, FIFO admission under an HBM budget."""

    def __init__(self, device: int = 0, workers: int = 4, hbm_budget_bytes: int = 0, max_batch: int = 1):
        self.handle = ctypes.c_void_p()
        _check(lib.lg_server_create(device, hbm_budget_bytes, workers, ctypes.byref(self.handle)))
        self._keep = {}
        if max_batch != 1:
            self.set_max_batch(max_batch)

    def set_max_batch(self, max_batch: int) -> None:
        """Same-config queued requests a worker proves in lockstep (1..64)."""
        _check(lib.lg_server_set_max_batch(self.handle, max_batch))

    def submit(self, config: ProverConfig, poly, copy_input: bool = False) -> int:
        c = config.to_c()
        t = ctypes.c_uint64()
        if _is_torch(poly):
            st = lib.lg_server_submit(self.handle, ctypes.byref(c), _dev_ptr(poly), poly.numel(), 1, 0, ctypes.byref(t))
        else:
            a = _u32(poly)
            st = lib.lg_server_submit(self.handle, ctypes.byref(c), a.ctypes.data, a.size, 0, 1 if copy_input else 0,
                                      ctypes.byref(t))
            poly = a
        _check(st)
        if not copy_input or _is_torch(poly):
            self._keep[t.value] = poly  # the server reads it until wait() returns
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = -1):
        """-> (FinalizedLigeritoProof, latency_ms, queue_ms)"""
        h = ctypes.c_void_p()
        lat, q = ctypes.c_double(), ctypes.c_double()
        st = lib.lg_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(h), ctypes.byref(lat), ctypes.byref(q))
        if st == 10:
            return None
        self._keep.pop(ticket, None)
        _check(st)
        return FinalizedLigeritoProof(h), float(lat.value), float(q.value)

    def warm(self, configs: Sequence[ProverConfig]) -> None:
        """One proof of each config on every worker at once (lg_server_warm):
        later requests pay no first-use costs."""
        n = len(configs)
        cfgs = (LgConfig * n)(*[c.to_c() for c in configs])
        _check(lib.lg_server_warm(self.handle, cfgs, n))

    def stats(self) -> dict:
        c, q, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib.lg_server_stats(self.handle, ctypes.byref(c), ctypes.byref(q), ctypes.byref(b)))
        return {"completed": c.value, "queued": q.value, "in_flight_bytes": b.value}

    def close(self) -> None:
        if self.handle:
            lib.lg_server_destroy(self.handle)
            self.handle = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prove_batch(configs: Sequence[ProverConfig], polys, workers: int = 4, device: int = 0) -> list:
    """Prove many polynomials (uneven sizes) concurrently; same bytes as
    `prover` on each alone."""
    n = len(polys)
    cfgs = (LgConfig * n)(*[c.to_c() for c in configs])
    on_dev = 1 if n and _is_torch(polys[0]) else 0
    keep = []
    ptrs = (ctypes.c_void_p * n)()
    lens = (ctypes.c_uint64 * n)()
    for i, p in enumerate(polys):
        if on_dev:
            ptrs[i], lens[i] = _dev_ptr(p), p.numel()
        else:
            a = _u32(p)
            keep.append(a)
            ptrs[i], lens[i] = a.ctypes.data, a.size
    out = (ctypes.c_void_p * n)()
    _check(lib.lg_prove_batch(device, workers, cfgs, ptrs, lens, on_dev, n, out))
    return [FinalizedLigeritoProof(ctypes.c_void_p(out[i])) for i in range(n)]
