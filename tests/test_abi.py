"""liblgpu.so on the CPU: it loads, exports every symbol the header
declares, and its host-side protocol parts (configs, twiddles, transcript,
Merkle verification, proof codec) agree with the oracle.  No GPU needed."""
import ctypes
import hashlib
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ligerito_b200.h"


def declared_symbols():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(lg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lg):
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lg.lib, s)]
    assert not missing, missing


def test_library_is_sm100a_cuda_build():
    so = ROOT / "ligerito-rust_b200" / "_build" / "liblgpu.so"
    assert so.exists() and so.stat().st_size > 100_000


def test_status_strings(lg):
    assert lg.lib.lg_status_string(0) == b"ok"
    assert lg.lib.lg_status_string(5) == b"verifier panic"
    assert lg.lib.lg_abi_version() == 1


def test_hardcoded_configs(lg):
    # src/config.rs:6-134
    c20, c24 = lg.hardcoded_config_20(), lg.hardcoded_config_24()
    assert (c20.recursive_steps, c20.initial_dims, c20.dims, c20.initial_k, c20.ks) == (
        1, (1 << 14, 1 << 6), [(1 << 10, 1 << 4)], 6, [4])
    assert (c24.recursive_steps, c24.initial_dims, c24.dims, c24.initial_k, c24.ks) == (
        2, (1 << 18, 1 << 6), [(1 << 14, 1 << 4), (1 << 10, 1 << 4)], 6, [4, 4])
    v20 = lg.hardcoded_config_20_verifier()
    assert (v20.initial_dim, v20.log_dims, v20.ks) == (14, [10], [4])
    v24 = lg.hardcoded_config_24_verifier()
    assert (v24.initial_dim, v24.log_dims, v24.ks) == (18, [14, 10], [4, 4])


@pytest.mark.parametrize("L", range(16, 31))
def test_config_generator_matches_oracle(lg, ref, L):
    a = lg.config_for_size(L).to_c()
    b = ref.config_make(L)
    s = a.recursive_steps
    assert (s, a.initial_log_m, a.initial_log_n, a.initial_k, tuple(a.log_m[:s]), tuple(a.log_n[:s]),
            tuple(a.ks[:s])) == b.as_tuple()
    lg.validate_config(lg.config_for_size(L))


def test_config_validation_rejects(lg):
    good = lg.hardcoded_config_20()
    with pytest.raises(lg.LigeritoError) as e:
        lg.validate_config(good, poly_len=(1 << 20) + 1)
    assert e.value.status == 2
    bad = lg.ProverConfig(1, (1 << 14, 64), [(1 << 9, 16)], 6, [4])  # 14 != 9 + 4
    with pytest.raises(lg.LigeritoError):
        lg.validate_config(bad)
    few_rows = lg.ProverConfig(1, (1 << 9, 16), [(32, 16)], 4, [4])  # 128 rows < 148 queries
    with pytest.raises(lg.LigeritoError):
        lg.validate_config(few_rows)
    for L in (0, 15, 31):
        c = lg.LgConfig()
        assert lg.lib.lg_config_make(L, ctypes.byref(c)) == 1


@pytest.mark.parametrize("log_n", [1, 2, 3, 7, 12, 16, 20])
def test_twiddles_match_oracle(lg, ref, log_n):
    # compute_twiddles (src/binary_fft.rs:30-58); the library fills each
    # layer from its GF(2)-linear basis, the oracle runs the reference loop
    assert (lg.compute_twiddles(log_n) == ref.twiddles(log_n)).all()


def test_splitmix_host_matches_oracle(lg, ref):
    for seed in (0, 1, 2, 2**40 + 7):
        assert (lg.splitmix_coeffs(seed, 4096) == ref.splitmix(seed, 4096)).all()


def test_transcript_matches_oracle(lg, ref):
    L = ref.lib()
    h = L.lgref_fs_new(1234)
    fs = lg.FS(1234)
    try:
        for step in range(40):
            data = bytes((step * 7 + i) & 255 for i in range(step * 3))
            fs.absorb(data)
            L.lgref_fs_absorb(h, data, len(data))
            out = (ctypes.c_uint64 * 2)()
            L.lgref_fs_squeeze(h, out)
            assert fs.squeeze() == out[0] | (out[1] << 64)
            assert fs.get_field() == L.lgref_fs_get_field32(h)
            assert fs.get_query(1000003) == L.lgref_fs_get_query(h, 1000003)
        q = np.zeros(148, np.uint64)
        assert L.lgref_fs_get_distinct_queries(h, 1 << 16, 148, q.ctypes.data) == 0
        assert fs.get_distinct_queries(1 << 16, 148) == q.tolist()
        with pytest.raises(lg.LigeritoError):
            fs.get_distinct_queries(100, 148)  # the reference would never return
    finally:
        L.lgref_fs_free(h)


def test_host_merkle_verify(lg, ref):
    # merkle_tree::verify with BLAKE3, against an oracle tree
    leaves = [bytes([i]) * (5 + i) for i in range(16)]
    buf = b"".join(leaves)
    off = np.cumsum([0] + [len(x) for x in leaves]).astype(np.uint64)
    tree = np.zeros(32 * 31, np.uint8)
    assert ref.lib().lgref_merkle_build(0, buf, off.ctypes.data, 16, tree.ctypes.data) == 0
    root = bytes(tree[-32:])
    for q in ([0], [3, 4], [0, 1, 2, 3], [5, 9, 15], list(range(16))):
        qa = np.asarray(q, np.uint64)
        sib = np.zeros(32 * 64, np.uint8)
        ns = ctypes.c_size_t()
        ref.lib().lgref_merkle_prove(tree.ctypes.data, 16, qa.ctypes.data, len(q), sib.ctypes.data, 64,
                                     ctypes.byref(ns))
        proof = [bytes(sib[32 * i:32 * i + 32]) for i in range(ns.value)]
        assert lg.merkle_verify(root, proof, 4, [leaves[i] for i in q], q)
        assert not lg.merkle_verify(root, proof, 4, [b"x" + leaves[i] for i in q], q)
        if proof:
            with pytest.raises(lg.LigeritoPanic):
                lg.merkle_verify(root, proof[:-1], 4, [leaves[i] for i in q], q)


def _oracle_proof(ref, L=16, seed=16):
    cfg = ref.config_make(L)
    return ref.prove(cfg, ref.splitmix(seed, 1 << L), nthreads=8)


def test_proof_codec_roundtrip(lg, ref):
    b = _oracle_proof(ref)
    p = lg.FinalizedLigeritoProof.from_bytes(b)
    assert p.to_bytes() == b
    f = p.fields()
    assert len(f.initial_root) == 32 and len(f.recursive_roots) == 1
    assert len(f.initial_ligero_proof.opened_rows) == 148
    assert all(r.size == 64 for r in f.initial_ligero_proof.opened_rows)
    assert f.yr.size == 1 << 6 - 4 + 4 and len(f.sumcheck_transcript) == 1 + 4
    # ProofSize (src/data_structures.rs:105-194)
    expect = 32 + 32 + sum(4 * r.size for r in f.initial_ligero_proof.opened_rows)
    expect += sum(len(s) for s in f.initial_ligero_proof.merkle_proof)
    expect += 4 * f.yr.size + sum(4 * r.size for r in f.final_ligero_proof.opened_rows)
    expect += sum(len(s) for s in f.final_ligero_proof.merkle_proof) + 12 * len(f.sumcheck_transcript)
    assert p.proof_size() == expect


def test_proof_codec_rejects_malformed(lg, ref):
    b = _oracle_proof(ref)
    for bad in (b[:-1], b + b"\0", b"XXXX" + b[4:], b[:8]):
        with pytest.raises(lg.LigeritoError) as e:
            lg.FinalizedLigeritoProof.from_bytes(bad)
        assert e.value.status == 8


def test_no_gpu_fails_loudly(lg):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(lg.LigeritoError) as e:
        lg.Context(0)
    assert e.value.status == 7


def test_config_text_round_trip(lg):
    # the hard-coded configs (src/config.rs:6-134) and generated ones survive
    # text and back; the text of config 24 reads as expected
    for cfg in [lg.hardcoded_config_20(), lg.hardcoded_config_24()] + [lg.config_for_size(L) for L in (16, 19, 22, 28)]:
        txt = lg.config_to_text(cfg)
        back = lg.config_from_text(txt)
        assert back == cfg and lg.config_to_text(back) == txt
    txt = lg.config_to_text(lg.hardcoded_config_24())
    assert "initial_dims = 262144 64" in txt and "dims = 16384 16, 1024 16" in txt and "ks = 4 4" in txt
    # comments, blank lines, spacing and key order are free
    alt = "# config 24\n\nks = 4 4\ndims=16384 16 ,1024 16  # two steps\ninitial_k=6\n" \
          "recursive_steps = 2\n  initial_dims =262144 64\n"
    assert lg.config_from_text(alt) == lg.hardcoded_config_24()


@pytest.mark.parametrize("bad", [
    "",                                                                       # nothing
    "recursive_steps = 1\ninitial_dims = 256 16\ninitial_k = 4\ndims = 64 4\n",  # no ks
    "recursive_steps = 1\ninitial_dims = 250 16\ninitial_k = 4\ndims = 64 4\nks = 2\n",  # not a power of two
    "recursive_steps = 2\ninitial_dims = 256 16\ninitial_k = 4\ndims = 64 4\nks = 2\n",  # too few steps
    "recursive_steps = 1\ninitial_dims = 256 16\ninitial_k = 4\ndims = 64 4\nks = 2\nks = 2\n",  # repeated key
    "recursive_steps = 1\ninitial_dims = 256 16\ninitial_k = x\ndims = 64 4\nks = 2\n",  # not a number
    "recursive_steps = 1\ninitial_dims = 256 16\ninitial_k = 4\ndims = 64 4\nks = 2\ncolour = 3\n",  # unknown key
    "recursive_steps 1\n",                                                    # no '='
])
def test_config_text_errors(lg, bad):
    with pytest.raises(lg.LigeritoError) as e:
        lg.config_from_text(bad)
    assert e.value.status == 2  # LG_ERR_INVALID_CONFIG
