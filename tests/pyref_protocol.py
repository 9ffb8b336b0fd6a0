"""An independent pure-Python restatement of the reference prover and
verifier, for small sizes (2^10 - 2^14).

TEST INFRASTRUCTURE ONLY.  It exists to check the C oracle's composition of
the protocol -- the order of transcript absorbs and squeezes, the queries
drawn on the previous witness's rows, introduce_new / glue, the verifier's
replay -- against a second restatement written straight from the reference
sources, with different building blocks: Python integers for GF(2^32)
(bit-serial, src/binary_field.rs:52-105), hashlib's SHA-256 for the
transcript (the sha2 crate, src/emulated_fs.rs) and the `blake3` module for
the Merkle hashes (the blake3 crate, src/merkle_tree.rs).  It shares no code
with oracle/lgref.c.  Each function cites the reference file:line it follows.
"""
from __future__ import annotations

import hashlib
import struct

import blake3

POLY32 = 0x8299  # x^32 + x^15 + x^9 + x^7 + x^4 + x^3 + 1, src/binary_field.rs:179-181
S_QUERIES = 148  # src/prover.rs:30
FS_SEED = 1234  # src/prover.rs:29
INV_RATE = 4  # src/ligero.rs:81


# ----------------------------------------------------------------- GF(2^32)
def gf_mul(a: int, b: int) -> int:
    """poly_multiply_gf2 then mod_irreducible (src/binary_field.rs:52-105)."""
    prod = 0
    while b:
        if b & 1:
            prod ^= a
        a <<= 1
        b >>= 1
    for i in range(63, 31, -1):  # fold the high word down, top bit first
        if (prod >> i) & 1:
            prod ^= POLY32 << (i - 32)
            prod ^= 1 << i
    return prod


def gf_pow(a: int, e: int) -> int:
    r = 1
    while e:
        if e & 1:
            r = gf_mul(r, a)
        a = gf_mul(a, a)
        e >>= 1
    return r


def gf_inv(a: int) -> int:  # Fermat, src/binary_field.rs:40-50
    assert a
    return gf_pow(a, (1 << 32) - 2)


# ---------------------------------------------------------- additive FFT
def next_s(s_prev: int, s_prev_at_root: int) -> int:  # src/binary_fft.rs:100-107
    return gf_mul(s_prev, s_prev) ^ gf_mul(s_prev_at_root, s_prev)


def compute_twiddles(log_n: int) -> list:  # src/binary_fft.rs:30-98, beta = 0
    tw = [0] * ((1 << log_n) - 1)
    layer_size = 1 << (log_n - 1)
    layer = [i << 1 for i in range(layer_size)]  # layer_0
    write_at = layer_size
    s_prev_at_root = 1
    tw[write_at - 1:] = layer
    for _ in range(log_n - 1):
        write_at >>= 1
        layer_size = write_at
        # layer_i: s_at_root from the previous layer, then the layer halves
        s_at_root = next_s(layer[1] ^ layer[0], s_prev_at_root)
        layer = [next_s(layer[2 * k], s_prev_at_root) for k in range(layer_size)]
        s_prev_at_root = s_at_root
        s_inv = gf_inv(s_prev_at_root)
        for i in range(layer_size):
            tw[write_at + i - 1] = gf_mul(s_inv, layer[i])
    return tw


def fft(v: list, tw: list) -> list:
    """fft_twiddles / fft_mul (src/binary_fft.rs:143-192): at heap node idx,
    u += lambda * w; w += u over the halves, then the children."""
    v = list(v)

    def rec(lo: int, n: int, idx: int):
        if n == 1:
            return
        lam, h = tw[idx - 1], n // 2
        for i in range(h):
            u = v[lo + i] ^ gf_mul(lam, v[lo + h + i])
            v[lo + i] = u
            v[lo + h + i] ^= u
        rec(lo, h, 2 * idx)
        rec(lo + h, h, 2 * idx + 1)

    rec(0, len(v), 1)
    return v


def eval_sk_at_vks(n: int) -> list:  # src/binary_fft.rs:217-246
    k = n.bit_length() - 1
    sks = [1]
    layer = [1 << i for i in range(1, k + 1)]
    cur = k
    for i in range(1, k + 1):
        for j in range(1, cur + 1):
            if j == 1:
                sks.append(gf_mul(layer[0], layer[0]) ^ gf_mul(sks[i - 1], layer[0]))
            else:
                layer[j - 2] = gf_mul(layer[j - 1], layer[j - 1]) ^ gf_mul(sks[i - 1], layer[j - 1])
        cur -= 1
    return sks


def compute_pis(m: int, sks: list) -> list:  # src/binary_fft.rs:303-322
    pis = [0] * m
    pis[0] = 1
    for i in range(2, len(sks) + 1):
        cur = 1 << (i - 2)
        for j in range(1, cur + 1):
            pis[j + cur - 1] = gf_mul(sks[i - 2], pis[j - 1])
    return pis


def scaled_basis(sks_vks: list, x: int, alpha: int, length: int) -> list:
    """evaluate_scaled_basis_inplace (src/binary_fft.rs:276-301)."""
    k = length.bit_length() - 1
    sx = [0] * max(k, 1)
    sx[0] = x
    for i in range(2, k + 1):
        sx[i - 1] = next_s(sx[i - 2], sks_vks[i - 2])
    basis = [0] * length
    basis[0] = alpha
    for i in range(1, k + 1):
        cur = 1 << (i - 1)
        for j in range(1, cur + 1):
            basis[j + cur - 1] = gf_mul(sx[i - 1], basis[j - 1])
    return basis


# ------------------------------------------------------------------ codes
class Code:
    """ReedSolomonEncoding::new(m, 4m) (src/reed_solomon.rs:49-64)."""

    def __init__(self, m: int):
        self.m = m
        self.tw = compute_twiddles((INV_RATE * m).bit_length() - 1)
        self.pis = compute_pis(m, eval_sk_at_vks(m))

    def encode_non_systematic(self, col: list) -> list:  # src/reed_solomon.rs:104-113
        v = [gf_mul(col[i], self.pis[i]) if i < self.m else col[i] for i in range(len(col))]
        return fft(v, self.tw)


# ----------------------------------------------------------------- merkle
def build_merkle_tree(leaves: list) -> list:  # src/merkle_tree.rs:4-60
    layer = [blake3.blake3(x).digest() for x in leaves]
    layers = [layer]
    while len(layer) > 1:
        layer = [blake3.blake3(layer[2 * i] + layer[2 * i + 1]).digest() for i in range(len(layer) // 2)]
        layers.append(layer)
    return layers


def merkle_prove(tree: list, queries: list) -> list:  # src/merkle_tree.rs:62-111
    proof = []
    q = list(queries)
    cnt = len(q)
    for depth in range(len(tree) - 1):
        layer = tree[depth]
        nxt, i = 0, 0
        while i < cnt:
            query = q[i]
            sib = query ^ 1
            nxt += 1
            q[nxt - 1] = query >> 1
            if i == cnt - 1:
                proof.append(layer[sib])
                break
            if query % 2 != 0 or q[i + 1] != sib:
                proof.append(layer[sib])
                i += 1
            else:
                i += 2
        cnt = nxt
    return proof


def merkle_verify(root: bytes, proof: list, depth: int, leaves: list, queries: list) -> bool:
    """merkle_tree::verify (src/merkle_tree.rs:120-188); an index past the
    proof is the reference's panic, raised here as IndexError."""
    layer = [blake3.blake3(x).digest() for x in leaves]
    q = list(queries)
    cnt, pc = len(q), 0
    for _ in range(depth):
        nxt, i = 0, 0
        while i < cnt:
            query = q[i]
            sib = query ^ 1
            nxt += 1
            q[nxt - 1] = query >> 1
            if i == cnt - 1:
                pc += 1
                pair = (proof[pc - 1], layer[i]) if query % 2 != 0 else (layer[i], proof[pc - 1])
                layer[nxt - 1] = blake3.blake3(pair[0] + pair[1]).digest()
                break
            if query % 2 != 0:
                pc += 1
                layer[nxt - 1] = blake3.blake3(proof[pc - 1] + layer[i]).digest()
                i += 1
            elif q[i + 1] != sib:
                pc += 1
                layer[nxt - 1] = blake3.blake3(layer[i] + proof[pc - 1]).digest()
                i += 1
            else:
                layer[nxt - 1] = blake3.blake3(layer[i] + layer[i + 1]).digest()
                i += 2
        cnt = nxt
    return cnt == 1 and layer[0] == root


# ------------------------------------------------------------------ ligero
def le_bytes(words: list) -> bytes:
    return struct.pack(f"<{len(words)}I", *words)


class Witness:
    """ligero_commit (src/ligero.rs:11-95): columns j of m words, each padded
    to 4m and encoded; leaf i = row i's words as LE bytes."""

    def __init__(self, poly: list, m: int, n: int, code: Code):
        rows = INV_RATE * m
        self.cols = [code.encode_non_systematic(poly[j * m:(j + 1) * m] + [0] * (rows - m)) for j in range(n)]
        self.num_rows, self.num_cols = rows, n
        self.tree = build_merkle_tree([le_bytes(self.row(i)) for i in range(rows)])

    def row(self, i: int) -> list:  # extract_row, src/ligero.rs:40-51
        return [c[i] for c in self.cols]

    @property
    def root(self) -> bytes:
        return self.tree[-1][0]


def lagrange_basis(rs: list) -> list:  # evaluate_lagrange_basis, src/utils.rs:4-27
    cur = [1 ^ rs[0], rs[0]]
    for r in rs[1:]:
        nxt = []
        for c in cur:
            nxt += [gf_mul(c, 1 ^ r), gf_mul(c, r)]
        cur = nxt
    return cur


def ligero_verify(queries, rows, yr, challenges) -> None:  # src/ligero.rs:97-131
    gr = lagrange_basis(challenges)
    sks = eval_sk_at_vks(len(yr))
    for q, row in zip(queries, rows):
        dot = 0
        for a, g in zip(row, gr):
            dot ^= gf_mul(a, g)
        basis = scaled_basis(sks, q, 1, len(yr))
        e = 0
        for y, b in zip(yr, basis):
            e ^= gf_mul(y, b)
        assert e == dot, "ligero_verify"


# ----------------------------------------------------------- multilinear
def partial_eval(evals: list, rs: list) -> list:  # src/multilinear_poly.rs:66-87
    n = len(evals) // 2
    out = [gf_mul(1 ^ rs[0], evals[i]) ^ gf_mul(rs[0], evals[i + n]) for i in range(n)]
    for r in rs[1:]:
        n //= 2
        out = [gf_mul(1 ^ r, out[i]) ^ gf_mul(r, out[i + n]) for i in range(n)]
    return out


def evals_at_x(e0, e1, x=3):  # src/ligerito.rs:130-141
    return [gf_mul(x, b) ^ gf_mul(1 ^ x, a) for a, b in zip(e0, e1)]


def dotp(a, b) -> int:
    s = 0
    for x, y in zip(a, b):
        s ^= gf_mul(x, y)
    return s


def eval_013_product(f, g):  # src/multilinear_poly.rs:90-131
    h = len(f) // 2
    f0, f1, g0, g1 = f[:h], f[h:], g[:h], g[h:]
    return dotp(f0, g0), dotp(f1, g1), dotp(evals_at_x(f0, f1), evals_at_x(g0, g1))


def induce(n, sks_vks, rows, v_challenges, queries, alpha):
    """induce_sumcheck_poly (src/sumcheck_polys.rs:22-72; the parallel twin
    at :74-160 sums the same terms)."""
    gr = lagrange_basis(v_challenges)
    assert all(len(r) == len(gr) for r in rows) and len(rows) == len(queries)
    apow, basis_poly, enforced = 1, [0] * (1 << n), 0
    for row, q in zip(rows, queries):
        enforced ^= gf_mul(dotp(row, gr), apow)
        for j, b in enumerate(scaled_basis(sks_vks, q, apow, 1 << n)):
            basis_poly[j] ^= b
        apow = gf_mul(apow, alpha)
    return basis_poly, enforced


class SumcheckProver:
    """SumcheckProverInstance (src/ligerito.rs:7-128)."""

    def __init__(self, f, b1, h1):
        s = eval_013_product(f, b1)
        assert s[0] ^ s[1] == h1
        self.f, self.basis, self.transcript, self.to_glue = f, [b1], [s], None
        self.first = s

    def introduce_new(self, bi, h):
        s = eval_013_product(self.f, bi)
        assert s[0] ^ s[1] == h
        self.transcript.append(s)
        self.to_glue = bi
        return s

    def glue(self, alpha):
        self.basis.append([gf_mul(x, alpha) for x in self.to_glue])
        self.to_glue = None

    def fold(self, r):
        self.f = partial_eval(self.f, [r])
        self.basis = [partial_eval(b, [r]) for b in self.basis]
        h = len(self.f) // 2
        f0, f1 = self.f[:h], self.f[h:]
        b0 = [0] * h
        b1 = [0] * h
        for b in self.basis:
            b0 = [x ^ y for x, y in zip(b0, b[:h])]
            b1 = [x ^ y for x, y in zip(b1, b[h:])]
        # eval_01x_product sums evals_at_x of each basis poly, the same as
        # evals_at_x of the sums (linear)
        s = (dotp(f0, b0), dotp(f1, b1), dotp(evals_at_x(f0, f1), evals_at_x(b0, b1)))
        self.transcript.append(s)
        return s


def quad_bytes(s) -> bytes:  # QuadraticEvals::to_bytes, src/sumcheck.rs:29-36
    return le_bytes(list(s))


# ------------------------------------------------------------- transcript
class FS:
    """src/emulated_fs.rs:6-76 over hashlib's SHA-256."""

    def __init__(self, seed: int):
        self.h = hashlib.sha256(struct.pack("<I", seed))
        self.counter = 0

    def absorb(self, b: bytes):
        self.h.update(b)

    def squeeze(self) -> int:
        self.h.update(struct.pack("<I", self.counter))
        self.counter += 1
        return int.from_bytes(self.h.copy().digest()[:16], "little")

    def get_field(self) -> int:
        return self.squeeze() & 0xFFFFFFFF

    def get_query(self, n: int) -> int:
        return (self.squeeze() & ((1 << 64) - 1)) % n

    def get_distinct_queries(self, n: int, s: int) -> list:
        seen, out = set(), []
        while len(out) < s:
            q = self.get_query(n)
            if q not in seen:
                seen.add(q)
                out.append(q)
        return sorted(out)


# ------------------------------------------------------------------ prover
class Config:
    """ProverConfig (src/data_structures.rs:9-22) with its codes."""

    def __init__(self, steps, initial_log_m, initial_log_n, initial_k, log_m, log_n, ks):
        self.steps, self.m0, self.n0, self.k0 = steps, 1 << initial_log_m, 1 << initial_log_n, initial_k
        self.dims = [(1 << a, 1 << b) for a, b in zip(log_m, log_n)]
        self.ks = list(ks)
        self.code0 = Code(self.m0)
        self.codes = [Code(m) for m, _ in self.dims]


def prove(cfg: Config, poly: list) -> dict:
    """prover (src/prover.rs:15-199) -> the proof's fields plus the
    challenges drawn, for comparison."""
    fs = FS(FS_SEED)
    s = S_QUERIES
    w0 = Witness(poly, cfg.m0, cfg.n0, cfg.code0)
    out = {"initial_root": w0.root, "recursive_roots": [], "recursive": [], "challenges": []}
    fs.absorb(w0.root)
    pe0 = [fs.get_field() for _ in range(cfg.k0)]
    out["challenges"] += pe0
    f = partial_eval(poly, pe0)
    w1 = Witness(f, cfg.dims[0][0], cfg.dims[0][1], cfg.codes[0])
    fs.absorb(w1.root)
    out["recursive_roots"].append(w1.root)
    queries = fs.get_distinct_queries(w0.num_rows, s)
    alpha = fs.get_field()
    out["challenges"].append(alpha)
    nv = len(f).bit_length() - 1
    sks = eval_sk_at_vks(1 << nv)
    rows = [w0.row(q) for q in queries]
    out["initial"] = (rows, merkle_prove(w0.tree, queries))
    basis, enforced = induce(nv, sks, rows, pe0, queries, alpha)
    sc = SumcheckProver(f, basis, enforced)
    fs.absorb(quad_bytes(sc.first))
    wprev = w1
    for i in range(cfg.steps):
        rs = []
        for _ in range(cfg.ks[i]):
            ri = fs.get_field()
            out["challenges"].append(ri)
            fs.absorb(quad_bytes(sc.fold(ri)))
            rs.append(ri)
        if i == cfg.steps - 1:
            fs.absorb(le_bytes(sc.f))
            queries = fs.get_distinct_queries(wprev.num_rows, s)
            rows = [wprev.row(q) for q in queries]
            out["yr"] = list(sc.f)
            out["final"] = (rows, merkle_prove(wprev.tree, queries))
            out["transcript"] = list(sc.transcript)
            return out
        wn = Witness(sc.f, cfg.dims[i + 1][0], cfg.dims[i + 1][1], cfg.codes[i + 1])
        fs.absorb(wn.root)
        out["recursive_roots"].append(wn.root)
        queries = fs.get_distinct_queries(wprev.num_rows, s)
        alpha = fs.get_field()
        out["challenges"].append(alpha)
        nv = len(sc.f).bit_length() - 1
        sks = eval_sk_at_vks(1 << nv)
        rows = [wprev.row(q) for q in queries]
        out["recursive"].append((rows, merkle_prove(wprev.tree, queries)))
        basis, enforced = induce(nv, sks, rows, rs, queries, alpha)
        fs.absorb(quad_bytes(sc.introduce_new(basis, enforced)))
        beta = fs.get_field()
        out["challenges"].append(beta)
        sc.glue(beta)
        wprev = wn
    raise AssertionError("prover completed without the final step")  # src/prover.rs:198


# ------------------------------------------------------------------ verifier
def quad_from_evals(at0, at1, atx, x=3):  # src/sumcheck.rs:67-81
    num = atx ^ at0 ^ gf_mul(x, at1 ^ at0)
    a = gf_mul(num, gf_inv(gf_mul(x, x) ^ x))
    return a, at1 ^ at0 ^ a, at0


def eval_quad(p, r):  # QuadraticPoly::eval_quadratic, src/sumcheck.rs:62-64
    a, b, c = p
    return gf_mul(gf_mul(a, r), r) ^ gf_mul(b, r) ^ c


class SumcheckVerifier:
    """SumcheckVerifierInstance (src/ligerito.rs:143-296); its assert_eq!s
    raise AssertionError (the reference panics)."""

    def __init__(self, b1, h1, transcript):
        self.basis, self.sep, self.sum = [b1], [1], h1
        self.tr, self.reader, self.ris, self.to_glue = list(transcript), 0, [], None
        g = self.read_tr()
        assert g[0] ^ g[1] == self.sum
        self.running = quad_from_evals(*g)
        self.first = g

    def read_tr(self):
        assert self.reader < len(self.tr)
        g = self.tr[self.reader]
        self.reader += 1
        return g

    def fold(self, r):
        self.ris.append(r)
        self.sum = eval_quad(self.running, r)
        g = self.read_tr()
        assert g[0] ^ g[1] == self.sum
        self.running = quad_from_evals(*g)
        return g

    def introduce_new(self, bi, h):
        g = self.read_tr()
        assert g[0] ^ g[1] == h
        self.basis.append(bi)
        self.to_glue = quad_from_evals(*g)
        return g

    def glue(self, alpha):  # fold_quadratic, src/sumcheck.rs:83-94
        self.sep.append(alpha)
        self.running = tuple(x ^ gf_mul(alpha, y) for x, y in zip(self.running, self.to_glue))

    def verify_partial(self, r, f_partial):
        k = len(f_partial).bit_length() - 1
        self.sum = eval_quad(self.running, r)
        self.ris.append(r)
        acc = partial_eval(self.basis[0], self.ris)
        for i in range(1, len(self.basis)):
            n = len(self.basis[i]).bit_length() - 1
            ev = partial_eval(self.basis[i], self.ris[len(self.ris) - (n - k):])
            assert len(acc) == len(ev)
            acc = [a ^ gf_mul(self.sep[i], b) for a, b in zip(acc, ev)]
        assert len(f_partial) == len(acc)
        return dotp(f_partial, acc) == self.sum


def verify(cfg: Config, P: dict) -> bool:
    """verifier (src/verifier.rs:10-164): the reference's bool, or
    AssertionError / IndexError where it panics."""
    fs = FS(FS_SEED)
    s = S_QUERIES
    log_inv_rate = 2
    fs.absorb(P["initial_root"])
    pe0 = [fs.get_field() for _ in range(cfg.k0)]
    fs.absorb(P["recursive_roots"][0])
    initial_dim = cfg.m0.bit_length() - 1
    depth = initial_dim + log_inv_rate
    queries = fs.get_distinct_queries(1 << depth, s)
    rows, mp = P["initial"]
    assert merkle_verify(P["initial_root"], mp, depth, [le_bytes(r) for r in rows], queries)
    alpha = fs.get_field()
    sks = eval_sk_at_vks(1 << initial_dim)
    basis, enforced = induce(initial_dim, sks, rows, pe0, queries, alpha)
    sv = SumcheckVerifier(basis, enforced, P["transcript"])
    fs.absorb(quad_bytes(sv.first))
    for i in range(cfg.steps):
        rs = []
        for _ in range(cfg.ks[i]):
            ri = fs.get_field()
            fs.absorb(quad_bytes(sv.fold(ri)))
            rs.append(ri)
        root = P["recursive_roots"][i]
        log_dim = cfg.dims[i][0].bit_length() - 1
        if i == cfg.steps - 1:
            yr = P["yr"]
            fs.absorb(le_bytes(yr))
            depth = log_dim + log_inv_rate
            queries = fs.get_distinct_queries(1 << depth, s)
            rows, mp = P["final"]
            assert merkle_verify(root, mp, depth, [le_bytes(r) for r in rows], queries)
            ligero_verify(queries, rows, yr, rs)
            final_r = fs.get_field()
            return sv.verify_partial(final_r, partial_eval(yr, [final_r]))
        fs.absorb(P["recursive_roots"][i + 1])
        depth = log_dim + log_inv_rate
        queries = fs.get_distinct_queries(1 << depth, s)
        rows, mp = P["recursive"][i]
        assert merkle_verify(root, mp, depth, [le_bytes(r) for r in rows], queries)
        alpha = fs.get_field()
        sks = eval_sk_at_vks(1 << log_dim)
        basis, enforced = induce(log_dim, sks, rows, rs, queries, alpha)
        fs.absorb(quad_bytes(sv.introduce_new(basis, enforced)))
        sv.glue(fs.get_field())
    raise AssertionError("verifier completed without the final step")  # src/verifier.rs:163


# ------------------------------------------------------------ wire format
def serialize(P: dict) -> bytes:
    """This project's proof encoding ("LGRP" v1, the field order of
    FinalizedLigeritoProof, src/data_structures.rs:91-103): u32 LE counts,
    LE words, length-prefixed byte strings."""
    out = bytearray(b"LGRP") + struct.pack("<II", 1, 4)

    def bstr(b):
        out.extend(struct.pack("<I", len(b)) + b)

    def words(w):
        out.extend(struct.pack("<I", len(w)) + le_bytes(w))

    def opening(o):
        rows, mp = o
        out.extend(struct.pack("<I", len(rows)))
        for r in rows:
            words(r)
        out.extend(struct.pack("<I", len(mp)))
        for h in mp:
            bstr(h)

    bstr(P["initial_root"])
    out.extend(struct.pack("<I", len(P["recursive_roots"])))
    for r in P["recursive_roots"]:
        bstr(r)
    opening(P["initial"])
    out.extend(struct.pack("<I", len(P["recursive"])))
    for o in P["recursive"]:
        opening(o)
    words(P["yr"])
    opening(P["final"])
    out.extend(struct.pack("<I", len(P["transcript"])))
    for t in P["transcript"]:
        out.extend(le_bytes(list(t)))
    return bytes(out)
