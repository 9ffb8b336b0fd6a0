/*
 * lgref.c -- CPU restatement of the Ligerito prover/verifier of
 * ashutosh1206/ligerito-rust.  TEST INFRASTRUCTURE ONLY: the parity oracle
 * for the CUDA path and the timed CPU baseline.  The shipped library never
 * links or calls this file.
 *
 * All citations are paths inside the reference project.  OpenMP marks the
 * places where the reference runs rayon; everything else is serial like the
 * reference.
 */
#include "lgref.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================
 * Small arena so the long prover/verifier bodies can bail out anywhere.
 * ==================================================================== */
typedef struct ablk { struct ablk *next; size_t pad; } ablk;
typedef struct { ablk *head; int oom; } arena;

static void *ar_alloc(arena *a, size_t n) {
    ablk *b = (ablk *)malloc(sizeof(ablk) + (n ? n : 1));
    if (!b) { a->oom = 1; return NULL; }
    b->next = a->head;
    a->head = b;
    return (void *)(b + 1);
}
static void ar_free(arena *a) {
    while (a->head) { ablk *n = a->head->next; free(a->head); a->head = n; }
}

/* ======================================================================
 * Binary fields.  src/binary_field.rs:13-189.
 * Elements of GF(2^16) and GF(2^32) live in uint32_t.
 * ==================================================================== */
static uint32_t irr_of(int bits) { return bits == 16 ? 0x2Du : 0x8299u; } /* :178, :181 */
static uint32_t mask_of(int bits) { return bits == 32 ? 0xFFFFFFFFu : ((1u << bits) - 1u); }

/* poly_multiply_gf2, src/binary_field.rs:83-105: shift-and-xor over the
   bits of b, carrying a's shifted copy across a (hi, lo) word pair. */
static inline void clmul_serial(int bits, uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
    const uint32_t m = mask_of(bits);
    uint32_t rh = 0, rl = 0, th = 0, tl = a, tb = b;
    while (tb != 0) {
        if (tb & 1u) { rl ^= tl; rh ^= th; }
        th = ((th << 1) | (tl >> (bits - 1))) & m;
        tl = (tl << 1) & m;
        tb >>= 1;
    }
    *hi = rh;
    *lo = rl;
}

/* mod_irreducible, src/binary_field.rs:52-81: walk the high word from its
   top bit down, folding each set bit back with the irreducible tail. */
static inline uint32_t reduce_serial(int bits, uint32_t hi, uint32_t lo) {
    const uint32_t m = mask_of(bits), irr = irr_of(bits);
    for (int i = 2 * bits - 1; i >= bits; --i) {
        int s = i - bits;
        if (hi & (1u << s)) {
            if (s == 0) {
                lo ^= irr;
            } else {
                hi ^= (irr >> (bits - s)) & m;
                lo ^= (irr << s) & m;
            }
        }
    }
    return lo;
}

static inline uint32_t gmul(int bits, uint32_t a, uint32_t b) { /* Mul, :132-140 */
    uint32_t hi, lo;
    clmul_serial(bits, a, b, &hi, &lo);
    return reduce_serial(bits, hi, lo);
}

uint32_t lgref_gf_mul(int bits, uint32_t a, uint32_t b) { return gmul(bits, a, b); }

/* pow, src/binary_field.rs:21-38 */
uint32_t lgref_gf_pow(int bits, uint32_t a, uint64_t e) {
    if (e == 0) return 1;
    uint32_t r = 1, base = a;
    while (e > 0) {
        if (e & 1) r = gmul(bits, r, base);
        base = gmul(bits, base, base);
        e >>= 1;
    }
    return r;
}

/* inverse, src/binary_field.rs:40-50 (Fermat: a^(2^k - 2)) */
int lgref_gf_inv(int bits, uint32_t a, uint32_t *out) {
    if (a == 0) return LGREF_PANIC;
    *out = lgref_gf_pow(bits, a, bits == 16 ? 65534ull : 4294967294ull);
    return LGREF_OK;
}

/* GF(2^128), irreducible x^128 + x^7 + x^2 + x + 1 (src/binary_field.rs:182-189).
   Only exercised by field-axiom tests; off the prove path. */
typedef unsigned __int128 u128;
static u128 gmul128(u128 a, u128 b) {
    u128 rh = 0, rl = 0, th = 0, tl = a, tb = b;
    while (tb != 0) {
        if (tb & 1) { rl ^= tl; rh ^= th; }
        th = (th << 1) | (tl >> 127);
        tl <<= 1;
        tb >>= 1;
    }
    const u128 irr = 0x87;
    for (int i = 255; i >= 128; --i) {
        int s = i - 128;
        if ((rh >> s) & 1) {
            if (s == 0) rl ^= irr;
            else { rh ^= irr >> (128 - s); rl ^= irr << s; }
        }
    }
    return rl;
}
static u128 ld128(const uint64_t v[2]) { return ((u128)v[1] << 64) | v[0]; }
static void st128(u128 x, uint64_t v[2]) { v[0] = (uint64_t)x; v[1] = (uint64_t)(x >> 64); }
void lgref_gf128_mul(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]) {
    st128(gmul128(ld128(a), ld128(b)), out);
}
int lgref_gf128_inv(const uint64_t a[2], uint64_t out[2]) {
    u128 x = ld128(a);
    if (x == 0) return LGREF_PANIC;
    u128 e = ~(u128)0 - 1; /* 2^128 - 2 */
    u128 r = 1, base = x;
    while (e > 0) {
        if (e & 1) r = gmul128(r, base);
        base = gmul128(base, base);
        e >>= 1;
    }
    st128(r, out);
    return LGREF_OK;
}

/* ======================================================================
 * Additive FFT.  src/binary_fft.rs.
 * ==================================================================== */
static inline uint32_t next_s(int bits, uint32_t s_prev, uint32_t s_prev_at_root) {
    /* :100-107  s^2 + s_root * s */
    return gmul(bits, s_prev, s_prev) ^ gmul(bits, s_prev_at_root, s_prev);
}

/* compute_twiddles with beta = 0, :30-58 (layer_0 :60-72, layer_i :74-89,
   compute_s_at_root :91-98).  Heap order: node idx (1-based) -> out[idx-1]. */
void lgref_compute_twiddles(int bits, int log_n, uint32_t *tw) {
    size_t layer_size = (size_t)1 << (log_n - 1);
    uint32_t *layer = (uint32_t *)calloc(layer_size, sizeof(uint32_t));
    size_t write_at = layer_size;
    for (size_t i = 0; i < layer_size; ++i) layer[i] = (uint32_t)(i << 1); /* beta + 2i */
    uint32_t s_prev_at_root = 1;
    memcpy(tw + (write_at - 1), layer, layer_size * sizeof(uint32_t));
    for (int it = 0; it < log_n - 1; ++it) {
        write_at >>= 1;
        layer_size = write_at;
        uint32_t s_at_root = next_s(bits, layer[1] ^ layer[0], s_prev_at_root);
        for (size_t w = 0; w < layer_size; ++w) layer[w] = next_s(bits, layer[2 * w], s_prev_at_root);
        s_prev_at_root = s_at_root;
        uint32_t s_inv = 0;
        lgref_gf_inv(bits, s_prev_at_root, &s_inv);
        for (size_t i = 0; i < layer_size; ++i) tw[write_at + i - 1] = gmul(bits, s_inv, layer[i]);
    }
    free(layer);
}

/* fft_mul, :180-192 */
static void fft_mul(int bits, uint32_t *v, size_t n, uint32_t lambda) {
    size_t h = n / 2;
    uint32_t *u = v, *w = v + h;
    for (size_t i = 0; i < h; ++i) {
        u[i] ^= gmul(bits, lambda, w[i]);
        w[i] ^= u[i];
    }
}
/* ifft_mul, :194-206 */
static void ifft_mul(int bits, uint32_t *v, size_t n, uint32_t lambda) {
    size_t h = n / 2;
    uint32_t *u = v, *w = v + h;
    for (size_t i = 0; i < h; ++i) {
        w[i] ^= u[i];
        u[i] ^= gmul(bits, lambda, w[i]);
    }
}

/* fft_twiddles / fft_twiddles_parallel, :109-159.  `depth` plays the role
   of rayon's thread_depth (ilog2 of the pool size). */
static void fft_rec(int bits, uint32_t *v, size_t n, const uint32_t *tw, size_t idx, int depth) {
    if (n == 1) return;
    fft_mul(bits, v, n, tw[idx - 1]);
    size_t h = n / 2;
    if (depth > 0) {
#pragma omp task
        fft_rec(bits, v, h, tw, 2 * idx, depth - 1);
        fft_rec(bits, v + h, h, tw, 2 * idx + 1, depth - 1);
#pragma omp taskwait
    } else {
        fft_rec(bits, v, h, tw, 2 * idx, 0);
        fft_rec(bits, v + h, h, tw, 2 * idx + 1, 0);
    }
}

/* ifft_twiddles, :161-178 (children first, then the butterfly) */
static void ifft_rec(int bits, uint32_t *v, size_t n, const uint32_t *tw, size_t idx) {
    if (n == 1) return;
    size_t h = n / 2;
    ifft_rec(bits, v, h, tw, 2 * idx);
    ifft_rec(bits, v + h, h, tw, 2 * idx + 1);
    ifft_mul(bits, v, n, tw[idx - 1]);
}

static int ilog2_int(int x) { int r = 0; while (x > 1) { x >>= 1; ++r; } return r; }

/* fft, :4-17.  Both flag values run the same butterflies; the parallel one
   only changes scheduling. */
void lgref_fft(int bits, uint32_t *v, size_t n, const uint32_t *tw, int nthreads) {
    if (nthreads <= 1) { fft_rec(bits, v, n, tw, 1, 0); return; }
#pragma omp parallel num_threads(nthreads)
#pragma omp single
    fft_rec(bits, v, n, tw, 1, ilog2_int(nthreads));
}

/* ifft, :19-28 */
void lgref_ifft(int bits, uint32_t *v, size_t n, const uint32_t *tw) { ifft_rec(bits, v, n, tw, 1); }

static int log2_sz(size_t n) { int r = 0; while (n > 1) { n >>= 1; ++r; } return r; }
static int is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; } /* :213-215 */

/* eval_sk_at_vks, :217-246 */
void lgref_eval_sk_at_vks(int bits, size_t n, uint32_t *sk) {
    int ns = log2_sz(n);
    uint32_t *layer = (uint32_t *)malloc((ns + 1) * sizeof(uint32_t));
    for (int i = 1; i <= ns; ++i) layer[i - 1] = (uint32_t)1u << i;
    sk[0] = 1;
    int cur_len = ns;
    for (int i = 1; i <= ns; ++i) {
        for (int j = 1; j <= cur_len; ++j) {
            if (j == 1)
                sk[i] = gmul(bits, layer[0], layer[0]) ^ gmul(bits, sk[i - 1], layer[0]);
            else
                layer[j - 2] = gmul(bits, layer[j - 1], layer[j - 1]) ^ gmul(bits, sk[i - 1], layer[j - 1]);
        }
        --cur_len;
    }
    free(layer);
}

/* evaluate_scaled_basis_inplace, :276-301 (evaluate_basis :248-274 is the
   alpha = 1 case). sks_at_x needs log2(len) entries. */
static void scaled_basis(int bits, uint32_t *sks_at_x, uint32_t *basis, size_t len,
                         const uint32_t *sks_vks, uint32_t x, uint32_t alpha) {
    int ns = log2_sz(len);
    sks_at_x[0] = x;
    for (int i = 2; i <= ns; ++i) sks_at_x[i - 1] = next_s(bits, sks_at_x[i - 2], sks_vks[i - 2]);
    basis[0] = alpha;
    for (int i = 1; i <= ns; ++i) {
        size_t cur = (size_t)1 << (i - 1);
        for (size_t j = 1; j <= cur; ++j) basis[j + cur - 1] = gmul(bits, sks_at_x[i - 1], basis[j - 1]);
    }
}

void lgref_evaluate_basis(int bits, size_t basis_len, const uint32_t *sks_vks, uint32_t x,
                          uint32_t *out) {
    uint32_t sx[64];
    scaled_basis(bits, sx, out, basis_len, sks_vks, x, 1);
}

/* compute_pis, :303-322 */
void lgref_compute_pis(int bits, size_t pis_len, const uint32_t *sks_vks, uint32_t *pis) {
    int nsk = log2_sz(pis_len) + 1;
    pis[0] = 1;
    for (int i = 2; i <= nsk; ++i) {
        size_t cur = (size_t)1 << (i - 2);
        for (size_t j = 1; j <= cur; ++j) pis[j + cur - 1] = gmul(bits, sks_vks[i - 2], pis[j - 1]);
    }
}

/* ======================================================================
 * Reed-Solomon.  src/reed_solomon.rs.
 * ==================================================================== */
/* short_from_long_tw, :19-41 */
void lgref_short_from_long_tw(const uint32_t *l_tw, int n, int k, uint32_t *s_tw) {
    size_t jump = (size_t)1 << (n - k);
    s_tw[0] = l_tw[jump - 1];
    size_t idx = 2;
    for (int i = 1; i < k; ++i) {
        jump *= 2;
        size_t take = (size_t)1 << i;
        for (size_t j = 0; j < take; ++j) s_tw[idx + j - 1] = l_tw[jump + j - 1];
        idx += take;
    }
}

typedef struct {
    int bits, log_msg, log_block;
    uint32_t *twiddles; /* 2^log_block - 1 */
    uint32_t *pis;      /* 2^log_msg */
} rs_code;

/* ReedSolomonEncoding::new, :49-64 */
static int rs_new(rs_code *rs, int bits, size_t msg_len, size_t block_len, arena *a) {
    if (!is_pow2(msg_len) || !is_pow2(block_len) || msg_len >= block_len) return LGREF_PANIC;
    rs->bits = bits;
    rs->log_msg = log2_sz(msg_len);
    rs->log_block = log2_sz(block_len);
    rs->twiddles = (uint32_t *)ar_alloc(a, (block_len - 1) * sizeof(uint32_t) + 4);
    rs->pis = (uint32_t *)ar_alloc(a, msg_len * sizeof(uint32_t));
    uint32_t *sk = (uint32_t *)ar_alloc(a, (rs->log_msg + 1) * sizeof(uint32_t));
    if (!rs->twiddles || !rs->pis || !sk) return LGREF_OOM;
    lgref_compute_twiddles(bits, rs->log_block, rs->twiddles);
    lgref_eval_sk_at_vks(bits, msg_len, sk);
    lgref_compute_pis(bits, msg_len, sk, rs->pis);
    return LGREF_OK;
}

/* encode_non_systematic, :104-113 (the column task of encode_cols) */
static void rs_encode_ns(const rs_code *rs, uint32_t *v, int depth) {
    size_t m = (size_t)1 << rs->log_msg, blk = (size_t)1 << rs->log_block;
    for (size_t i = 0; i < m; ++i) v[i] = gmul(rs->bits, v[i], rs->pis[i]);
    fft_rec(rs->bits, v, blk, rs->twiddles, 1, depth);
}

int lgref_rs_encode_non_systematic(int bits, uint32_t *v, size_t msg_len, size_t block_len,
                                   int nthreads) {
    arena a = {0};
    rs_code rs;
    int st = rs_new(&rs, bits, msg_len, block_len, &a);
    if (st == LGREF_OK) {
        if (nthreads <= 1) {
            rs_encode_ns(&rs, v, 0);
        } else {
#pragma omp parallel num_threads(nthreads)
#pragma omp single
            rs_encode_ns(&rs, v, ilog2_int(nthreads));
        }
    }
    ar_free(&a);
    return st;
}

/* encode (systematic), :90-102 */
int lgref_rs_encode(int bits, const uint32_t *msg, size_t msg_len, size_t block_len,
                    uint32_t *out) {
    arena a = {0};
    rs_code rs;
    int st = rs_new(&rs, bits, msg_len, block_len, &a);
    if (st == LGREF_OK) {
        memset(out, 0, block_len * sizeof(uint32_t));
        memcpy(out, msg, msg_len * sizeof(uint32_t));
        uint32_t *s_tw = (uint32_t *)ar_alloc(&a, msg_len * sizeof(uint32_t));
        lgref_short_from_long_tw(rs.twiddles, rs.log_block, rs.log_msg, s_tw);
        ifft_rec(bits, out, msg_len, s_tw, 1);
        fft_rec(bits, out, block_len, rs.twiddles, 1, 0);
    }
    ar_free(&a);
    return st;
}

/* ======================================================================
 * SHA-256 (FIPS 180-4).  The reference calls sha2 0.10.9
 * (src/emulated_fs.rs:2,13-31); restated from the standard.
 * ==================================================================== */
typedef struct {
    uint32_t h[8];
    uint8_t buf[64];
    uint64_t total;
    size_t n;
} sha256_st;

static const uint32_t SHA_K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static inline uint32_t ror32(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }

static void sha_block(uint32_t h[8], const uint8_t *p) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
        w[i] = ((uint32_t)p[4 * i] << 24) | ((uint32_t)p[4 * i + 1] << 16) |
               ((uint32_t)p[4 * i + 2] << 8) | p[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
        uint32_t s0 = ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
        uint32_t S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = hh + S1 + ch + SHA_K[i] + w[i];
        uint32_t S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint32_t t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

static void sha_init(sha256_st *s) {
    static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    memcpy(s->h, iv, sizeof iv);
    s->total = 0;
    s->n = 0;
}

static void sha_update(sha256_st *s, const uint8_t *p, size_t len) {
    s->total += len;
    while (len > 0) {
        size_t take = 64 - s->n;
        if (take > len) take = len;
        memcpy(s->buf + s->n, p, take);
        s->n += take;
        p += take;
        len -= take;
        if (s->n == 64) { sha_block(s->h, s->buf); s->n = 0; }
    }
}

static void sha_final(const sha256_st *in, uint8_t out[32]) { /* finalizes a copy */
    sha256_st s = *in;
    uint64_t bitlen = s.total * 8;
    uint8_t pad = 0x80;
    sha_update(&s, &pad, 1);
    uint8_t z = 0;
    while (s.n != 56) sha_update(&s, &z, 1);
    uint8_t lenb[8];
    for (int i = 0; i < 8; ++i) lenb[i] = (uint8_t)(bitlen >> (56 - 8 * i));
    sha_update(&s, lenb, 8);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(s.h[i] >> 24);
        out[4 * i + 1] = (uint8_t)(s.h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(s.h[i] >> 8);
        out[4 * i + 3] = (uint8_t)s.h[i];
    }
}

void lgref_sha256(const uint8_t *msg, size_t len, uint8_t out[32]) {
    sha256_st s;
    sha_init(&s);
    sha_update(&s, msg, len);
    sha_final(&s, out);
}

/* ======================================================================
 * BLAKE3 (hash mode), restated from the BLAKE3 specification.  The
 * reference calls blake3 1.8.2 `blake3::hash` / `Hasher`
 * (src/merkle_tree.rs:15,50,113-118,176).
 * ==================================================================== */
static const uint32_t B3_IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                  0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
static const uint8_t B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
enum { B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_PARENT = 4, B3_ROOT = 8 };

static inline void b3_g(uint32_t *v, int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] = v[a] + v[b] + x;
    v[d] = ror32(v[d] ^ v[a], 16);
    v[c] = v[c] + v[d];
    v[b] = ror32(v[b] ^ v[c], 12);
    v[a] = v[a] + v[b] + y;
    v[d] = ror32(v[d] ^ v[a], 8);
    v[c] = v[c] + v[d];
    v[b] = ror32(v[b] ^ v[c], 7);
}

static void b3_compress(const uint32_t cv[8], const uint32_t blk[16], uint64_t counter,
                        uint32_t blen, uint32_t flags, uint32_t out[16]) {
    uint32_t v[16], m[16], t[16];
    memcpy(v, cv, 32);
    memcpy(v + 8, B3_IV, 16);
    v[12] = (uint32_t)counter;
    v[13] = (uint32_t)(counter >> 32);
    v[14] = blen;
    v[15] = flags;
    memcpy(m, blk, 64);
    for (int r = 0; r < 7; ++r) {
        b3_g(v, 0, 4, 8, 12, m[0], m[1]);
        b3_g(v, 1, 5, 9, 13, m[2], m[3]);
        b3_g(v, 2, 6, 10, 14, m[4], m[5]);
        b3_g(v, 3, 7, 11, 15, m[6], m[7]);
        b3_g(v, 0, 5, 10, 15, m[8], m[9]);
        b3_g(v, 1, 6, 11, 12, m[10], m[11]);
        b3_g(v, 2, 7, 8, 13, m[12], m[13]);
        b3_g(v, 3, 4, 9, 14, m[14], m[15]);
        for (int i = 0; i < 16; ++i) t[i] = m[B3_PERM[i]];
        memcpy(m, t, 64);
    }
    for (int i = 0; i < 8; ++i) {
        out[i] = v[i] ^ v[i + 8];
        out[i + 8] = v[i + 8] ^ cv[i];
    }
}

static void b3_load_block(const uint8_t *p, size_t len, uint32_t blk[16]) {
    uint8_t tmp[64];
    memset(tmp, 0, 64);
    memcpy(tmp, p, len);
    for (int i = 0; i < 16; ++i)
        blk[i] = (uint32_t)tmp[4 * i] | ((uint32_t)tmp[4 * i + 1] << 8) |
                 ((uint32_t)tmp[4 * i + 2] << 16) | ((uint32_t)tmp[4 * i + 3] << 24);
}

typedef struct { uint32_t cv[8]; uint32_t blk[16]; uint64_t counter; uint32_t blen, flags; } b3_out;

static void b3_chunk_output(const uint8_t *p, size_t len, uint64_t chunk_idx, b3_out *o) {
    uint32_t cv[8], blk[16], res[16];
    memcpy(cv, B3_IV, 32);
    size_t nblocks = len == 0 ? 1 : (len + 63) / 64;
    for (size_t b = 0; b + 1 < nblocks; ++b) {
        b3_load_block(p + 64 * b, 64, blk);
        b3_compress(cv, blk, chunk_idx, 64, b == 0 ? B3_CHUNK_START : 0, res);
        memcpy(cv, res, 32);
    }
    size_t last = len - 64 * (nblocks - 1);
    memcpy(o->cv, cv, 32);
    b3_load_block(p + 64 * (nblocks - 1), last, o->blk);
    o->counter = chunk_idx;
    o->blen = (uint32_t)last;
    o->flags = (nblocks == 1 ? B3_CHUNK_START : 0) | B3_CHUNK_END;
}

static void b3_out_cv(const b3_out *o, uint32_t cv[8]) {
    uint32_t res[16];
    b3_compress(o->cv, o->blk, o->counter, o->blen, o->flags, res);
    memcpy(cv, res, 32);
}

static void b3_parent(const uint32_t l[8], const uint32_t r[8], b3_out *o) {
    memcpy(o->cv, B3_IV, 32);
    memcpy(o->blk, l, 32);
    memcpy(o->blk + 8, r, 32);
    o->counter = 0;
    o->blen = 64;
    o->flags = B3_PARENT;
}

void lgref_blake3(const uint8_t *msg, size_t len, uint8_t out[32]) {
    uint32_t stack[64][8];
    int sp = 0;
    size_t nchunks = len == 0 ? 1 : (len + 1023) / 1024;
    for (size_t c = 0; c + 1 < nchunks; ++c) {
        b3_out o;
        uint32_t cv[8];
        b3_chunk_output(msg + 1024 * c, 1024, c, &o);
        b3_out_cv(&o, cv);
        uint64_t total = c + 1; /* merge completed subtrees (lazy: last chunk kept) */
        while ((total & 1) == 0) {
            b3_out po;
            b3_parent(stack[--sp], cv, &po);
            b3_out_cv(&po, cv);
            total >>= 1;
        }
        memcpy(stack[sp++], cv, 32);
    }
    b3_out o;
    b3_chunk_output(msg + 1024 * (nchunks - 1), len - 1024 * (nchunks - 1), nchunks - 1, &o);
    while (sp > 0) {
        uint32_t cv[8];
        b3_out_cv(&o, cv);
        b3_parent(stack[--sp], cv, &o);
    }
    uint32_t res[16];
    b3_compress(o.cv, o.blk, 0, o.blen, o.flags | B3_ROOT, res);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)res[i];
        out[4 * i + 1] = (uint8_t)(res[i] >> 8);
        out[4 * i + 2] = (uint8_t)(res[i] >> 16);
        out[4 * i + 3] = (uint8_t)(res[i] >> 24);
    }
}

/* ======================================================================
 * Merkle tree.  src/merkle_tree.rs.  Layers are stored back to back,
 * leaves first, each node 32 bytes.
 * ==================================================================== */
/* The reference hashes with blake3 (:15,:50,:114,:176).  Its Merkle KATs
   (:206-209, :223-232, :248-251) are SHA-256 values carried over from the
   Julia port, so the hash is a parameter: LGREF_HASH_SHA256 replays those
   KATs and pins the layout / multi-proof order; the prover uses BLAKE3. */
static void hash_any(int kind, const uint8_t *m, size_t len, uint8_t out[32]) {
    if (kind == LGREF_HASH_SHA256) lgref_sha256(m, len, out);
    else lgref_blake3(m, len, out);
}
static void hash_pair(int kind, const uint8_t *l, const uint8_t *r, uint8_t out[32]) { /* :113-118 */
    uint8_t c[64];
    memcpy(c, l, 32);
    memcpy(c + 32, r, 32);
    hash_any(kind, c, 64, out);
}

/* build_merkle_tree, :22-60.  hash_array (:4-20) and the layer loop are
   serial in the reference. */
int lgref_merkle_build(int kind, const uint8_t *buf, const size_t *off, size_t nl, uint8_t *tree) {
    if (!is_pow2(nl)) return LGREF_PANIC;
    for (size_t i = 0; i < nl; ++i) hash_any(kind, buf + off[i], off[i + 1] - off[i], tree + 32 * i);
    uint8_t *cur = tree;
    size_t cn = nl;
    while (cn > 1) {
        size_t nn = (cn + 1) / 2;
        uint8_t *nxt = cur + 32 * cn;
        for (size_t i = 0; i < nn; ++i) hash_pair(kind, cur + 64 * i, cur + 64 * i + 32, nxt + 32 * i);
        cur = nxt;
        cn = nn;
    }
    return LGREF_OK;
}

/* prove / ith_layer, :62-111 */
int lgref_merkle_prove(const uint8_t *tree, size_t nl, const size_t *queries, size_t nq,
                       uint8_t *sib, size_t cap, size_t *n_sib) {
    size_t *q = (size_t *)malloc((nq ? nq : 1) * sizeof(size_t));
    memcpy(q, queries, nq * sizeof(size_t));
    size_t depth = (size_t)log2_sz(nl), cnt = nq, np = 0, lsize = nl;
    const uint8_t *layer = tree;
    int st = LGREF_OK;
    for (size_t d = 0; d < depth && st == LGREF_OK; ++d) {
        size_t next = 0, i = 0;
        while (i < cnt) {
            size_t query = q[i], sibling = query ^ 1;
            ++next;
            q[next - 1] = query >> 1;
            if (sibling >= lsize || np >= cap) { st = LGREF_PANIC; break; }
            const uint8_t *sh = layer + 32 * sibling;
            if (i == cnt - 1) { memcpy(sib + 32 * np++, sh, 32); break; }
            if (query % 2 != 0) { memcpy(sib + 32 * np++, sh, 32); i += 1; }
            else if (q[i + 1] != sibling) { memcpy(sib + 32 * np++, sh, 32); i += 1; }
            else { i += 2; }
        }
        cnt = next;
        layer += 32 * lsize;
        lsize = (lsize + 1) / 2;
    }
    free(q);
    *n_sib = np;
    return st;
}

/* verify / verify_ith_layer, :120-188.  Out-of-range proof reads panic in
   the reference; here they return PANIC. */
static int merkle_verify_hashed(int kind, const uint8_t root[32], const uint8_t *sibs, size_t n_sib,
                                size_t depth, uint8_t *layer /* nq*32, clobbered */,
                                const size_t *queries, size_t nq, int *ok) {
    size_t *q = (size_t *)malloc((nq ? nq : 1) * sizeof(size_t));
    memcpy(q, queries, nq * sizeof(size_t));
    size_t cur = nq, pc = 0;
    int st = LGREF_OK;
    for (size_t d = 0; d < depth && st == LGREF_OK; ++d) {
        size_t next = 0, i = 0;
        while (i < cur) {
            size_t query = q[i], sibling = query ^ 1;
            ++next;
            q[next - 1] = query >> 1;
            uint8_t h[32];
            if (i == cur - 1) {
                ++pc;
                if (pc - 1 >= n_sib) { st = LGREF_PANIC; break; }
                if (query % 2 != 0) hash_pair(kind, sibs + 32 * (pc - 1), layer + 32 * i, h);
                else hash_pair(kind, layer + 32 * i, sibs + 32 * (pc - 1), h);
                memcpy(layer + 32 * (next - 1), h, 32);
                break;
            }
            if (query % 2 != 0) {
                ++pc;
                if (pc - 1 >= n_sib) { st = LGREF_PANIC; break; }
                hash_pair(kind, sibs + 32 * (pc - 1), layer + 32 * i, h);
                memcpy(layer + 32 * (next - 1), h, 32);
                i += 1;
            } else if (q[i + 1] != sibling) {
                ++pc;
                if (pc - 1 >= n_sib) { st = LGREF_PANIC; break; }
                hash_pair(kind, layer + 32 * i, sibs + 32 * (pc - 1), h);
                memcpy(layer + 32 * (next - 1), h, 32);
                i += 1;
            } else {
                hash_pair(kind, layer + 32 * i, layer + 32 * (i + 1), h);
                memcpy(layer + 32 * (next - 1), h, 32);
                i += 2;
            }
        }
        cur = next;
    }
    free(q);
    *ok = (st == LGREF_OK) && cur == 1 && memcmp(layer, root, 32) == 0;
    return st;
}

int lgref_merkle_verify(int kind, const uint8_t root[32], const uint8_t *sibs, size_t n_sib,
                        size_t depth, const uint8_t *buf, const size_t *off, const size_t *queries,
                        size_t nq, int *ok) {
    uint8_t *layer = (uint8_t *)malloc(32 * (nq ? nq : 1));
    for (size_t i = 0; i < nq; ++i) hash_any(kind, buf + off[i], off[i + 1] - off[i], layer + 32 * i);
    int st = merkle_verify_hashed(kind, root, sibs, n_sib, depth, layer, queries, nq, ok);
    free(layer);
    return st;
}

/* ======================================================================
 * Ligero.  src/ligero.rs.
 * ==================================================================== */
/* extract_leaves (:53-68, rayon over rows) + build_merkle_tree (serial). */
static int commit_tree(const uint32_t *flat, size_t rows, size_t n, uint8_t *tree, int nthreads) {
    size_t lb = 4 * n;
    uint8_t *leaves = (uint8_t *)malloc(rows * lb);
    size_t *off = (size_t *)malloc((rows + 1) * sizeof(size_t));
    if (!leaves || !off) { free(leaves); free(off); return LGREF_OOM; }
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
    for (long long r = 0; r < (long long)rows; ++r) {
        uint8_t *p = leaves + (size_t)r * lb;
        for (size_t j = 0; j < n; ++j) {
            uint32_t v = flat[j * rows + (size_t)r];
            p[4 * j] = (uint8_t)v;
            p[4 * j + 1] = (uint8_t)(v >> 8);
            p[4 * j + 2] = (uint8_t)(v >> 16);
            p[4 * j + 3] = (uint8_t)(v >> 24);
        }
    }
    for (size_t i = 0; i <= rows; ++i) off[i] = i * lb;
    int st = lgref_merkle_build(LGREF_HASH_BLAKE3, leaves, off, rows, tree);
    free(leaves);
    free(off);
    return st;
}

/* poly2flatmat (:11-27) + encode_cols (:29-38, rayon over columns, each
   column's FFT itself rayon-split) */
static void encode_matrix(const rs_code *rs, const uint32_t *poly, size_t m, size_t n,
                          uint32_t *flat, int nthreads) {
    size_t mt = 4 * m;
    for (size_t j = 0; j < n; ++j) {
        memcpy(flat + j * mt, poly + j * m, m * sizeof(uint32_t));
        memset(flat + j * mt + m, 0, (mt - m) * sizeof(uint32_t));
    }
    if (nthreads <= 1) {
        for (size_t j = 0; j < n; ++j) rs_encode_ns(rs, flat + j * mt, 0);
        return;
    }
    int depth = ilog2_int(nthreads);
#pragma omp parallel num_threads(nthreads)
#pragma omp single
    for (size_t j = 0; j < n; ++j) {
#pragma omp task firstprivate(j)
        rs_encode_ns(rs, flat + j * mt, depth);
    }
}

/* ligero_commit, :70-95 */
int lgref_ligero_commit(const uint32_t *poly, size_t m, size_t n, uint32_t *flat,
                        uint8_t *tree, int nthreads) {
    arena a = {0};
    rs_code rs;
    int st = rs_new(&rs, 32, m, 4 * m, &a);
    if (st == LGREF_OK) {
        encode_matrix(&rs, poly, m, n, flat, nthreads);
        st = commit_tree(flat, 4 * m, n, tree, nthreads);
    }
    ar_free(&a);
    return st;
}

/* evaluate_lagrange_basis, src/utils.rs:4-27 (rs[0] ends up the MSB) */
void lgref_lagrange_basis(const uint32_t *rs, size_t k, uint32_t *out) {
    out[0] = 1u ^ rs[0];
    out[1] = rs[0];
    size_t len = 2;
    uint32_t *tmp = (uint32_t *)malloc(((size_t)1 << k) * sizeof(uint32_t));
    for (size_t i = 1; i < k; ++i) {
        uint32_t rp1 = 1u ^ rs[i];
        for (size_t j = 0; j < len; ++j) {
            tmp[2 * j] = gmul(32, out[j], rp1);
            tmp[2 * j + 1] = gmul(32, out[j], rs[i]);
        }
        len *= 2;
        memcpy(out, tmp, len * sizeof(uint32_t));
    }
    free(tmp);
}

/* ligero_verify, src/ligero.rs:97-131 (panics on mismatch).  Rows are
   given as pointers + lengths because `zip` truncates ragged rows. */
static int ligero_verify_core(const size_t *queries, size_t nrows, const uint32_t *const *rows,
                              const uint32_t *rlen, const uint32_t *yr, size_t yr_len,
                              const uint32_t *ch, size_t nch) {
    if (nch == 0 || !is_pow2(yr_len)) return LGREF_PANIC;
    size_t glen = (size_t)1 << nch;
    uint32_t *gr = (uint32_t *)malloc(glen * 4);
    lgref_lagrange_basis(ch, nch, gr);
    int nlog = log2_sz(yr_len);
    uint32_t *sk = (uint32_t *)malloc((nlog + 1) * 4);
    lgref_eval_sk_at_vks(32, yr_len, sk);
    uint32_t *basis = (uint32_t *)malloc(yr_len * 4);
    uint32_t sx[64];
    int st = LGREF_OK;
    for (size_t i = 0; i < nrows; ++i) {
        size_t zl = rlen[i] < glen ? rlen[i] : glen;
        uint32_t dot = 0;
        for (size_t j = 0; j < zl; ++j) dot ^= gmul(32, rows[i][j], gr[j]);
        if (queries[i] > 0xFFFFFFFFull) { st = LGREF_PANIC; break; }
        scaled_basis(32, sx, basis, yr_len, sk, (uint32_t)queries[i], 1);
        uint32_t e = 0;
        for (size_t j = 0; j < yr_len; ++j) e ^= gmul(32, yr[j], basis[j]);
        if (e != dot) { st = LGREF_PANIC; break; }
    }
    free(gr);
    free(sk);
    free(basis);
    return st;
}

int lgref_ligero_verify(const size_t *queries, const uint32_t *rows, size_t nrows, size_t row_len,
                        const uint32_t *yr, size_t yr_len, const uint32_t *ch, size_t nch) {
    const uint32_t **rp = (const uint32_t **)malloc((nrows + 1) * sizeof(uint32_t *));
    uint32_t *rl = (uint32_t *)malloc((nrows + 1) * 4);
    for (size_t i = 0; i < nrows; ++i) { rp[i] = rows + i * row_len; rl[i] = (uint32_t)row_len; }
    int st = ligero_verify_core(queries, nrows, rp, rl, yr, yr_len, ch, nch);
    free(rp);
    free(rl);
    return st;
}

/* ======================================================================
 * Multilinear polynomials + sumcheck.  src/multilinear_poly.rs,
 * src/sumcheck_polys.rs, src/sumcheck.rs, src/ligerito.rs.
 * ==================================================================== */
/* partial_eval, src/multilinear_poly.rs:66-87: the top variable folds
   first; the first pass is serial, later passes rayon-parallel. */
static void partial_eval_core(const uint32_t *ev, size_t len, const uint32_t *rs, size_t k,
                              uint32_t *tmp, int nthreads) {
    size_t n = len / 2;
    uint32_t r0 = rs[0], r0p1 = 1u ^ rs[0];
    for (size_t i = 0; i < n; ++i) tmp[i] = gmul(32, r0p1, ev[i]) ^ gmul(32, r0, ev[i + n]);
    for (size_t t = 1; t < k; ++t) {
        n /= 2;
        uint32_t r = rs[t], rp1 = 1u ^ rs[t];
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static) if (nthreads > 1)
        for (long long i = 0; i < (long long)n; ++i)
            tmp[i] = gmul(32, rp1, tmp[i]) ^ gmul(32, r, tmp[i + n]);
    }
}

int lgref_partial_eval(const uint32_t *ev, size_t len, const uint32_t *rs, size_t k, uint32_t *out,
                       int nthreads) {
    if (k == 0 || !is_pow2(len) || (len >> k) == 0) return LGREF_PANIC;
    uint32_t *tmp = (uint32_t *)malloc((len / 2) * 4);
    if (!tmp) return LGREF_OOM;
    partial_eval_core(ev, len, rs, k, tmp, nthreads);
    memcpy(out, tmp, (len >> k) * 4);
    free(tmp);
    return LGREF_OK;
}

/* eval_013_product, src/multilinear_poly.rs:90-131 (x = 3) */
void lgref_eval_013_product(const uint32_t *f, const uint32_t *g, size_t len, uint32_t out[3]) {
    size_t h = len / 2;
    uint32_t s0 = 0, s1 = 0, s2 = 0;
    const uint32_t three = 3, one_p_three = 1u ^ 3u;
    for (size_t i = 0; i < h; ++i) s0 ^= gmul(32, f[i], g[i]);
    for (size_t i = 0; i < h; ++i) s1 ^= gmul(32, f[h + i], g[h + i]);
    for (size_t i = 0; i < h; ++i) {
        uint32_t f2 = gmul(32, f[h + i], three) ^ gmul(32, one_p_three, f[i]);
        uint32_t g2 = gmul(32, g[h + i], three) ^ gmul(32, one_p_three, g[i]);
        s2 ^= gmul(32, f2, g2);
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
}

/* induce_sumcheck_poly_parallel, src/sumcheck_polys.rs:74-160, with
   precompute_alpha_powers (:6-20) and evaluate_scaled_basis_inplace.
   rayon's fold/reduce becomes per-thread accumulators XOR-reduced. */
int lgref_induce_sumcheck_poly(size_t n, const uint32_t *sks_vks, const uint32_t *rows,
                               size_t nrows, size_t row_len, const uint32_t *v_ch, size_t nch,
                               const size_t *queries, uint32_t alpha, uint32_t *basis_out,
                               uint32_t *enforced_sum, int nthreads) {
    if (nch == 0) return LGREF_PANIC;
    size_t glen = (size_t)1 << nch;
    if (row_len != glen) return LGREF_PANIC; /* :97 */
    size_t blen = (size_t)1 << n;
    for (size_t i = 0; i < nrows; ++i)
        if (queries[i] > 0xFFFFFFFFull) return LGREF_PANIC; /* try_from, :116 */
    uint32_t *gr = (uint32_t *)malloc(glen * 4);
    lgref_lagrange_basis(v_ch, nch, gr);
    uint32_t *apow = (uint32_t *)malloc((nrows ? nrows : 1) * 4);
    if (nrows) apow[0] = 1;
    for (size_t i = 1; i < nrows; ++i) apow[i] = gmul(32, apow[i - 1], alpha);
    memset(basis_out, 0, blen * 4);
    uint32_t total = 0;
    int nt = nthreads > 0 ? nthreads : 1;
#pragma omp parallel num_threads(nt)
    {
        uint32_t *acc = (uint32_t *)calloc(blen, 4);
        uint32_t *loc = (uint32_t *)malloc(blen * 4);
        uint32_t sx[64];
        uint32_t lsum = 0;
#pragma omp for schedule(dynamic, 1)
        for (long long i = 0; i < (long long)nrows; ++i) {
            const uint32_t *row = rows + (size_t)i * row_len;
            uint32_t dot = 0;
            for (size_t j = 0; j < glen; ++j) dot ^= gmul(32, row[j], gr[j]);
            lsum ^= gmul(32, dot, apow[i]);
            scaled_basis(32, sx, loc, blen, sks_vks, (uint32_t)queries[i], apow[i]);
            for (size_t j = 0; j < blen; ++j) acc[j] ^= loc[j];
        }
#pragma omp critical
        {
            for (size_t j = 0; j < blen; ++j) basis_out[j] ^= acc[j];
            total ^= lsum;
        }
        free(acc);
        free(loc);
    }
    *enforced_sum = total;
    free(gr);
    free(apow);
    return LGREF_OK;
}

/* quadratic_from_evals, src/sumcheck.rs:67-81 (x = 3) */
void lgref_quadratic_from_evals(uint32_t at0, uint32_t at1, uint32_t atx, uint32_t abc[3]) {
    const uint32_t x = 3;
    uint32_t num = atx ^ at0 ^ gmul(32, x, at1 ^ at0);
    uint32_t den = gmul(32, x, x) ^ x, inv = 0;
    lgref_gf_inv(32, den, &inv);
    uint32_t a = gmul(32, num, inv);
    abc[0] = a;
    abc[1] = at1 ^ at0 ^ a;
    abc[2] = at0;
}
static uint32_t eval_quadratic(const uint32_t abc[3], uint32_t r) { /* :62-64 */
    return gmul(32, gmul(32, abc[0], r), r) ^ gmul(32, abc[1], r) ^ abc[2];
}

/* ======================================================================
 * Fiat-Shamir.  src/emulated_fs.rs:6-76.
 * ==================================================================== */
struct lgref_fs { sha256_st h; uint32_t counter; };

static void fs_init(struct lgref_fs *fs, uint32_t seed) { /* :12-16 */
    uint8_t b[4] = {(uint8_t)seed, (uint8_t)(seed >> 8), (uint8_t)(seed >> 16), (uint8_t)(seed >> 24)};
    sha_init(&fs->h);
    sha_update(&fs->h, b, 4);
    fs->counter = 0;
}
lgref_fs *lgref_fs_new(uint32_t seed) {
    lgref_fs *fs = (lgref_fs *)malloc(sizeof(lgref_fs));
    fs_init(fs, seed);
    return fs;
}
void lgref_fs_free(lgref_fs *fs) { free(fs); }
void lgref_fs_absorb(lgref_fs *fs, const uint8_t *b, size_t len) { sha_update(&fs->h, b, len); }

/* squeeze, :22-32: absorb the counter, then finalize a clone */
void lgref_fs_squeeze(lgref_fs *fs, uint64_t out[2]) {
    uint32_t c = fs->counter;
    uint8_t b[4] = {(uint8_t)c, (uint8_t)(c >> 8), (uint8_t)(c >> 16), (uint8_t)(c >> 24)};
    sha_update(&fs->h, b, 4);
    fs->counter += 1;
    uint8_t d[32];
    sha_final(&fs->h, d);
    uint64_t lo = 0, hi = 0;
    for (int i = 0; i < 8; ++i) lo |= (uint64_t)d[i] << (8 * i);
    for (int i = 0; i < 8; ++i) hi |= (uint64_t)d[8 + i] << (8 * i);
    out[0] = lo;
    out[1] = hi;
}
/* get_field::<BinaryElem32>, :34-54: low 32 bits of the squeeze */
uint32_t lgref_fs_get_field32(lgref_fs *fs) {
    uint64_t v[2];
    lgref_fs_squeeze(fs, v);
    return (uint32_t)v[0];
}
/* get_query, :56-59: (squeeze as usize) % n, usize = 64 bits */
uint64_t lgref_fs_get_query(lgref_fs *fs, uint64_t n) {
    uint64_t v[2];
    lgref_fs_squeeze(fs, v);
    return v[0] % n;
}
static int cmp_size(const void *a, const void *b) {
    size_t x = *(const size_t *)a, y = *(const size_t *)b;
    return x < y ? -1 : x > y;
}
/* get_distinct_queries, :61-76: rejection of repeats, then sort.  The
   reference loops forever when n < s; that is reported as PANIC here. */
int lgref_fs_get_distinct_queries(lgref_fs *fs, uint64_t n, size_t s, size_t *out) {
    if (n < s || n == 0) return LGREF_PANIC;
    size_t got = 0;
    size_t cap = 1;
    while (cap < 4 * s + 16) cap <<= 1;
    uint64_t *seen = (uint64_t *)malloc(cap * sizeof(uint64_t));
    unsigned char *used = (unsigned char *)calloc(cap, 1);
    while (got < s) {
        uint64_t q = lgref_fs_get_query(fs, n);
        size_t h = (size_t)((q * 0x9E3779B97F4A7C15ull) >> 40) & (cap - 1);
        int dup = 0;
        while (used[h]) {
            if (seen[h] == q) { dup = 1; break; }
            h = (h + 1) & (cap - 1);
        }
        if (!dup) {
            used[h] = 1;
            seen[h] = q;
            out[got++] = (size_t)q;
        }
    }
    free(seen);
    free(used);
    qsort(out, s, sizeof(size_t), cmp_size);
    return LGREF_OK;
}

/* ======================================================================
 * Configs.  src/config.rs:6-134, plus the size generator for the sizes the
 * reference has no function for: initial (2^(L-6), 2^6), k = 6, then
 * (2^(d-4), 2^4) steps while d-4 >= 10; L = 16..19 get one step
 * (2^(L-10), 2^4).  It reproduces config 20 and 24 exactly.
 * ==================================================================== */
int lgref_config_make(uint32_t L, lgref_config *c) {
    if (L < 16 || L > 30) return LGREF_BAD_ARG;
    memset(c, 0, sizeof *c);
    c->initial_log_m = L - 6;
    c->initial_log_n = 6;
    c->initial_k = 6;
    uint32_t d = L - 6, s = 0;
    while (d >= 14 && s < LGREF_MAX_STEPS) {
        c->log_m[s] = d - 4;
        c->log_n[s] = 4;
        c->ks[s] = 4;
        ++s;
        d -= 4;
    }
    if (s == 0) {
        c->log_m[0] = L - 10;
        c->log_n[0] = 4;
        c->ks[0] = 4;
        s = 1;
    }
    c->recursive_steps = s;
    return LGREF_OK;
}

/* Structural checks the reference's asserts would hit while proving. */
static int config_ok(const lgref_config *c, size_t len) {
    if (c->recursive_steps < 1 || c->recursive_steps > LGREF_MAX_STEPS) return 0;
    if (c->initial_log_m + c->initial_log_n >= 62) return 0;
    if (len != ((size_t)1 << (c->initial_log_m + c->initial_log_n))) return 0;
    if (c->initial_k != c->initial_log_n || c->initial_k == 0 || c->initial_k > 32) return 0;
    uint32_t nch = c->initial_k + 1, ntr = 1;
    for (uint32_t i = 0; i < c->recursive_steps; ++i) { nch += c->ks[i] + 2; ntr += c->ks[i] + 1; }
    if (nch > 200 || ntr > 120) return 0;
    if (c->initial_log_m + 2 < 8) return 0; /* >= 148 rows for the queries */
    uint32_t fvars = c->initial_log_m;
    for (uint32_t i = 0; i < c->recursive_steps; ++i) {
        if (c->log_m[i] + c->log_n[i] != fvars) return 0;
        if (c->ks[i] != c->log_n[i] || c->ks[i] == 0 || c->ks[i] > 32) return 0;
        if (c->log_m[i] + 2 < 8) return 0;
        fvars -= c->ks[i];
    }
    return 1;
}

/* ======================================================================
 * Canonical proof encoding (little-endian), in the field order of
 * FinalizedLigeritoProof (src/data_structures.rs:91-103):
 *   "LGRP" u32 version=1 u32 field_bytes=4
 *   bytes  initial_ligero_cm.root
 *   u32 n; n x bytes                      recursive_commitments
 *   opening initial_ligero_proof
 *   u32 n; n x opening                    recursive_proofs
 *   u32 n; n x u32 yr; opening            final_ligero_proof
 *   u32 n; n x (u32,u32,u32)              sumcheck_transcript
 * bytes   = u32 len, len bytes
 * opening = u32 rows; rows x (u32 len, len x u32);  u32 sibs; sibs x bytes
 * ==================================================================== */
typedef struct { uint8_t *p; size_t n, cap; int oom; } wbuf;
static void wb_put(wbuf *w, const void *src, size_t len) {
    if (w->oom) return;
    if (w->n + len > w->cap) {
        size_t nc = w->cap ? w->cap : 4096;
        while (nc < w->n + len) nc *= 2;
        uint8_t *np = (uint8_t *)realloc(w->p, nc);
        if (!np) { w->oom = 1; return; }
        w->p = np;
        w->cap = nc;
    }
    memcpy(w->p + w->n, src, len);
    w->n += len;
}
static void wb_u32(wbuf *w, uint32_t v) {
    uint8_t b[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
    wb_put(w, b, 4);
}
static void wb_bytes(wbuf *w, const uint8_t *p, uint32_t len) { wb_u32(w, len); wb_put(w, p, len); }
static void wb_opening(wbuf *w, const uint32_t *rows, uint32_t nrows, uint32_t rlen,
                       const uint8_t *sibs, uint32_t nsib) {
    wb_u32(w, nrows);
    for (uint32_t i = 0; i < nrows; ++i) {
        wb_u32(w, rlen);
        for (uint32_t j = 0; j < rlen; ++j) wb_u32(w, rows[(size_t)i * rlen + j]);
    }
    wb_u32(w, nsib);
    for (uint32_t i = 0; i < nsib; ++i) wb_bytes(w, sibs + 32 * (size_t)i, 32);
}

typedef struct { const uint8_t *p; size_t n, at; int bad; } rbuf;
static uint32_t rb_u32(rbuf *r) {
    if (r->bad || r->at + 4 > r->n) { r->bad = 1; return 0; }
    const uint8_t *b = r->p + r->at;
    r->at += 4;
    return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
}
static const uint8_t *rb_take(rbuf *r, size_t len) {
    if (r->bad || r->at + len > r->n) { r->bad = 1; return NULL; }
    const uint8_t *p = r->p + r->at;
    r->at += len;
    return p;
}

/* Parsed opening: rows may be ragged in the encoding; kept as given. */
typedef struct {
    uint32_t nrows;
    uint32_t *rlen;
    uint32_t **rows;
    uint32_t nsib;
    uint32_t *siblen;
    const uint8_t **sibs;
} opening_t;

static int rb_opening(rbuf *r, arena *a, opening_t *o) {
    o->nrows = rb_u32(r);
    if (r->bad || o->nrows > r->n) return 0;
    o->rlen = (uint32_t *)ar_alloc(a, (o->nrows + 1) * 4);
    o->rows = (uint32_t **)ar_alloc(a, (o->nrows + 1) * sizeof(uint32_t *));
    for (uint32_t i = 0; i < o->nrows && !r->bad; ++i) {
        o->rlen[i] = rb_u32(r);
        if (r->bad || (size_t)o->rlen[i] * 4 > r->n) return 0;
        o->rows[i] = (uint32_t *)ar_alloc(a, (size_t)o->rlen[i] * 4 + 4);
        for (uint32_t j = 0; j < o->rlen[i]; ++j) o->rows[i][j] = rb_u32(r);
    }
    o->nsib = rb_u32(r);
    if (r->bad || o->nsib > r->n) return 0;
    o->siblen = (uint32_t *)ar_alloc(a, (o->nsib + 1) * 4);
    o->sibs = (const uint8_t **)ar_alloc(a, (o->nsib + 1) * sizeof(uint8_t *));
    for (uint32_t i = 0; i < o->nsib && !r->bad; ++i) {
        o->siblen[i] = rb_u32(r);
        o->sibs[i] = rb_take(r, o->siblen[i]);
    }
    return !r->bad;
}

/* ======================================================================
 * Prover.  src/prover.rs:15-199.
 * ==================================================================== */
static __thread lgref_trace g_trace;
void lgref_last_trace(lgref_trace *out) { *out = g_trace; }

/* Test hook: a dishonest prover for negative tests.  Bit 0 flips s2 of the
   final sumcheck round before it is recorded and absorbed, so the proof is
   transcript-consistent and only the verifier's last check fails. */
static __thread int g_tamper;
void lgref_set_tamper(int flags) { g_tamper = flags; }

typedef struct {
    uint32_t *flat; /* column-major, n columns x rows */
    uint8_t *tree;
    size_t rows, cols;
} witness;

static int commit(const uint32_t *poly, size_t m, size_t n, witness *w, int nthreads, arena *a) {
    w->rows = 4 * m;
    w->cols = n;
    w->flat = (uint32_t *)ar_alloc(a, w->rows * n * 4);
    w->tree = (uint8_t *)ar_alloc(a, 32 * (2 * w->rows - 1));
    if (!w->flat || !w->tree) return LGREF_OOM;
    return lgref_ligero_commit(poly, m, n, w->flat, w->tree, nthreads);
}
static const uint8_t *root_of(const witness *w) { return w->tree + 32 * (2 * w->rows - 2); }

/* extract_row (src/ligero.rs:40-51) for each query + merkle prove */
static int open_rows(const witness *w, const size_t *q, size_t s, wbuf *out) {
    uint32_t *rows = (uint32_t *)malloc(s * w->cols * 4);
    size_t cap = s * 64 + 64, nsib = 0;
    uint8_t *sib = (uint8_t *)malloc(32 * cap);
    for (size_t i = 0; i < s; ++i)
        for (size_t j = 0; j < w->cols; ++j) rows[i * w->cols + j] = w->flat[j * w->rows + q[i]];
    int st = lgref_merkle_prove(w->tree, w->rows, q, s, sib, cap, &nsib);
    if (st == LGREF_OK) wb_opening(out, rows, (uint32_t)s, (uint32_t)w->cols, sib, (uint32_t)nsib);
    free(rows);
    free(sib);
    return st;
}

static void put_le32(uint8_t *p, uint32_t v) {
    p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

/* The prover's sumcheck state.  SumcheckProverInstance (src/ligerito.rs:7-141)
   keeps f and a list of basis polynomials that are only ever folded together
   and summed inside eval_01x_product; the list is kept as in the reference. */
typedef struct {
    uint32_t *f;
    size_t flen;
    uint32_t **basis;
    size_t nb, cap_b;
    uint32_t *glue_pending;
    uint32_t *tr;
    size_t ntr;
} sc_prover;

static void sc_push_tr(sc_prover *sc, const uint32_t s[3]) {
    sc->tr[3 * sc->ntr] = s[0];
    sc->tr[3 * sc->ntr + 1] = s[1];
    sc->tr[3 * sc->ntr + 2] = s[2];
    sc->ntr++;
}

/* eval_01x_product, src/ligerito.rs:69-117 (x = 3; evals_at_x :130-141) */
static void sc_eval_01x(const sc_prover *sc, uint32_t out[3]) {
    size_t h = sc->flen / 2;
    const uint32_t x = 3, xp1 = 1u ^ 3u;
    uint32_t s0 = 0, s1 = 0, s2 = 0;
    for (size_t i = 0; i < h; ++i) {
        uint32_t b0 = 0, b1 = 0, b2 = 0;
        for (size_t k = 0; k < sc->nb; ++k) {
            uint32_t lo = sc->basis[k][i], hi = sc->basis[k][h + i];
            b0 ^= lo;
            b1 ^= hi;
            b2 ^= gmul(32, x, hi) ^ gmul(32, xp1, lo);
        }
        uint32_t f0 = sc->f[i], f1 = sc->f[h + i];
        uint32_t f2 = gmul(32, x, f1) ^ gmul(32, xp1, f0);
        s0 ^= gmul(32, f0, b0);
        s1 ^= gmul(32, f1, b1);
        s2 ^= gmul(32, f2, b2);
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
}

/* fold, src/ligerito.rs:119-127 */
static void sc_fold(sc_prover *sc, uint32_t r, uint32_t out[3], int nthreads) {
    uint32_t *tmp = (uint32_t *)malloc((sc->flen / 2) * 4);
    partial_eval_core(sc->f, sc->flen, &r, 1, tmp, nthreads);
    memcpy(sc->f, tmp, (sc->flen / 2) * 4);
    for (size_t k = 0; k < sc->nb; ++k) {
        partial_eval_core(sc->basis[k], sc->flen, &r, 1, tmp, nthreads);
        memcpy(sc->basis[k], tmp, (sc->flen / 2) * 4);
    }
    free(tmp);
    sc->flen /= 2;
    sc_eval_01x(sc, out);
    sc_push_tr(sc, out);
}

int lgref_prove(const lgref_config *cfg, const uint32_t *poly, size_t len, int nthreads,
                uint8_t **proof_out, size_t *proof_len) {
    if (!config_ok(cfg, len)) return LGREF_PANIC;
    arena a = {0};
    int st = LGREF_OK;
    const size_t s = 148; /* :30 */
    memset(&g_trace, 0, sizeof g_trace);
    wbuf rec_roots = {0}, rec_proofs = {0}, init_open = {0}, fin = {0};
    uint32_t n_rec_proofs = 0;
    struct lgref_fs fs;
    fs_init(&fs, 1234); /* :29 */

    size_t m0 = (size_t)1 << cfg->initial_log_m, n0 = (size_t)1 << cfg->initial_log_n;
    witness w0, wprev;
    st = commit(poly, m0, n0, &w0, nthreads, &a); /* :32-37 */
    if (st) goto done;
    uint8_t root0[32];
    memcpy(root0, root_of(&w0), 32);
    memcpy(g_trace.roots[g_trace.n_roots++], root0, 32);
    lgref_fs_absorb(&fs, root0, 32); /* :48 */

    uint32_t pe0[64];
    for (uint32_t i = 0; i < cfg->initial_k; ++i) { /* :50 */
        pe0[i] = lgref_fs_get_field32(&fs);
        g_trace.challenges[g_trace.n_challenges++] = pe0[i];
    }
    size_t flen = len >> cfg->initial_k;
    sc_prover sc = {0};
    sc.f = (uint32_t *)ar_alloc(&a, flen * 4);
    sc.tr = (uint32_t *)ar_alloc(&a, 3 * 4 * (64 + 8 * LGREF_MAX_STEPS));
    sc.cap_b = LGREF_MAX_STEPS + 2;
    sc.basis = (uint32_t **)ar_alloc(&a, sc.cap_b * sizeof(uint32_t *));
    if (!sc.f || !sc.tr || !sc.basis) { st = LGREF_OOM; goto done; }
    {
        uint32_t *tmp = (uint32_t *)malloc((len / 2) * 4);
        partial_eval_core(poly, len, pe0, cfg->initial_k, tmp, nthreads); /* :52-53 */
        memcpy(sc.f, tmp, flen * 4);
        free(tmp);
    }
    sc.flen = flen;

    witness w1;
    st = commit(sc.f, (size_t)1 << cfg->log_m[0], (size_t)1 << cfg->log_n[0], &w1, nthreads, &a);
    if (st) goto done; /* :55-60 */
    memcpy(g_trace.roots[g_trace.n_roots++], root_of(&w1), 32);
    lgref_fs_absorb(&fs, root_of(&w1), 32); /* :64 */
    wb_bytes(&rec_roots, root_of(&w1), 32);

    size_t q[148];
    st = lgref_fs_get_distinct_queries(&fs, w0.rows, s, q); /* :67 */
    if (st) goto done;
    uint32_t alpha = lgref_fs_get_field32(&fs); /* :68 */
    g_trace.challenges[g_trace.n_challenges++] = alpha;

    int nv = log2_sz(sc.flen);
    uint32_t *sk = (uint32_t *)ar_alloc(&a, (nv + 1) * 4);
    lgref_eval_sk_at_vks(32, sc.flen, sk); /* :70 */
    uint32_t *rows = (uint32_t *)ar_alloc(&a, s * w0.cols * 4);
    for (size_t i = 0; i < s; ++i)
        for (size_t j = 0; j < w0.cols; ++j) rows[i * w0.cols + j] = w0.flat[j * w0.rows + q[i]];
    st = open_rows(&w0, q, s, &init_open); /* :72-76 */
    if (st) goto done;
    uint32_t *b1 = (uint32_t *)ar_alloc(&a, sc.flen * 4);
    uint32_t h1;
    st = lgref_induce_sumcheck_poly((size_t)nv, sk, rows, s, w0.cols, pe0, cfg->initial_k, q, alpha,
                                    b1, &h1, nthreads); /* :78-85 */
    if (st) goto done;
    g_trace.enforced_sums[g_trace.n_sums++] = h1;

    /* SumcheckProverInstance::new, src/ligerito.rs:32-48 */
    sc.basis[sc.nb++] = b1;
    uint32_t s3[3];
    lgref_eval_013_product(sc.f, b1, sc.flen, s3);
    if ((s3[0] ^ s3[1]) != h1) { st = LGREF_PANIC; goto done; }
    sc_push_tr(&sc, s3);
    uint8_t qb[12];
    put_le32(qb, s3[0]); put_le32(qb + 4, s3[1]); put_le32(qb + 8, s3[2]);
    lgref_fs_absorb(&fs, qb, 12); /* :93 */

    wprev = w1;
    for (uint32_t i = 0; i < cfg->recursive_steps; ++i) { /* :96 */
        uint32_t rsv[64];
        for (uint32_t t = 0; t < cfg->ks[i]; ++t) { /* :97-102 */
            uint32_t ri = lgref_fs_get_field32(&fs);
            g_trace.challenges[g_trace.n_challenges++] = ri;
            sc_fold(&sc, ri, s3, nthreads);
            if ((g_tamper & 1) && i == cfg->recursive_steps - 1 && t == cfg->ks[i] - 1) {
                s3[2] ^= 1u;
                sc.tr[3 * (sc.ntr - 1) + 2] ^= 1u;
            }
            put_le32(qb, s3[0]); put_le32(qb + 4, s3[1]); put_le32(qb + 8, s3[2]);
            lgref_fs_absorb(&fs, qb, 12);
            rsv[t] = ri;
        }
        if (i == cfg->recursive_steps - 1) { /* :104-143 */
            uint8_t *yb = (uint8_t *)malloc(sc.flen * 4);
            for (size_t j = 0; j < sc.flen; ++j) put_le32(yb + 4 * j, sc.f[j]);
            lgref_fs_absorb(&fs, yb, sc.flen * 4);
            free(yb);
            st = lgref_fs_get_distinct_queries(&fs, wprev.rows, s, q);
            if (st) goto done;
            wb_u32(&fin, (uint32_t)sc.flen);
            for (size_t j = 0; j < sc.flen; ++j) wb_u32(&fin, sc.f[j]);
            st = open_rows(&wprev, q, s, &fin);
            if (st) goto done;
            break;
        }
        witness wn; /* :145-155 */
        st = commit(sc.f, (size_t)1 << cfg->log_m[i + 1], (size_t)1 << cfg->log_n[i + 1], &wn,
                    nthreads, &a);
        if (st) goto done;
        memcpy(g_trace.roots[g_trace.n_roots++], root_of(&wn), 32);
        lgref_fs_absorb(&fs, root_of(&wn), 32);
        wb_bytes(&rec_roots, root_of(&wn), 32);

        st = lgref_fs_get_distinct_queries(&fs, wprev.rows, s, q); /* :157 */
        if (st) goto done;
        uint32_t al = lgref_fs_get_field32(&fs); /* :158 */
        g_trace.challenges[g_trace.n_challenges++] = al;
        nv = log2_sz(sc.flen);
        sk = (uint32_t *)ar_alloc(&a, (nv + 1) * 4);
        lgref_eval_sk_at_vks(32, sc.flen, sk); /* :160 */
        rows = (uint32_t *)ar_alloc(&a, s * wprev.cols * 4);
        for (size_t r = 0; r < s; ++r)
            for (size_t j = 0; j < wprev.cols; ++j) rows[r * wprev.cols + j] = wprev.flat[j * wprev.rows + q[r]];
        st = open_rows(&wprev, q, s, &rec_proofs); /* :161-172 */
        if (st) goto done;
        n_rec_proofs++;
        uint32_t *bi = (uint32_t *)ar_alloc(&a, sc.flen * 4);
        uint32_t hi;
        st = lgref_induce_sumcheck_poly((size_t)nv, sk, rows, s, wprev.cols, rsv, cfg->ks[i], q, al, bi,
                                        &hi, nthreads); /* :174-181 */
        if (st) goto done;
        g_trace.enforced_sums[g_trace.n_sums++] = hi;
        /* introduce_new, src/ligerito.rs:50-57 */
        lgref_eval_013_product(sc.f, bi, sc.flen, s3);
        if ((s3[0] ^ s3[1]) != hi) { st = LGREF_PANIC; goto done; }
        sc_push_tr(&sc, s3);
        put_le32(qb, s3[0]); put_le32(qb + 4, s3[1]); put_le32(qb + 8, s3[2]);
        lgref_fs_absorb(&fs, qb, 12); /* :187-191 */
        /* glue, src/ligerito.rs:59-67 */
        uint32_t beta = lgref_fs_get_field32(&fs); /* :193 */
        g_trace.challenges[g_trace.n_challenges++] = beta;
        for (size_t j = 0; j < sc.flen; ++j) bi[j] = gmul(32, bi[j], beta);
        sc.basis[sc.nb++] = bi;
        wprev = wn;
    }

    {
        wbuf out = {0};
        wb_put(&out, "LGRP", 4);
        wb_u32(&out, 1);
        wb_u32(&out, 4);
        wb_bytes(&out, root0, 32);
        wb_u32(&out, cfg->recursive_steps);
        wb_put(&out, rec_roots.p, rec_roots.n);
        wb_put(&out, init_open.p, init_open.n);
        wb_u32(&out, n_rec_proofs);
        wb_put(&out, rec_proofs.p, rec_proofs.n);
        wb_put(&out, fin.p, fin.n);
        wb_u32(&out, (uint32_t)sc.ntr);
        for (size_t t = 0; t < 3 * sc.ntr; ++t) wb_u32(&out, sc.tr[t]);
        if (out.oom || rec_roots.oom || init_open.oom || rec_proofs.oom || fin.oom) {
            free(out.p);
            st = LGREF_OOM;
        } else {
            *proof_out = out.p;
            *proof_len = out.n;
        }
    }
done:
    free(rec_roots.p);
    free(rec_proofs.p);
    free(init_open.p);
    free(fin.p);
    if (a.oom && st == LGREF_OK) st = LGREF_OOM;
    ar_free(&a);
    return st;
}

void lgref_free(void *p) { free(p); }

/* ======================================================================
 * Verifier.  src/verifier.rs:10-164 with SumcheckVerifierInstance
 * (src/ligerito.rs:143-296).  Returns PANIC wherever the reference panics.
 * ==================================================================== */
typedef struct {
    uint32_t **basis; /* basis_polys */
    uint32_t *bvars;  /* num_vars of each */
    size_t nb;
    uint32_t sep[LGREF_MAX_STEPS + 2]; /* separation_challenges */
    uint32_t sum;
    const uint32_t *tr;
    size_t ntr, rd;
    uint32_t ris[256];
    size_t nris;
    uint32_t running[3];
    int has_running;
    uint32_t to_glue[3];
    int has_glue;
} sc_verifier;

static int scv_read(sc_verifier *v, uint32_t g[3]) { /* read_tr, :194-199 */
    if (v->rd >= v->ntr) return 0;
    g[0] = v->tr[3 * v->rd];
    g[1] = v->tr[3 * v->rd + 1];
    g[2] = v->tr[3 * v->rd + 2];
    v->rd++;
    return 1;
}

/* Opened-row byte strings for the Merkle leaves (src/verifier.rs:35-40) */
static void rows_as_leaves(const opening_t *o, arena *a, uint8_t **buf, size_t **off) {
    size_t tot = 0;
    for (uint32_t i = 0; i < o->nrows; ++i) tot += 4 * (size_t)o->rlen[i];
    *buf = (uint8_t *)ar_alloc(a, tot + 1);
    *off = (size_t *)ar_alloc(a, (o->nrows + 1) * sizeof(size_t));
    size_t at = 0;
    for (uint32_t i = 0; i < o->nrows; ++i) {
        (*off)[i] = at;
        for (uint32_t j = 0; j < o->rlen[i]; ++j) put_le32(*buf + at + 4 * j, o->rows[i][j]);
        at += 4 * (size_t)o->rlen[i];
    }
    (*off)[o->nrows] = at;
}

/* merkle_tree::verify against an opening (sibling byte strings must be 32) */
static int verify_opening(const uint8_t *root, uint32_t root_len, const opening_t *o, size_t depth,
                          const size_t *q, size_t nq, arena *a, int *ok) {
    uint8_t *buf;
    size_t *off;
    if (nq != o->nrows) { *ok = 0; return LGREF_PANIC; } /* zip would truncate; the layer
                                   count then disagrees with queries: index panic */
    rows_as_leaves(o, a, &buf, &off);
    uint8_t *sib = (uint8_t *)ar_alloc(a, 32 * (size_t)o->nsib + 1);
    for (uint32_t i = 0; i < o->nsib; ++i) {
        if (o->siblen[i] != 32) { *ok = 0; return LGREF_PANIC; }
        memcpy(sib + 32 * (size_t)i, o->sibs[i], 32);
    }
    uint8_t *layer = (uint8_t *)ar_alloc(a, 32 * (nq ? nq : 1));
    for (size_t i = 0; i < nq; ++i) lgref_blake3(buf + off[i], off[i + 1] - off[i], layer + 32 * i);
    int st = merkle_verify_hashed(LGREF_HASH_BLAKE3, root, sib, o->nsib, depth, layer, q, nq, ok);
    if (root_len != 32) *ok = 0;
    return st;
}

/* Flatten an opening to a dense rows array; PANIC if ragged or mismatched. */
static int dense_rows(const opening_t *o, size_t want_len, arena *a, uint32_t **out) {
    *out = (uint32_t *)ar_alloc(a, (size_t)o->nrows * want_len * 4 + 4);
    for (uint32_t i = 0; i < o->nrows; ++i) {
        if (o->rlen[i] != want_len) return LGREF_PANIC;
        memcpy(*out + (size_t)i * want_len, o->rows[i], want_len * 4);
    }
    return LGREF_OK;
}

int lgref_verify(const lgref_config *cfg, const uint8_t *proof, size_t len, int nthreads,
                 int *accepted) {
    *accepted = 0;
    arena a = {0};
    int st = LGREF_OK, ok = 0;
    const size_t s = 148;
    const uint32_t log_inv_rate = 2; /* :26 */
    rbuf r = {proof, len, 0, 0};
    const uint8_t *mg = rb_take(&r, 4);
    if (!mg || memcmp(mg, "LGRP", 4) != 0 || rb_u32(&r) != 1 || rb_u32(&r) != 4) return LGREF_BAD_ARG;
    /* parse */
    uint32_t root0_len = rb_u32(&r);
    const uint8_t *root0 = rb_take(&r, root0_len);
    uint32_t nrc = rb_u32(&r);
    if (r.bad || nrc > len) return LGREF_BAD_ARG;
    const uint8_t **rroots = (const uint8_t **)ar_alloc(&a, (nrc + 1) * sizeof(uint8_t *));
    uint32_t *rroot_len = (uint32_t *)ar_alloc(&a, (nrc + 1) * 4);
    for (uint32_t i = 0; i < nrc; ++i) { rroot_len[i] = rb_u32(&r); rroots[i] = rb_take(&r, rroot_len[i]); }
    opening_t init;
    if (!rb_opening(&r, &a, &init)) { ar_free(&a); return LGREF_BAD_ARG; }
    uint32_t nrp = rb_u32(&r);
    if (r.bad || nrp > len) { ar_free(&a); return LGREF_BAD_ARG; }
    opening_t *rp = (opening_t *)ar_alloc(&a, (nrp + 1) * sizeof(opening_t));
    for (uint32_t i = 0; i < nrp; ++i)
        if (!rb_opening(&r, &a, &rp[i])) { ar_free(&a); return LGREF_BAD_ARG; }
    uint32_t yr_len = rb_u32(&r);
    if (r.bad || (size_t)yr_len * 4 > len) { ar_free(&a); return LGREF_BAD_ARG; }
    uint32_t *yr = (uint32_t *)ar_alloc(&a, (size_t)yr_len * 4 + 4);
    for (uint32_t i = 0; i < yr_len; ++i) yr[i] = rb_u32(&r);
    opening_t fin;
    if (!rb_opening(&r, &a, &fin)) { ar_free(&a); return LGREF_BAD_ARG; }
    uint32_t ntr = rb_u32(&r);
    if (r.bad || (size_t)ntr * 12 > len) { ar_free(&a); return LGREF_BAD_ARG; }
    uint32_t *tr = (uint32_t *)ar_alloc(&a, (size_t)ntr * 12 + 4);
    for (uint32_t i = 0; i < 3 * ntr; ++i) tr[i] = rb_u32(&r);
    if (r.bad || r.at != len) { ar_free(&a); return LGREF_BAD_ARG; }

    /* VerifierConfig, src/config.rs:49-67,114-134 */
    const uint32_t initial_dim = cfg->initial_log_m;
    struct lgref_fs fs;
    fs_init(&fs, 1234); /* :24 */
    if (root0_len) lgref_fs_absorb(&fs, root0, root0_len); /* :27 */
    uint32_t pe0[64];
    if (cfg->initial_k > 64) { st = LGREF_PANIC; goto done; }
    for (uint32_t i = 0; i < cfg->initial_k; ++i) pe0[i] = lgref_fs_get_field32(&fs); /* :29 */
    if (nrc < 1) { st = LGREF_PANIC; goto done; }
    lgref_fs_absorb(&fs, rroots[0], rroot_len[0]); /* :30 */
    size_t depth = initial_dim + log_inv_rate; /* :32 */
    size_t q[148];
    st = lgref_fs_get_distinct_queries(&fs, (uint64_t)1 << depth, s, q); /* :33 */
    if (st) goto done;
    st = verify_opening(root0, root0_len, &init, depth, q, s, &a, &ok); /* :42-49 */
    if (st || !ok) { st = LGREF_PANIC; goto done; }

    uint32_t alpha = lgref_fs_get_field32(&fs); /* :51 */
    size_t blen = (size_t)1 << initial_dim;
    uint32_t *sk = (uint32_t *)ar_alloc(&a, (initial_dim + 1) * 4);
    lgref_eval_sk_at_vks(32, blen, sk); /* :52 */
    uint32_t *rows;
    size_t rl = (size_t)1 << cfg->initial_k;
    if (dense_rows(&init, rl, &a, &rows) != LGREF_OK) { st = LGREF_PANIC; goto done; }
    uint32_t *b1 = (uint32_t *)ar_alloc(&a, blen * 4);
    uint32_t h1;
    st = lgref_induce_sumcheck_poly(initial_dim, sk, rows, init.nrows, rl, pe0, cfg->initial_k, q, alpha,
                                    b1, &h1, nthreads); /* :53-60 */
    if (st) goto done;

    sc_verifier v;
    memset(&v, 0, sizeof v);
    v.basis = (uint32_t **)ar_alloc(&a, (LGREF_MAX_STEPS + 2) * sizeof(uint32_t *));
    v.bvars = (uint32_t *)ar_alloc(&a, (LGREF_MAX_STEPS + 2) * 4);
    v.basis[0] = b1;
    v.bvars[0] = initial_dim;
    v.nb = 1;
    v.sep[0] = 1;
    v.sum = h1;
    v.tr = tr;
    v.ntr = ntr;
    uint32_t g[3];
    /* SumcheckVerifierInstance::new, src/ligerito.rs:172-192 */
    if (!scv_read(&v, g) || (g[0] ^ g[1]) != v.sum) { st = LGREF_PANIC; goto done; }
    lgref_quadratic_from_evals(g[0], g[1], g[2], v.running);
    v.has_running = 1;
    uint8_t qb[12];
    put_le32(qb, g[0]); put_le32(qb + 4, g[1]); put_le32(qb + 8, g[2]);
    lgref_fs_absorb(&fs, qb, 12); /* :67 */

    for (uint32_t i = 0; i < cfg->recursive_steps; ++i) { /* :69 */
        uint32_t rsv[64];
        if (cfg->ks[i] > 64) { st = LGREF_PANIC; goto done; }
        for (uint32_t t = 0; t < cfg->ks[i]; ++t) { /* :70-76 */
            uint32_t ri = lgref_fs_get_field32(&fs);
            /* SumcheckVerifierInstance::fold, src/ligerito.rs:201-210 */
            if (v.nris >= 255) { st = LGREF_PANIC; goto done; }
            v.ris[v.nris++] = ri;
            v.sum = eval_quadratic(v.running, ri);
            if (!scv_read(&v, g) || (g[0] ^ g[1]) != v.sum) { st = LGREF_PANIC; goto done; }
            lgref_quadratic_from_evals(g[0], g[1], g[2], v.running);
            put_le32(qb, g[0]); put_le32(qb + 4, g[1]); put_le32(qb + 8, g[2]);
            lgref_fs_absorb(&fs, qb, 12);
            rsv[t] = ri;
        }
        if (i >= nrc) { st = LGREF_PANIC; goto done; }
        const uint8_t *root = rroots[i];
        uint32_t root_len = rroot_len[i];
        if (i == cfg->recursive_steps - 1) { /* :78-120 */
            uint8_t *yb = (uint8_t *)ar_alloc(&a, (size_t)yr_len * 4 + 1);
            for (uint32_t j = 0; j < yr_len; ++j) put_le32(yb + 4 * j, yr[j]);
            lgref_fs_absorb(&fs, yb, (size_t)yr_len * 4);
            depth = cfg->log_m[i] + log_inv_rate;
            st = lgref_fs_get_distinct_queries(&fs, (uint64_t)1 << depth, s, q);
            if (st) goto done;
            st = verify_opening(root, root_len, &fin, depth, q, s, &a, &ok); /* :96-106 */
            if (st || !ok) { st = LGREF_PANIC; goto done; }
            /* ligero_verify, :107-112; rows zip against gr of length 2^k */
            st = ligero_verify_core(q, fin.nrows, (const uint32_t *const *)fin.rows, fin.rlen, yr,
                                    yr_len, rsv, cfg->ks[i]);
            if (st) goto done;
            uint32_t final_r = lgref_fs_get_field32(&fs); /* :114 */
            if (yr_len < 2 || !is_pow2(yr_len)) { st = LGREF_PANIC; goto done; }
            uint32_t *fev = (uint32_t *)ar_alloc(&a, (yr_len / 2) * 4);
            partial_eval_core(yr, yr_len, &final_r, 1, fev, 1); /* :115-117 */
            size_t fl = yr_len / 2;
            /* verify_partial, src/ligerito.rs:282-295 */
            uint32_t k = (uint32_t)log2_sz(fl);
            uint32_t sum = eval_quadratic(v.running, final_r);
            v.ris[v.nris++] = final_r;
            /* evaluate_basis_polys_partially, :257-280 */
            uint32_t *acc = NULL;
            for (size_t bi = 0; bi < v.nb; ++bi) {
                uint32_t nvars = v.bvars[bi];
                const uint32_t *pts;
                size_t npts;
                if (bi == 0) { pts = v.ris; npts = v.nris; }
                else {
                    if (nvars < k || nvars - k > v.nris) { st = LGREF_PANIC; goto done; }
                    npts = nvars - k;
                    pts = v.ris + (v.nris - npts);
                }
                if (npts == 0 || npts > nvars) { st = LGREF_PANIC; goto done; }
                size_t outl = (size_t)1 << (nvars - npts);
                uint32_t *pe = (uint32_t *)ar_alloc(&a, outl * 4);
                st = lgref_partial_eval(v.basis[bi], (size_t)1 << nvars, pts, npts, pe, nthreads);
                if (st) goto done;
                if (bi == 0) { acc = pe; if (outl != fl) { st = LGREF_PANIC; goto done; } }
                else {
                    if (outl != fl) { st = LGREF_PANIC; goto done; }
                    for (size_t j = 0; j < fl; ++j) acc[j] ^= gmul(32, v.sep[bi], pe[j]);
                }
            }
            uint32_t dot = 0;
            for (size_t j = 0; j < fl; ++j) dot ^= gmul(32, fev[j], acc[j]);
            *accepted = (dot == sum);
            goto done;
        }
        if (i + 1 >= nrc || i >= nrp) { st = LGREF_PANIC; goto done; }
        lgref_fs_absorb(&fs, rroots[i + 1], rroot_len[i + 1]); /* :122 */
        depth = cfg->log_m[i] + log_inv_rate;
        st = lgref_fs_get_distinct_queries(&fs, (uint64_t)1 << depth, s, q); /* :126 */
        if (st) goto done;
        st = verify_opening(root, root_len, &rp[i], depth, q, s, &a, &ok); /* :334-343 */
        if (st || !ok) { st = LGREF_PANIC; goto done; }
        uint32_t al = lgref_fs_get_field32(&fs); /* :145 */
        size_t bl = (size_t)1 << cfg->log_m[i];
        uint32_t *ski = (uint32_t *)ar_alloc(&a, (cfg->log_m[i] + 1) * 4);
        lgref_eval_sk_at_vks(32, bl, ski);
        uint32_t *rrows;
        size_t rrl = (size_t)1 << cfg->ks[i];
        if (dense_rows(&rp[i], rrl, &a, &rrows) != LGREF_OK) { st = LGREF_PANIC; goto done; }
        uint32_t *bnew = (uint32_t *)ar_alloc(&a, bl * 4);
        uint32_t hn;
        st = lgref_induce_sumcheck_poly(cfg->log_m[i], ski, rrows, rp[i].nrows, rrl, rsv, cfg->ks[i], q, al,
                                        bnew, &hn, nthreads);
        if (st) goto done;
        /* introduce_new, src/ligerito.rs:212-220 */
        if (!scv_read(&v, g) || (g[0] ^ g[1]) != hn) { st = LGREF_PANIC; goto done; }
        v.basis[v.nb] = bnew;
        v.bvars[v.nb] = cfg->log_m[i];
        v.nb++;
        lgref_quadratic_from_evals(g[0], g[1], g[2], v.to_glue);
        v.has_glue = 1;
        put_le32(qb, g[0]); put_le32(qb + 4, g[1]); put_le32(qb + 8, g[2]);
        lgref_fs_absorb(&fs, qb, 12); /* :356 */
        uint32_t beta = lgref_fs_get_field32(&fs); /* :358 */
        /* glue, src/ligerito.rs:222-232 */
        v.sep[v.nb - 1] = beta;
        for (int t = 0; t < 3; ++t) v.running[t] ^= gmul(32, beta, v.to_glue[t]);
        v.has_glue = 0;
    }
    st = LGREF_PANIC; /* :362 */
done:
    if (a.oom && st == LGREF_OK) st = LGREF_OOM;
    ar_free(&a);
    if (st != LGREF_OK) *accepted = 0;
    return st;
}

/* ======================================================================
 * Seeded input generator (ours): SplitMix64, coefficient i = low 32 bits
 * of the i-th output.
 * ==================================================================== */
void lgref_splitmix_coeffs(uint64_t seed, uint32_t *out, size_t n) {
    uint64_t x = seed;
    for (size_t i = 0; i < n; ++i) {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        out[i] = (uint32_t)(z ^ (z >> 31));
    }
}
