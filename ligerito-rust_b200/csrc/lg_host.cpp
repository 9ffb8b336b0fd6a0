// Host-side pieces of liblgpu (see lg_host.h).
#include "lg_host.h"

#include <algorithm>
#include <cstring>
#include <unordered_set>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace lg {

// ===================================================================== GF
static inline uint32_t reduce64(uint64_t c) {
    // fold bits 32..62 with x^32 = x^15+x^9+x^7+x^4+x^3+1, twice
    uint32_t hi = (uint32_t)(c >> 32), lo = (uint32_t)c;
    uint32_t lo2 = hi ^ (hi << 3) ^ (hi << 4) ^ (hi << 7) ^ (hi << 9) ^ (hi << 15);
    uint32_t ov = (hi >> 29) ^ (hi >> 28) ^ (hi >> 25) ^ (hi >> 23) ^ (hi >> 17);
    uint32_t lo3 = ov ^ (ov << 3) ^ (ov << 4) ^ (ov << 7) ^ (ov << 9) ^ (ov << 15);
    return lo ^ lo2 ^ lo3;
}

static uint64_t clmul_portable(uint32_t a, uint32_t b) {
    // 4-bit windows of b over a precomputed 16-entry table of a's multiples
    uint64_t t[16];
    t[0] = 0;
    t[1] = a;
    for (int i = 2; i < 16; i += 2) {
        t[i] = t[i / 2] << 1;
        t[i + 1] = t[i] ^ a;
    }
    uint64_t r = 0;
    for (int s = 28; s >= 0; s -= 4) r = (r << 4) ^ t[(b >> s) & 15];
    return r;
}

#if defined(__x86_64__)
__attribute__((target("pclmul,sse4.1"))) static uint64_t clmul_hw(uint32_t a, uint32_t b) {
    __m128i x = _mm_cvtsi32_si128((int)a), y = _mm_cvtsi32_si128((int)b);
    return (uint64_t)_mm_cvtsi128_si64(_mm_clmulepi64_si128(x, y, 0));
}
static const bool g_has_pclmul = __builtin_cpu_supports("pclmul");
#endif

uint32_t gf_mul(uint32_t a, uint32_t b) {
#if defined(__x86_64__)
    if (g_has_pclmul) return reduce64(clmul_hw(a, b));
#endif
    return reduce64(clmul_portable(a, b));
}

uint32_t gf_pow(uint32_t a, uint64_t e) {
    uint32_t r = 1, base = a;
    while (e) {
        if (e & 1) r = gf_mul(r, base);
        base = gf_mul(base, base);
        e >>= 1;
    }
    return r;
}

uint32_t gf_inv(uint32_t a) { return gf_pow(a, 0xFFFFFFFEull); }  // a^(2^32-2)

// ================================================================= SHA-256
static const uint32_t K256[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static inline uint32_t rotr(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }

static void sha256_compress(uint32_t st[8], const uint8_t blk[64]) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
        w[i] = (uint32_t)blk[4 * i] << 24 | (uint32_t)blk[4 * i + 1] << 16 |
               (uint32_t)blk[4 * i + 2] << 8 | blk[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
        uint32_t a = w[i - 15], b = w[i - 2];
        w[i] = w[i - 16] + (rotr(a, 7) ^ rotr(a, 18) ^ (a >> 3)) + w[i - 7] +
               (rotr(b, 17) ^ rotr(b, 19) ^ (b >> 10));
    }
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
    for (int i = 0; i < 64; ++i) {
        uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + K256[i] + w[i];
        uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d; st[4] += e; st[5] += f; st[6] += g; st[7] += h;
}

#if defined(__x86_64__)
// The same compression with the x86 SHA extensions.  The state is kept as
// (A,B,E,F) / (C,D,G,H) halves as sha256rnds2 expects; each 4-round group
// adds the schedule words and round constants, and words 16..63 come from
// sha256msg1 / sha256msg2: W[t..t+3] = msg2(msg1(W[t-16..], W[t-12..]) +
// W[t-7..t-4], W[t-4..t-1]).
__attribute__((target("sha,sse4.1,ssse3"))) static void sha256_compress_ni(uint32_t st[8], const uint8_t blk[64]) {
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bULL, 0x0405060700010203ULL);
    __m128i dcba = _mm_loadu_si128(reinterpret_cast<const __m128i *>(st));
    __m128i hgfe = _mm_loadu_si128(reinterpret_cast<const __m128i *>(st + 4));
    __m128i cdab = _mm_shuffle_epi32(dcba, 0xB1);
    __m128i efgh = _mm_shuffle_epi32(hgfe, 0x1B);
    __m128i abef = _mm_alignr_epi8(cdab, efgh, 8);
    __m128i cdgh = _mm_blend_epi16(efgh, cdab, 0xF0);
    const __m128i abef0 = abef, cdgh0 = cdgh;
    __m128i m[4];
    for (int i = 0; i < 4; ++i)
        m[i] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i *>(blk + 16 * i)), bswap);
    for (int i = 0; i < 16; ++i) {
        __m128i w;
        if (i < 4) {
            w = m[i];
        } else {
            __m128i x = _mm_sha256msg1_epu32(m[i & 3], m[(i + 1) & 3]);
            x = _mm_add_epi32(x, _mm_alignr_epi8(m[(i + 3) & 3], m[(i + 2) & 3], 4));
            w = m[i & 3] = _mm_sha256msg2_epu32(x, m[(i + 3) & 3]);
        }
        __m128i k = _mm_add_epi32(w, _mm_loadu_si128(reinterpret_cast<const __m128i *>(K256 + 4 * i)));
        cdgh = _mm_sha256rnds2_epu32(cdgh, abef, k);
        abef = _mm_sha256rnds2_epu32(abef, cdgh, _mm_shuffle_epi32(k, 0x0E));
    }
    abef = _mm_add_epi32(abef, abef0);
    cdgh = _mm_add_epi32(cdgh, cdgh0);
    __m128i feba = _mm_shuffle_epi32(abef, 0x1B);
    __m128i dchg = _mm_shuffle_epi32(cdgh, 0xB1);
    _mm_storeu_si128(reinterpret_cast<__m128i *>(st), _mm_blend_epi16(feba, dchg, 0xF0));
    _mm_storeu_si128(reinterpret_cast<__m128i *>(st + 4), _mm_alignr_epi8(dchg, feba, 8));
}
static const bool g_has_shani = __builtin_cpu_supports("sha") && __builtin_cpu_supports("sse4.1");
#endif

static void sha256_block(uint32_t st[8], const uint8_t blk[64]) {
#if defined(__x86_64__)
    if (g_has_shani) { sha256_compress_ni(st, blk); return; }
#endif
    sha256_compress(st, blk);
}

Sha256::Sha256() {
    static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    std::memcpy(h, iv, sizeof iv);
}

void Sha256::update(const uint8_t *p, size_t len) {
    total += len;
    if (n) {
        size_t take = std::min(len, 64 - n);
        std::memcpy(buf + n, p, take);
        n += take; p += take; len -= take;
        if (n == 64) { sha256_block(h, buf); n = 0; }
    }
    while (len >= 64) { sha256_block(h, p); p += 64; len -= 64; }
    if (len) { std::memcpy(buf, p, len); n = len; }
}

void Sha256::finish(uint8_t out[32]) const {
    uint32_t st[8];
    std::memcpy(st, h, sizeof st);
    uint8_t tail[128] = {0};
    std::memcpy(tail, buf, n);
    tail[n] = 0x80;
    size_t tl = (n + 1 + 8 <= 64) ? 64 : 128;
    uint64_t bits = total * 8;
    for (int i = 0; i < 8; ++i) tail[tl - 1 - i] = (uint8_t)(bits >> (8 * i));
    sha256_block(st, tail);
    if (tl == 128) sha256_block(st, tail + 64);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(st[i] >> 24); out[4 * i + 1] = (uint8_t)(st[i] >> 16);
        out[4 * i + 2] = (uint8_t)(st[i] >> 8); out[4 * i + 3] = (uint8_t)st[i];
    }
}

// FS::new (src/emulated_fs.rs:12-16): absorb the seed's LE bytes
Transcript::Transcript(uint32_t seed) {
    uint8_t b[4] = {(uint8_t)seed, (uint8_t)(seed >> 8), (uint8_t)(seed >> 16), (uint8_t)(seed >> 24)};
    h.update(b, 4);
}
void Transcript::absorb(const void *p, size_t len) { h.update((const uint8_t *)p, len); }
void Transcript::absorb_u32s(const uint32_t *v, size_t n) {
    uint8_t tmp[256];
    size_t at = 0;
    for (size_t i = 0; i < n; ++i) {
        uint32_t x = v[i];
        tmp[at++] = (uint8_t)x; tmp[at++] = (uint8_t)(x >> 8);
        tmp[at++] = (uint8_t)(x >> 16); tmp[at++] = (uint8_t)(x >> 24);
        if (at == sizeof tmp) { h.update(tmp, at); at = 0; }
    }
    if (at) h.update(tmp, at);
}
// squeeze (src/emulated_fs.rs:22-32): absorb the counter, finalize a clone
std::array<uint64_t, 2> Transcript::squeeze() {
    uint8_t b[4] = {(uint8_t)counter, (uint8_t)(counter >> 8), (uint8_t)(counter >> 16),
                    (uint8_t)(counter >> 24)};
    h.update(b, 4);
    counter += 1;
    uint8_t d[32];
    h.finish(d);
    uint64_t lo = 0, hi = 0;
    for (int i = 7; i >= 0; --i) lo = (lo << 8) | d[i];
    for (int i = 15; i >= 8; --i) hi = (hi << 8) | d[i];
    return {lo, hi};
}
// The low 64 bits of squeeze(): the counter's 4 bytes join the pending
// bytes (a block is compressed when they fill one), then a copy of the
// state is finalised straight from the pending bytes; the result is the
// first 8 digest bytes read little-endian.
uint64_t Transcript::squeeze_lo() {
    const uint8_t c4[4] = {(uint8_t)counter, (uint8_t)(counter >> 8), (uint8_t)(counter >> 16),
                           (uint8_t)(counter >> 24)};
    counter += 1;
    h.update(c4, 4);
    uint32_t st[8];
    std::memcpy(st, h.h, sizeof st);
    alignas(16) uint8_t tail[128];
    const size_t n = h.n, tl = (n + 1 + 8 <= 64) ? 64 : 128;
    std::memcpy(tail, h.buf, n);
    tail[n] = 0x80;
    std::memset(tail + n + 1, 0, tl - 8 - (n + 1));
    const uint64_t bits = h.total * 8;
    for (int i = 0; i < 8; ++i) tail[tl - 1 - i] = (uint8_t)(bits >> (8 * i));
    sha256_block(st, tail);
    if (tl == 128) sha256_block(st, tail + 64);
    return (uint64_t)__builtin_bswap32(st[0]) | ((uint64_t)__builtin_bswap32(st[1]) << 32);
}

// get_distinct_queries (src/emulated_fs.rs:61-76)
bool Transcript::get_distinct_queries(uint64_t n, size_t s, std::vector<uint64_t> &out) {
    out.clear();
    if (n < s || n == 0) return false;
    // values seen so far: open addressing over at least 4s slots; ~0 marks
    // an empty slot and is never a query (queries are < n)
    size_t cap = 64;
    while (cap < 4 * s) cap <<= 1;
    std::vector<uint64_t> seen(cap, ~0ull);
    while (out.size() < s) {
        const uint64_t q = get_query(n);
        size_t h = (size_t)((q * 0x9E3779B97F4A7C15ull) >> 40) & (cap - 1);
        while (seen[h] != ~0ull && seen[h] != q) h = (h + 1) & (cap - 1);
        if (seen[h] == ~0ull) {
            seen[h] = q;
            out.push_back(q);
        }
    }
    std::sort(out.begin(), out.end());
    return true;
}

// ================================================================== BLAKE3
static const uint32_t B3IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
static const uint8_t B3P[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

static void b3_round_g(uint32_t *v, int a, int b, int c, int d, uint32_t x, uint32_t y) {
    v[a] += v[b] + x; v[d] = rotr(v[d] ^ v[a], 16);
    v[c] += v[d];     v[b] = rotr(v[b] ^ v[c], 12);
    v[a] += v[b] + y; v[d] = rotr(v[d] ^ v[a], 8);
    v[c] += v[d];     v[b] = rotr(v[b] ^ v[c], 7);
}

// compression; out = 16 words (first 8 = next chaining value)
static void b3_compress(const uint32_t cv[8], const uint32_t m_in[16], uint64_t ctr, uint32_t blen,
                        uint32_t flags, uint32_t out[16]) {
    uint32_t v[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      B3IV[0], B3IV[1], B3IV[2], B3IV[3], (uint32_t)ctr, (uint32_t)(ctr >> 32), blen, flags};
    uint32_t m[16];
    std::memcpy(m, m_in, 64);
    for (int r = 0; r < 7; ++r) {
        b3_round_g(v, 0, 4, 8, 12, m[0], m[1]);
        b3_round_g(v, 1, 5, 9, 13, m[2], m[3]);
        b3_round_g(v, 2, 6, 10, 14, m[4], m[5]);
        b3_round_g(v, 3, 7, 11, 15, m[6], m[7]);
        b3_round_g(v, 0, 5, 10, 15, m[8], m[9]);
        b3_round_g(v, 1, 6, 11, 12, m[10], m[11]);
        b3_round_g(v, 2, 7, 8, 13, m[12], m[13]);
        b3_round_g(v, 3, 4, 9, 14, m[14], m[15]);
        uint32_t p[16];
        for (int i = 0; i < 16; ++i) p[i] = m[B3P[i]];
        std::memcpy(m, p, 64);
    }
    for (int i = 0; i < 8; ++i) { out[i] = v[i] ^ v[i + 8]; out[i + 8] = v[i + 8] ^ cv[i]; }
}

namespace {
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };
struct B3Node { uint32_t cv[8]; uint32_t m[16]; uint64_t ctr; uint32_t blen, flags; };
void load_words(const uint8_t *p, size_t len, uint32_t m[16]) {
    uint8_t b[64] = {0};
    std::memcpy(b, p, len);
    for (int i = 0; i < 16; ++i) m[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 |
                                        (uint32_t)b[4 * i + 2] << 16 | (uint32_t)b[4 * i + 3] << 24;
}
B3Node chunk_node(const uint8_t *p, size_t len, uint64_t idx) {
    B3Node o;
    std::memcpy(o.cv, B3IV, 32);
    size_t nb = len ? (len + 63) / 64 : 1;
    uint32_t out[16];
    for (size_t b = 0; b + 1 < nb; ++b) {
        load_words(p + 64 * b, 64, o.m);
        b3_compress(o.cv, o.m, idx, 64, b ? 0 : CHUNK_START, out);
        std::memcpy(o.cv, out, 32);
    }
    size_t last = len - 64 * (nb - 1);
    load_words(p + 64 * (nb - 1), last, o.m);
    o.ctr = idx;
    o.blen = (uint32_t)last;
    o.flags = CHUNK_END | (nb == 1 ? CHUNK_START : 0);
    return o;
}
void node_cv(const B3Node &o, uint32_t cv[8]) {
    uint32_t out[16];
    b3_compress(o.cv, o.m, o.ctr, o.blen, o.flags, out);
    std::memcpy(cv, out, 32);
}
B3Node parent_node(const uint32_t l[8], const uint32_t r[8]) {
    B3Node o;
    std::memcpy(o.cv, B3IV, 32);
    std::memcpy(o.m, l, 32);
    std::memcpy(o.m + 8, r, 32);
    o.ctr = 0; o.blen = 64; o.flags = PARENT;
    return o;
}
}  // namespace

void blake3_hash(const uint8_t *msg, size_t len, uint8_t out[32]) {
    std::vector<std::array<uint32_t, 8>> stack;
    size_t chunks = len ? (len + 1023) / 1024 : 1;
    for (size_t c = 0; c + 1 < chunks; ++c) {
        std::array<uint32_t, 8> cv;
        node_cv(chunk_node(msg + 1024 * c, 1024, c), cv.data());
        for (uint64_t t = c + 1; (t & 1) == 0; t >>= 1) {
            node_cv(parent_node(stack.back().data(), cv.data()), cv.data());
            stack.pop_back();
        }
        stack.push_back(cv);
    }
    B3Node o = chunk_node(msg + 1024 * (chunks - 1), len - 1024 * (chunks - 1), chunks - 1);
    while (!stack.empty()) {
        uint32_t cv[8];
        node_cv(o, cv);
        o = parent_node(stack.back().data(), cv);
        stack.pop_back();
    }
    uint32_t res[16];
    b3_compress(o.cv, o.m, 0, o.blen, o.flags | ROOT, res);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)res[i]; out[4 * i + 1] = (uint8_t)(res[i] >> 8);
        out[4 * i + 2] = (uint8_t)(res[i] >> 16); out[4 * i + 3] = (uint8_t)(res[i] >> 24);
    }
}

// ================================================================= configs
// The reference asserts these relations while proving: poly length =
// initial m*n, initial_k = log2 n (rows vs gr, src/sumcheck_polys.rs:97),
// every committed size = the folded size, ks[i] = log2 dims[i].1, and at
// least 148 rows per commitment (get_distinct_queries terminates).
lg_status config_check(const lg_config &c, uint64_t poly_len) {
    if (c.recursive_steps < 1 || c.recursive_steps > LG_MAX_STEPS) return LG_ERR_INVALID_CONFIG;
    if (c.initial_log_m + c.initial_log_n > 34) return LG_ERR_INVALID_CONFIG;
    if (c.initial_k != c.initial_log_n || c.initial_k == 0 || c.initial_k > 8) return LG_ERR_INVALID_CONFIG;
    if (c.initial_log_m < 6 || c.initial_log_m > 26) return LG_ERR_INVALID_CONFIG;
    if (poly_len != (1ull << (c.initial_log_m + c.initial_log_n))) return LG_ERR_INVALID_CONFIG;
    uint32_t fv = c.initial_log_m;
    for (uint32_t i = 0; i < c.recursive_steps; ++i) {
        if (c.log_m[i] + c.log_n[i] != fv) return LG_ERR_INVALID_CONFIG;
        if (c.ks[i] != c.log_n[i] || c.ks[i] == 0 || c.ks[i] > 8) return LG_ERR_INVALID_CONFIG;
        if (c.log_m[i] < 6) return LG_ERR_INVALID_CONFIG;
        fv -= c.ks[i];
    }
    return LG_OK;
}

// ============================================================ proof codec
// "LGRP" u32 version=1 u32 field_bytes=4, then the fields of
// FinalizedLigeritoProof in order; byte strings and vectors carry a u32
// count (layout documented in the public header's design notes).
namespace {
struct Writer {
    std::vector<uint8_t> b;
    void raw(const void *p, size_t n) {
        const size_t at = b.size();
        b.resize(at + n);
        if (n) std::memcpy(b.data() + at, p, n);
    }
    void u32(uint32_t v) {
        const uint8_t x[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
        raw(x, 4);
    }
    void bytes(const uint8_t *p, size_t n) { u32((uint32_t)n); raw(p, n); }
    void bytes(const std::vector<uint8_t> &v) { bytes(v.data(), v.size()); }
    void words(const uint32_t *v, size_t n) {
        u32((uint32_t)n);
        const size_t at = b.size();
        b.resize(at + 4 * n);
        uint8_t *d = b.data() + at;
        for (size_t i = 0; i < n; ++i, d += 4) {
            const uint32_t x = v[i];
            d[0] = (uint8_t)x; d[1] = (uint8_t)(x >> 8); d[2] = (uint8_t)(x >> 16); d[3] = (uint8_t)(x >> 24);
        }
    }
    void words(const std::vector<uint32_t> &v) { words(v.data(), v.size()); }
    void opening(const Opening &o) {
        u32((uint32_t)o.rows.size());
        for (size_t i = 0; i < o.rows.size(); ++i) words(o.rows.ptr(i), o.rows.len(i));
        u32((uint32_t)o.merkle.size());
        for (size_t i = 0; i < o.merkle.size(); ++i) bytes(o.merkle.ptr(i), o.merkle.len(i));
    }
};
struct Reader {
    const uint8_t *p; size_t n, at = 0; bool bad = false;
    uint32_t u32() {
        if (bad || at + 4 > n) { bad = true; return 0; }
        uint32_t v = (uint32_t)p[at] | (uint32_t)p[at + 1] << 8 | (uint32_t)p[at + 2] << 16 | (uint32_t)p[at + 3] << 24;
        at += 4;
        return v;
    }
    bool count(uint32_t c, size_t unit) { if (bad || (uint64_t)c * unit > n - at) { bad = true; } return !bad; }
    void bytes(std::vector<uint8_t> &v) {
        uint32_t c = u32();
        if (!count(c, 1)) return;
        v.assign(p + at, p + at + c);
        at += c;
    }
    void words(std::vector<uint32_t> &v) {
        uint32_t c = u32();
        if (!count(c, 4)) return;
        v.resize(c);
        for (auto &x : v) x = u32();
    }
    void opening(Opening &o) {
        uint32_t r = u32();
        if (!count(r, 4)) return;
        o.rows.clear();
        o.rows.off.reserve(r + 1);
        std::vector<uint32_t> row;
        for (uint32_t i = 0; i < r && !bad; ++i) {
            words(row);
            if (!bad) o.rows.push(row.data(), row.size());
        }
        uint32_t s = u32();
        if (!count(s, 4)) return;
        o.merkle.clear();
        o.merkle.off.reserve(s + 1);
        for (uint32_t i = 0; i < s && !bad; ++i) {
            const uint32_t c = u32();
            if (!count(c, 1)) return;
            o.merkle.push(p + at, c);
            at += c;
        }
    }
};
}  // namespace

// Length of serialize(p), without building it
size_t serialized_size(const Proof &p) {
    auto op = [](const Opening &o) {
        size_t s = 8 + 4 * o.merkle.size() + o.merkle.data.size();
        s += 4 * o.rows.size() + 4 * o.rows.data.size();
        return s;
    };
    size_t s = 12 + 4 + p.initial_root.size() + 4 + op(p.initial) + 4 + 4 + 4 * p.yr.size() + op(p.final_) + 4 +
               12 * p.transcript.size();
    for (auto &r : p.recursive_roots) s += 4 + r.size();
    for (auto &o : p.recursive) s += op(o);
    return s;
}

std::vector<uint8_t> serialize(const Proof &p) {
    Writer w;
    w.b.reserve(serialized_size(p));
    w.b.insert(w.b.end(), {'L', 'G', 'R', 'P'});
    w.u32(1);
    w.u32(4);
    w.bytes(p.initial_root);
    w.u32((uint32_t)p.recursive_roots.size());
    for (auto &r : p.recursive_roots) w.bytes(r);
    w.opening(p.initial);
    w.u32((uint32_t)p.recursive.size());
    for (auto &o : p.recursive) w.opening(o);
    w.words(p.yr);
    w.opening(p.final_);
    w.u32((uint32_t)p.transcript.size());
    for (auto &t : p.transcript) { w.u32(t[0]); w.u32(t[1]); w.u32(t[2]); }
    return std::move(w.b);
}

bool deserialize(const uint8_t *buf, size_t len, Proof &p) {
    if (len < 12 || std::memcmp(buf, "LGRP", 4) != 0) return false;
    Reader r{buf, len, 4};
    if (r.u32() != 1 || r.u32() != 4) return false;
    r.bytes(p.initial_root);
    uint32_t nr = r.u32();
    if (!r.count(nr, 4)) return false;
    p.recursive_roots.resize(nr);
    for (auto &x : p.recursive_roots) r.bytes(x);
    r.opening(p.initial);
    uint32_t no = r.u32();
    if (!r.count(no, 8)) return false;
    p.recursive.resize(no);
    for (auto &o : p.recursive) r.opening(o);
    r.words(p.yr);
    r.opening(p.final_);
    uint32_t nt = r.u32();
    if (!r.count(nt, 12)) return false;
    p.transcript.resize(nt);
    for (auto &t : p.transcript) { t[0] = r.u32(); t[1] = r.u32(); t[2] = r.u32(); }
    return !r.bad && r.at == len;
}

// ProofSize: field bytes of rows + yr + transcript, plus proof / root bytes
uint64_t proof_size(const Proof &p) {
    auto op = [](const Opening &o) {
        uint64_t s = 0;
        s += 4 * o.rows.data.size();
        s += o.merkle.data.size();
        return s;
    };
    uint64_t s = p.initial_root.size() + op(p.initial) + op(p.final_) + 4 * p.yr.size() +
                 12 * p.transcript.size();
    for (auto &r : p.recursive_roots) s += r.size();
    for (auto &o : p.recursive) s += op(o);
    return s;
}

// ========================================================== Merkle indices
// ith_layer (src/merkle_tree.rs:62-96) without the hashes
void merkle_proof_nodes(const std::vector<uint64_t> &queries, uint64_t num_leaves,
                        std::vector<NodeRef> &out) {
    out.clear();
    std::vector<uint64_t> q = queries;
    size_t cnt = q.size();
    uint32_t depth = 0;
    while ((1ull << depth) < num_leaves) ++depth;
    for (uint32_t d = 0; d < depth; ++d) {
        size_t next = 0, i = 0;
        while (i < cnt) {
            uint64_t query = q[i], sib = query ^ 1;
            q[next++] = query >> 1;
            if (i == cnt - 1) { out.push_back({d, sib}); break; }
            if (query & 1) { out.push_back({d, sib}); i += 1; }
            else if (q[i + 1] != sib) { out.push_back({d, sib}); i += 1; }
            else { i += 2; }
        }
        cnt = next;
    }
}

static void hash_two(const uint8_t *l, const uint8_t *r, size_t rl_len, bool swap, uint8_t out[32]) {
    // hash_siblings (src/merkle_tree.rs:113-118): blake3(left || right)
    uint8_t buf[32 + 1024];
    size_t n = 0;
    if (!swap) { std::memcpy(buf, l, 32); std::memcpy(buf + 32, r, rl_len); n = 32 + rl_len; }
    else { std::memcpy(buf, r, rl_len); std::memcpy(buf + rl_len, l, 32); n = 32 + rl_len; }
    blake3_hash(buf, n, out);
}

// verify_ith_layer (src/merkle_tree.rs:120-162) + verify (:164-188)
bool merkle_verify(const uint8_t *root, size_t root_len,
                   const ByteList &proof, size_t depth,
                   std::vector<std::array<uint8_t, 32>> layer, std::vector<uint64_t> q, bool *ok) {
    size_t cur = q.size(), pc = 0;
    *ok = false;
    for (size_t d = 0; d < depth; ++d) {
        size_t next = 0, i = 0;
        while (i < cur) {
            uint64_t query = q[i], sib = query ^ 1;
            ++next;
            q[next - 1] = query >> 1;
            std::array<uint8_t, 32> h;
            if (i == cur - 1 || (query & 1) || q[i + 1] != sib) {
                ++pc;
                if (pc - 1 >= proof.size()) return false;  // index panic
                const size_t sl = proof.len(pc - 1);
                if (sl > 1024) return false;
                hash_two(layer[i].data(), proof.ptr(pc - 1), sl, (query & 1) != 0, h.data());
                layer[next - 1] = h;
                if (i == cur - 1) break;
                i += 1;
            } else {
                hash_two(layer[i].data(), layer[i + 1].data(), 32, false, h.data());
                layer[next - 1] = h;
                i += 2;
            }
        }
        cur = next;
    }
    *ok = cur == 1 && root_len == 32 && !layer.empty() && std::memcmp(layer[0].data(), root, 32) == 0;
    return true;
}

// ============================================================ setup tables
void compute_twiddles(uint32_t log_n, uint32_t *tw) {
    // Leaf layer (heap level log_n-1): 2u, written unscaled (s_prev_at_root = 1)
    std::vector<uint32_t> basis(log_n);  // layer value at index 2^b
    uint32_t L = log_n - 1;
    for (uint32_t b = 0; b < L; ++b) basis[b] = 2u << b;
    auto fill = [&](uint32_t level, uint32_t scale) {
        uint32_t *dst = tw + ((1ull << level) - 1);
        dst[0] = 0;  // layer value at index 0 is 0 (beta = 0), scaled stays 0
        for (uint32_t b = 0; b < level; ++b) {
            uint32_t add = gf_mul(scale, basis[b]);
            uint64_t half = 1ull << b;
            for (uint64_t u = 0; u < half; ++u) dst[half + u] = dst[u] ^ add;
        }
    };
    fill(L, 1);
    uint32_t c = 1;  // s_prev_at_root
    for (uint32_t level = L; level-- > 0;) {
        // layer_i (src/binary_fft.rs:74-89): s_at_root from layer[1] + layer[0]
        // (= basis[0]), new layer[w] = next_s(old[2w], c)
        uint32_t s_at_root = next_s(basis[0], c);
        for (uint32_t b = 0; b < level; ++b) basis[b] = next_s(basis[b + 1], c);
        c = s_at_root;
        fill(level, gf_inv(c));
    }
}

std::vector<uint32_t> eval_sk_at_vks(uint64_t n) {
    uint32_t ns = 0;
    while ((1ull << ns) < n) ++ns;
    std::vector<uint32_t> sk(ns + 1), layer(ns + 1);
    for (uint32_t i = 1; i <= ns; ++i) layer[i - 1] = 1u << i;
    sk[0] = 1;
    uint32_t cur = ns;
    for (uint32_t i = 1; i <= ns; ++i) {
        for (uint32_t j = 1; j <= cur; ++j) {
            if (j == 1) sk[i] = gf_mul(layer[0], layer[0]) ^ gf_mul(sk[i - 1], layer[0]);
            else layer[j - 2] = gf_mul(layer[j - 1], layer[j - 1]) ^ gf_mul(sk[i - 1], layer[j - 1]);
        }
        --cur;
    }
    return sk;
}

void compute_pis(uint64_t m, const std::vector<uint32_t> &sks, uint32_t *pis) {
    pis[0] = 1;
    for (size_t i = 2; i <= sks.size() && ((1ull << (i - 2)) < m); ++i) {
        uint64_t cur = 1ull << (i - 2);
        for (uint64_t j = 0; j < cur; ++j) pis[cur + j] = gf_mul(sks[i - 2], pis[j]);
    }
}

std::vector<uint32_t> lagrange_basis(const uint32_t *rs, size_t k) {
    std::vector<uint32_t> cur = {1u ^ rs[0], rs[0]}, nxt;
    for (size_t i = 1; i < k; ++i) {
        nxt.assign(cur.size() * 2, 0);
        uint32_t rp1 = 1u ^ rs[i];
        for (size_t j = 0; j < cur.size(); ++j) {
            nxt[2 * j] = gf_mul(cur[j], rp1);
            nxt[2 * j + 1] = gf_mul(cur[j], rs[i]);
        }
        cur.swap(nxt);
    }
    return cur;
}

void splitmix_fill(uint64_t seed, uint32_t *out, uint64_t n, uint64_t first) {
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t z = seed + (first + i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        out[i] = (uint32_t)(z ^ (z >> 31));
    }
}

}  // namespace lg
