// Device primitives for liblgpu (sm_100a): GF(2^32) arithmetic and BLAKE3.
//
// GF(2^32) = GF(2)[x] / (x^32 + x^15 + x^9 + x^7 + x^4 + x^3 + 1), the
// polynomial basis of src/binary_field.rs:179-181.  There is no carry-less
// multiply instruction, so two forms are used:
//   * gf_mul(a, b): a general product from 16 32x32->64 integer multiplies
//     of operands masked to every 4th bit (each partial-product coefficient
//     is a count <= 8 < 16, so the integer sums never carry into the next
//     4-bit lane), XOR-combined and reduced.
//   * MulTab: a per-constant table of c * e * x^(w*B) for every B-bit window
//     value e; c * v is then the XOR of one table word per window of v.
//     Warps look a constant's table up together, so all lanes read one
//     32-word bank row (conflict-free).  Used wherever many products share a
//     multiplier: FFT twiddles (shared across all matrix columns), fold
//     challenges, sumcheck challenges, basis-expansion constants.
#pragma once
#include <cstdint>

namespace lgd {

// Programmatic dependent launch: wait until the previous grid on the
// stream has completed and its writes are visible, then let the next grid
// start launching (its blocks in turn wait here).  A no-op for launches
// without the attribute.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

constexpr uint32_t kTail = 0x8299u;  // x^32 mod p

__device__ __forceinline__ uint32_t red_small(uint32_t t) {
    // t * (x^15 + x^9 + x^7 + x^4 + x^3 + 1) for deg t <= 16 (no overflow)
    return t ^ (t << 3) ^ (t << 4) ^ (t << 7) ^ (t << 9) ^ (t << 15);
}

__device__ __forceinline__ uint32_t gf_mulx(uint32_t a) {
    return (a << 1) ^ ((uint32_t)((int32_t)a >> 31) & kTail);
}
// a * x^k for 1 <= k <= 16
template <int K>
__device__ __forceinline__ uint32_t gf_mulxk(uint32_t a) {
    return (a << K) ^ red_small(a >> (32 - K));
}

__device__ __forceinline__ uint32_t gf_reduce(uint32_t hi, uint32_t lo) {
    uint32_t lo2 = hi ^ (hi << 3) ^ (hi << 4) ^ (hi << 7) ^ (hi << 9) ^ (hi << 15);
    uint32_t ov = (hi >> 29) ^ (hi >> 28) ^ (hi >> 25) ^ (hi >> 23) ^ (hi >> 17);
    return lo ^ lo2 ^ red_small(ov);
}

// Carry-less 32 x 32 -> 64-bit product: 16 integer multiplies of operands
// masked to every 4th bit (at most 8 ones meet at a position, so sums never
// carry into the next position of the same class).
__device__ __forceinline__ uint64_t clmul32(uint32_t a, uint32_t b) {
    const uint32_t m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u, m3 = 0x88888888u;
    uint32_t a0 = a & m0, a1 = a & m1, a2 = a & m2, a3 = a & m3;
    uint32_t b0 = b & m0, b1 = b & m1, b2 = b & m2, b3 = b & m3;
    uint64_t z0 = ((uint64_t)a0 * b0) ^ ((uint64_t)a1 * b3) ^ ((uint64_t)a2 * b2) ^ ((uint64_t)a3 * b1);
    uint64_t z1 = ((uint64_t)a0 * b1) ^ ((uint64_t)a1 * b0) ^ ((uint64_t)a2 * b3) ^ ((uint64_t)a3 * b2);
    uint64_t z2 = ((uint64_t)a0 * b2) ^ ((uint64_t)a1 * b1) ^ ((uint64_t)a2 * b0) ^ ((uint64_t)a3 * b3);
    uint64_t z3 = ((uint64_t)a0 * b3) ^ ((uint64_t)a1 * b2) ^ ((uint64_t)a2 * b1) ^ ((uint64_t)a3 * b0);
    return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) | (z2 & 0x4444444444444444ull) |
           (z3 & 0x8888888888888888ull);
}

__device__ __forceinline__ uint32_t gf_mul(uint32_t a, uint32_t b) {
    const uint64_t r = clmul32(a, b);
    return gf_reduce((uint32_t)(r >> 32), (uint32_t)r);
}

// ------------------------------------------------------------ GF(2^128)
// BinaryElem128 (x^128 + x^7 + x^2 + x + 1): two u64 limbs, low first.
struct U128 {
    uint64_t lo, hi;
};
// carry-less 64 x 64 -> 128 by Karatsuba over 32-bit halves (3 clmul32)
__device__ __forceinline__ U128 clmul64(uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    const uint64_t lo = clmul32(a0, b0), hi = clmul32(a1, b1), mid = clmul32(a0 ^ a1, b0 ^ b1) ^ lo ^ hi;
    return {lo ^ (mid << 32), hi ^ (mid >> 32)};
}
// product by Karatsuba over 64-bit halves (9 clmul32), then the 256-bit
// product's top half H folds down as H * (x^7 + x^2 + x + 1); the at most
// 7 bits that H * x^k (k = 1, 2, 7) pushes past x^127 fold once more.
__device__ __forceinline__ U128 gf128_mul(U128 a, U128 b) {
    const U128 l = clmul64(a.lo, b.lo), h = clmul64(a.hi, b.hi), m = clmul64(a.lo ^ a.hi, b.lo ^ b.hi);
    const uint64_t p0 = l.lo, p1 = l.hi ^ m.lo ^ l.lo ^ h.lo, p2 = h.lo ^ m.hi ^ l.hi ^ h.hi, p3 = h.hi;
    const uint64_t ov = (p3 >> 63) ^ (p3 >> 62) ^ (p3 >> 57);
    const uint64_t r0 = p0 ^ p2 ^ (p2 << 1) ^ (p2 << 2) ^ (p2 << 7) ^ ov ^ (ov << 1) ^ (ov << 2) ^ (ov << 7);
    const uint64_t r1 = p1 ^ p3 ^ (p3 << 1) ^ (p2 >> 63) ^ (p3 << 2) ^ (p2 >> 62) ^ (p3 << 7) ^ (p2 >> 57);
    return {r0, r1};
}

// ---------------------------------------------------------------- MulTab
// 4-bit windows: 8 windows x 16 entries = 128 words (512 B) per constant.
constexpr int kTabWords = 128;

// Table builds run their carry-less products on the multiply-add pipe,
// which the table kernels otherwise leave idle: an integer product t * k
// equals the carry-less one when the shifted copies of t that k's set bits
// make never overlap.  The multipliers come from constant memory so the
// compiler keeps them multiplies.
static __constant__ uint32_t kTabMul[9] = {
    256u,     // v x^8 (the low word)
    0x201u,   // t (1 + x^9), t < 2^8
    0x8080u,  // t (x^7 + x^15), t < 2^8
    8u,       // t x^3
    16u,      // t x^4, and v x^4 (the low word)
    0x8211u,  // t (1 + x^4 + x^9 + x^15), t < 2^4
    0x88u,    // t (x^3 + x^7), t < 2^4
    0x8089u,  // t (1 + x^3 + x^7 + x^15), t < 2^3
    0x210u,   // t (x^4 + x^9), t < 2^3
};
__device__ __forceinline__ uint32_t fma_mul(uint32_t a, uint32_t k) {
    uint32_t r;
    asm("mul.lo.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(k));
    return r;
}
__device__ __forceinline__ uint64_t fma_mul_wide(uint32_t a, uint32_t k) {
    uint64_t r;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(r) : "r"(a), "r"(k));
    return r;
}
// v x^8 mod p: (v << 8) ^ t (x^15 + x^9 + x^7 + x^4 + x^3 + 1), t = v >> 24,
// the tail split into the non-overlapping shift sets {0, 9}, {7, 15}, {3}, {4}
__device__ __forceinline__ uint32_t tab_mulx8(uint32_t v) {
    const uint32_t t = v >> 24;
    return fma_mul(v, kTabMul[0]) ^ fma_mul(t, kTabMul[1]) ^ fma_mul(t, kTabMul[2]) ^ fma_mul(t, kTabMul[3]) ^
           fma_mul(t, kTabMul[4]);
}

// One warp builds the table of constant c (all 32 lanes participate): lane
// l writes entries l, 32 + l, 64 + l, 96 + l, i.e. c e x^(4w) for e = l & 15
// and windows w = 2j + (l >> 4), j < 4.  c e is a carry-less product by a
// 4-bit e: c's bits taken every 4th (four masks) times e never carry, so it
// is four wide integer products XORed; the at most 3 bits past x^31 fold
// back through the tail.  Lanes 16-31 start from c x^4; each next pair of
// windows is a multiplication by x^8.
__device__ __forceinline__ void tab_entries(uint32_t c, int lane, uint32_t (&v)[4]) {
    const uint32_t t4 = c >> 28;
    const uint32_t c4 = fma_mul(c, kTabMul[4]) ^ fma_mul(t4, kTabMul[5]) ^ fma_mul(t4, kTabMul[6]);
    const uint32_t cs = (lane & 16) ? c4 : c, e = lane & 15;
    const uint64_t p = fma_mul_wide(cs & 0x11111111u, e) ^ fma_mul_wide(cs & 0x22222222u, e) ^
                       fma_mul_wide(cs & 0x44444444u, e) ^ fma_mul_wide(cs & 0x88888888u, e);
    const uint32_t hi = (uint32_t)(p >> 32);
    v[0] = (uint32_t)p ^ fma_mul(hi, kTabMul[7]) ^ fma_mul(hi, kTabMul[8]);
    v[1] = tab_mulx8(v[0]);
    v[2] = tab_mulx8(v[1]);
    v[3] = tab_mulx8(v[2]);
}
__device__ __forceinline__ void tab_build_warp(uint32_t *T, uint32_t c, int lane) {
    uint32_t v[4];
    tab_entries(c, lane, v);
#pragma unroll
    for (int j = 0; j < 4; ++j) T[32 * j + lane] = v[j];
}
// The same table with the products on the logic pipe only (shifts and
// XORs): fewer instructions than tab_build_warp's multiply-add form, which
// pays off where the kernel is bound by instruction issue and a table
// serves few products (rs_scale builds one per matrix row: 47.3 M against
// 52.9 M warp instructions per launch at 2^24).
__device__ __forceinline__ void tab_build_warp_logic(uint32_t *T, uint32_t c, int lane) {
    const uint32_t c1 = gf_mulx(c), c2 = gf_mulx(c1), c3 = gf_mulx(c2);
    const int e = lane & 15;
    uint32_t v = ((e & 1) ? c : 0u) ^ ((e & 2) ? c1 : 0u) ^ ((e & 4) ? c2 : 0u) ^ ((e & 8) ? c3 : 0u);
    if (lane & 16) v = gf_mulxk<4>(v);
    T[lane] = v;
    v = gf_mulxk<8>(v);
    T[32 + lane] = v;
    v = gf_mulxk<8>(v);
    T[64 + lane] = v;
    v = gf_mulxk<8>(v);
    T[96 + lane] = v;
}
// The tables of two constants interleaved: entry (w, e) = (c0 e x^(4w),
// c1 e x^(4w)) in 8 bytes at byte 128 w + 8 e (1 KB a pair).  For values
// multiplied by both constants (tab2_mul_sa) the nibble spreads and byte
// permutes are paid once and each window is one 64-bit load; a half-warp
// reads 16 distinct entries of a 128-byte window, conflict-free.
__device__ __forceinline__ void tab2_build_warp(uint2 *T, uint32_t c0, uint32_t c1, int lane) {
    uint32_t v0[4], v1[4];
    tab_entries(c0, lane, v0);
    tab_entries(c1, lane, v1);
#pragma unroll
    for (int j = 0; j < 4; ++j) T[32 * j + lane] = make_uint2(v0[j], v1[j]);
}

// Same product with the table at byte offset base + off of the shared
// array `sm`, base a multiple of 256 (its low byte is zero) and off a
// constant after unrolling.  Byte j of a (b) holds 4 * nibble 2j (2j+1) of
// w, the byte offset of that window's entry; one byte-permute splices it
// under `base`, and off + the window's 64-byte slot fold into the load's
// immediate.  Per product: 2 multiplies and 2 ANDs to spread the nibbles, 8
// permutes, 8 loads, 4 XORs.
// p + t * stride_bytes as one wide multiply-add on the multiply-add pipe
// (the strided FFT passes address 2^K pencil values this way, keeping the
// integer-logic pipe for the field products)
template <class T>
__device__ __forceinline__ T *strided(T *p, uint32_t t, uint32_t stride_bytes) {
    T *r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(t), "r"(stride_bytes), "l"(p));
    return r;
}

__device__ __forceinline__ uint32_t shared_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// The two nibble spreads' shifts run as multiplies on the multiply-add pipe
// (w * 4, and the high word of w * 2^30 = w >> 2): a table product is
// otherwise all integer-logic work (the byte permutes and XORs), and that
// pipe is what bounds the table kernels.  The multipliers come from
// constant memory so the compiler keeps them multiplies.
static __constant__ uint32_t kSpreadMul[2] = {4u, 1u << 30};
__device__ __forceinline__ uint32_t tab_mul_sa(const uint8_t *__restrict__ sm, uint32_t base, uint32_t off,
                                               uint32_t w) {
    uint32_t a, b;
    asm("mul.lo.u32 %0, %1, %2;" : "=r"(a) : "r"(w), "r"(kSpreadMul[0]));
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(b) : "r"(w), "r"(kSpreadMul[1]));
    a &= 0x3C3C3C3Cu;
    b &= 0x3C3C3C3Cu;
#define LGD_LD(x, sel, o) (*reinterpret_cast<const uint32_t *>(sm + __byte_perm((x), base, (sel)) + off + (o)))
    const uint32_t r0 = LGD_LD(a, 0x7650, 0), r1 = LGD_LD(b, 0x7650, 64);
    const uint32_t r2 = LGD_LD(a, 0x7651, 128), r3 = LGD_LD(b, 0x7651, 192);
    const uint32_t r4 = LGD_LD(a, 0x7652, 256), r5 = LGD_LD(b, 0x7652, 320);
    const uint32_t r6 = LGD_LD(a, 0x7653, 384), r7 = LGD_LD(b, 0x7653, 448);
#undef LGD_LD
    return (r0 ^ r1 ^ r2) ^ (r3 ^ r4 ^ r5) ^ (r6 ^ r7);
}
// w times both constants of the pair table at byte offset base of `sm`
// (base a multiple of 256): byte j of a (b) holds 8 * nibble 2j (2j+1) of
// w, the byte offset of that window's 8-byte entry.
static __constant__ uint32_t kSpreadMul2[2] = {8u, 1u << 31};
__device__ __forceinline__ uint2 tab2_mul_sa(const uint8_t *__restrict__ sm, uint32_t base, uint32_t w) {
    uint32_t a, b;
    asm("mul.lo.u32 %0, %1, %2;" : "=r"(a) : "r"(w), "r"(kSpreadMul2[0]));
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(b) : "r"(w), "r"(kSpreadMul2[1]));
    a &= 0x78787878u;
    b &= 0x78787878u;
#define LGD_LD2(x, sel, o) (*reinterpret_cast<const uint2 *>(sm + __byte_perm((x), base, (sel)) + (o)))
    const uint2 r0 = LGD_LD2(a, 0x7650, 0), r1 = LGD_LD2(b, 0x7650, 128);
    const uint2 r2 = LGD_LD2(a, 0x7651, 256), r3 = LGD_LD2(b, 0x7651, 384);
    const uint2 r4 = LGD_LD2(a, 0x7652, 512), r5 = LGD_LD2(b, 0x7652, 640);
    const uint2 r6 = LGD_LD2(a, 0x7653, 768), r7 = LGD_LD2(b, 0x7653, 896);
#undef LGD_LD2
    return make_uint2((r0.x ^ r1.x ^ r2.x) ^ (r3.x ^ r4.x ^ r5.x) ^ (r6.x ^ r7.x),
                      (r0.y ^ r1.y ^ r2.y) ^ (r3.y ^ r4.y ^ r5.y) ^ (r6.y ^ r7.y));
}

// ---------------------------------------------------------------- BLAKE3
// BLAKE3 compression (BLAKE3 specification; the reference calls the blake3
// crate, src/merkle_tree.rs:15,50).  Message schedule unrolled at compile
// time; rotations by 16/8 are byte permutes, 12/7 funnel shifts.
enum : uint32_t { B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_ROOT = 8 };

__device__ __forceinline__ uint32_t rotr16(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t rotr8(uint32_t x) { return __byte_perm(x, 0, 0x0321); }
__device__ __forceinline__ uint32_t rotr12(uint32_t x) { return __funnelshift_r(x, x, 12); }
__device__ __forceinline__ uint32_t rotr7(uint32_t x) { return __funnelshift_r(x, x, 7); }

// x + y*one on the multiply-add pipe: BLAKE3 is bound by the integer ALU
// pipe (adds, XORs, rotates) while the FMA pipe idles, so with `one` a
// runtime 1 (a kernel argument the compiler cannot fold) all the additions
// of G move there (six multiply-adds; measured 2.5% faster than keeping
// one three-input add on the ALU).  Same sum, modulo 2^32.
__device__ __forceinline__ uint32_t add_fma(uint32_t x, uint32_t y, uint32_t one) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(y), "r"(one), "r"(x));
    return r;
}

#define LGD_B3G(a, b, c, d, x, y)                                   \
    a = add_fma(add_fma(a, b, one), (x), one); d = rotr16(d ^ a);   \
    c = add_fma(c, d, one);                    b = rotr12(b ^ c);   \
    a = add_fma(add_fma(a, b, one), (y), one); d = rotr8(d ^ a);    \
    c = add_fma(c, d, one);                    b = rotr7(b ^ c);

// Message schedule: entry (r, i) is the message word at position i of
// round r, i.e. the spec's permutation applied r times, as compile-time
// constants so the message words stay in registers.
#define LGD_S(r, i) (B3SchedC<r, i>::value)
template <int R, int I> struct B3SchedC;
#define LGD_DEF_ROW(r, a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15) \
    template <> struct B3SchedC<r, 0> { static constexpr int value = a0; };                 \
    template <> struct B3SchedC<r, 1> { static constexpr int value = a1; };                 \
    template <> struct B3SchedC<r, 2> { static constexpr int value = a2; };                 \
    template <> struct B3SchedC<r, 3> { static constexpr int value = a3; };                 \
    template <> struct B3SchedC<r, 4> { static constexpr int value = a4; };                 \
    template <> struct B3SchedC<r, 5> { static constexpr int value = a5; };                 \
    template <> struct B3SchedC<r, 6> { static constexpr int value = a6; };                 \
    template <> struct B3SchedC<r, 7> { static constexpr int value = a7; };                 \
    template <> struct B3SchedC<r, 8> { static constexpr int value = a8; };                 \
    template <> struct B3SchedC<r, 9> { static constexpr int value = a9; };                 \
    template <> struct B3SchedC<r, 10> { static constexpr int value = a10; };               \
    template <> struct B3SchedC<r, 11> { static constexpr int value = a11; };               \
    template <> struct B3SchedC<r, 12> { static constexpr int value = a12; };               \
    template <> struct B3SchedC<r, 13> { static constexpr int value = a13; };               \
    template <> struct B3SchedC<r, 14> { static constexpr int value = a14; };               \
    template <> struct B3SchedC<r, 15> { static constexpr int value = a15; };
LGD_DEF_ROW(0, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
LGD_DEF_ROW(1, 2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8)
LGD_DEF_ROW(2, 3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1)
LGD_DEF_ROW(3, 10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6)
LGD_DEF_ROW(4, 12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4)
LGD_DEF_ROW(5, 9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7)
LGD_DEF_ROW(6, 11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13)
#undef LGD_DEF_ROW

template <int R>
__device__ __forceinline__ void b3_round(uint32_t (&v)[16], const uint32_t (&m)[16], uint32_t one) {
    LGD_B3G(v[0], v[4], v[8], v[12], m[LGD_S(R, 0)], m[LGD_S(R, 1)])
    LGD_B3G(v[1], v[5], v[9], v[13], m[LGD_S(R, 2)], m[LGD_S(R, 3)])
    LGD_B3G(v[2], v[6], v[10], v[14], m[LGD_S(R, 4)], m[LGD_S(R, 5)])
    LGD_B3G(v[3], v[7], v[11], v[15], m[LGD_S(R, 6)], m[LGD_S(R, 7)])
    LGD_B3G(v[0], v[5], v[10], v[15], m[LGD_S(R, 8)], m[LGD_S(R, 9)])
    LGD_B3G(v[1], v[6], v[11], v[12], m[LGD_S(R, 10)], m[LGD_S(R, 11)])
    LGD_B3G(v[2], v[7], v[8], v[13], m[LGD_S(R, 12)], m[LGD_S(R, 13)])
    LGD_B3G(v[3], v[4], v[9], v[14], m[LGD_S(R, 14)], m[LGD_S(R, 15)])
}

// cv <- first 8 words of compress(cv, m, counter = 0, blen, flags); `one`
// must be 1 (see add_fma).
__device__ __forceinline__ void b3_compress(uint32_t (&cv)[8], const uint32_t (&m)[16], uint32_t blen,
                                            uint32_t flags, uint32_t one) {
    uint32_t v[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au, 0u, 0u, blen, flags};
    b3_round<0>(v, m, one);
    b3_round<1>(v, m, one);
    b3_round<2>(v, m, one);
    b3_round<3>(v, m, one);
    b3_round<4>(v, m, one);
    b3_round<5>(v, m, one);
    b3_round<6>(v, m, one);
#pragma unroll
    for (int i = 0; i < 8; ++i) cv[i] = v[i] ^ v[i + 8];
}

__device__ __forceinline__ void b3_iv(uint32_t (&cv)[8]) {
    cv[0] = 0x6A09E667u; cv[1] = 0xBB67AE85u; cv[2] = 0x3C6EF372u; cv[3] = 0xA54FF53Au;
    cv[4] = 0x510E527Fu; cv[5] = 0x9B05688Cu; cv[6] = 0x1F83D9ABu; cv[7] = 0x5BE0CD19u;
}

}  // namespace lgd
