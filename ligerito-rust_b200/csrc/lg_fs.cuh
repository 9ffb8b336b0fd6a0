// Device-side Fiat-Shamir transcript primitives (see lg_fs.cu), shared by
// the transcript kernels and by the sumcheck kernels whose last block runs
// a transcript step.
#pragma once
#include <cstdint>

#include "lg_kernels.h"

namespace lgk {
namespace fsd {
namespace {  // each translation unit keeps its own copy

__constant__ uint32_t kK256[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

__device__ __forceinline__ uint32_t rr(uint32_t x, int r) { return __funnelshift_r(x, x, r); }

// x + y on the multiply-add pipe (y * 1 + x, the 1 read from constant
// memory so the compiler keeps the multiply-add).  The transcript runs on
// one thread, whose rounds are bound by the logic pipe's issue rate (a
// warp instruction occupies its 16 lanes for two cycles): the rotations and
// logic stay there, the additions move to the otherwise idle pipe.
__constant__ uint32_t kOne = 1u;
__device__ __forceinline__ uint32_t addm(uint32_t x, uint32_t y) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(y), "r"(kOne), "r"(x));
    return r;
}
__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// FIPS 180-4 compression of one block of 16 big-endian words (registers).
// The transcript runs it on one thread or a few warps, where instruction
// fetch rather than arithmetic sets the pace: the 64 rounds are a loop of
// eight 8-round bodies (an eighth of the code of a full unroll; measured
// faster than a full unroll and slightly faster than 16-round bodies).
__device__ __forceinline__ void sha_compress(uint32_t st[8], const uint32_t (&blk)[16]) {
    // w holds W[t0 .. t0+15]; each trip runs 8 rounds on w[0..7], computes
    // W[t0+16 .. t0+23] and slides the window by 8
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = blk[i];
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll 1
    for (int t0 = 0; t0 < 64; t0 += 8) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t hk = addm(addm(h, kK256[t0 + i]), w[i]);  // independent of e: off the serial path
            const uint32_t t1 = addm(addm(hk, rr(e, 6) ^ rr(e, 11) ^ rr(e, 25)), (e & f) ^ (~e & g));
            const uint32_t t2 = addm(rr(a, 2) ^ rr(a, 13) ^ rr(a, 22), (a & b) ^ (a & c) ^ (b & c));
            h = g; g = f; f = e; e = addm(d, t1); d = c; c = b; b = a; a = addm(t1, t2);
        }
        if (t0 < 48) {
            uint32_t nw[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t x = w[i + 1], y = i >= 2 ? nw[i - 2] : w[i + 14];
                nw[i] = addm(addm(addm(rr(x, 7) ^ rr(x, 18) ^ (x >> 3), w[i]), i >= 7 ? nw[0] : w[i + 9]),
                             rr(y, 17) ^ rr(y, 19) ^ (y >> 10));
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) { w[i] = w[i + 8]; w[i + 8] = nw[i]; }
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) w[i] = w[i + 8];
        }
    }
    st[0] = addm(st[0], a); st[1] = addm(st[1], b); st[2] = addm(st[2], c); st[3] = addm(st[3], d);
    st[4] = addm(st[4], e); st[5] = addm(st[5], f); st[6] = addm(st[6], g); st[7] = addm(st[7], h);
}

// The 64 rounds of a compression whose K[t] + W[t] are already in kw (the
// message schedule computed elsewhere): the serial part alone.
__device__ __forceinline__ void sha_rounds_kw(uint32_t st[8], const uint32_t *kw) {
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll 1
    for (int t0 = 0; t0 < 64; t0 += 16) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const uint32_t hk = addm(h, kw[t0 + i]);
            const uint32_t t1 = addm(addm(hk, rr(e, 6) ^ rr(e, 11) ^ rr(e, 25)), (e & f) ^ (~e & g));
            const uint32_t t2 = addm(rr(a, 2) ^ rr(a, 13) ^ rr(a, 22), (a & b) ^ (a & c) ^ (b & c));
            h = g; g = f; f = e; e = addm(d, t1); d = c; c = b; b = a; a = addm(t1, t2);
        }
    }
    st[0] = addm(st[0], a); st[1] = addm(st[1], b); st[2] = addm(st[2], c); st[3] = addm(st[3], d);
    st[4] = addm(st[4], e); st[5] = addm(st[5], f); st[6] = addm(st[6], g); st[7] = addm(st[7], h);
}

// K[t] + W[t] (t < 64) of a block of 16 big-endian words.
__device__ __forceinline__ void sha_schedule_kw(const uint32_t (&blk)[16], uint32_t *kw) {
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = blk[i];
#pragma unroll 1
    for (int t0 = 0; t0 < 64; t0 += 16) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            if (t0 > 0) {
                const uint32_t x = w[(i + 1) & 15], y = w[(i + 14) & 15];
                w[i] += (rr(x, 7) ^ rr(x, 18) ^ (x >> 3)) + w[(i + 9) & 15] + (rr(y, 17) ^ rr(y, 19) ^ (y >> 10));
            }
            kw[t0 + i] = kK256[t0 + i] + w[i];
        }
    }
}

// Serial absorb of nwords u32s (their LE bytes) by one thread.
__device__ void fs_absorb(FsState &S, const uint32_t *src, uint32_t nwords) {
    for (uint32_t i = 0; i < nwords; ++i) {
        S.w[S.nw++] = bswap32(src[i]);
        if (S.nw == 16) {
            uint32_t blk[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) blk[k] = S.w[k];
            sha_compress(S.h, blk);
            S.nw = 0;
        }
    }
    S.total += 4ull * nwords;
}

// The whole block absorbs nwords u32s from device memory: each run of up
// to `cap` words is loaded in parallel into the shared `stage`, then
// thread 0 absorbs it, so the words cost one memory round trip per run
// instead of one each.  A non-null mirror receives a copy of the words.
__device__ void fs_absorb_block(FsState &S, const uint32_t *src, uint32_t nwords, uint32_t *stage, uint32_t cap,
                                uint32_t *mirror) {
    for (uint32_t base = 0; base < nwords; base += cap) {
        const uint32_t n = min(cap, nwords - base);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            stage[i] = src[base + i];
            if (mirror) mirror[base + i] = stage[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) fs_absorb(S, stage, n);
        __syncthreads();
    }
}

// The whole block absorbs a long run of nwords u32s from device memory:
// the words up to the first SHA-256 block boundary and after the last one
// go through fs_absorb on thread 0, and the whole blocks between have
// their message schedules computed in parallel (one block per thread,
// kKwBlocks at a time, into kw) so that thread 0 runs only the 64 rounds
// of each.  A non-null mirror receives a copy of the words.
constexpr uint32_t kKwBlocks = 32;
__device__ void fs_absorb_sched(FsState &S, const uint32_t *src, uint32_t nwords, uint32_t (*kw)[64],
                                uint32_t *mirror) {
    const uint32_t head = min(nwords, (16u - S.nw) & 15u);
    const uint32_t full = (nwords - head) / 16, done = head + 16 * full;
    if (threadIdx.x == 0) fs_absorb(S, src, head);
    if (mirror)
        for (uint32_t i = threadIdx.x; i < head; i += blockDim.x) mirror[i] = src[i];
    __syncthreads();
    for (uint32_t b0 = 0; b0 < full; b0 += kKwBlocks) {
        const uint32_t nb = min(kKwBlocks, full - b0);
        for (uint32_t t = threadIdx.x; t < nb; t += blockDim.x) {
            const uint32_t off = head + 16 * (b0 + t);
            uint32_t blk[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const uint32_t v = src[off + k];
                if (mirror) mirror[off + k] = v;
                blk[k] = bswap32(v);
            }
            sha_schedule_kw(blk, kw[t]);
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (uint32_t i = 0; i < nb; ++i) sha_rounds_kw(S.h, kw[i]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        S.total += 64ull * full;
        fs_absorb(S, src + done, nwords - done);
    }
    if (mirror)
        for (uint32_t i = done + threadIdx.x; i < nwords; i += blockDim.x) mirror[i] = src[i];
    __syncthreads();
}

// Word j of the pending words followed by the counters c, c+1, ... (each
// counter's LE bytes as a big-endian message word).
__device__ __forceinline__ uint32_t stream_word(const FsState &S, uint32_t j) {
    return j < S.nw ? S.w[j] : bswap32(S.counter + (j - S.nw));
}

constexpr uint32_t kQBlock = 256;  // threads of the query kernel = squeezes per batch = max queries
constexpr uint32_t kMaxChain = (15 + kQBlock) / 16 + 1;

struct Batch {
    uint32_t chain[kMaxChain][8];  // state after 0, 1, ... more full blocks
};

// Thread 0: the chain states after the full blocks that `cnt` more
// counters complete.
__device__ void fs_chain(const FsState &S, Batch &B, uint32_t cnt) {
    uint32_t st[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) B.chain[0][k] = st[k] = S.h[k];
    const uint32_t full = (S.nw + cnt) / 16;
    for (uint32_t f = 0; f < full; ++f) {
        uint32_t blk[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) blk[k] = stream_word(S, 16 * f + k);
        sha_compress(st, blk);
#pragma unroll
        for (int k = 0; k < 8; ++k) B.chain[f + 1][k] = st[k];
    }
}

// Low 64 bits of squeeze i of the batch (the finalised clone after i+1
// counters), given the chain states.
__device__ uint64_t fs_squeeze_at(const FsState &S, const Batch &B, uint32_t i) {
    const uint32_t len = S.nw + i + 1, fb = len / 16, rem = len - 16 * fb;
    uint32_t st[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) st[k] = B.chain[fb][k];
    const uint64_t bits = (S.total + 4ull * (i + 1)) * 8;
    const uint32_t nblk = rem + 3 <= 16 ? 1 : 2;  // data, the 0x80 word, the 64-bit length
    for (uint32_t t = 0; t < nblk; ++t) {
        uint32_t blk[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const uint32_t j = 16 * t + k;
            uint32_t v = 0;
            if (j < rem) v = stream_word(S, 16 * fb + j);
            else if (j == rem) v = 0x80000000u;
            if (j == 16 * nblk - 2) v = (uint32_t)(bits >> 32);
            if (j == 16 * nblk - 1) v = (uint32_t)bits;
            blk[k] = v;
        }
        sha_compress(st, blk);
    }
    return (uint64_t)bswap32(st[0]) | ((uint64_t)bswap32(st[1]) << 32);
}

// Thread 0: advance the state past `take` squeezes of the batch.
__device__ void fs_commit(FsState &S, const Batch &B, uint32_t take) {
    const uint32_t len = S.nw + take, fb = len / 16, rem = len - 16 * fb;
    uint32_t nw[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) nw[k] = (uint32_t)k < rem ? stream_word(S, 16 * fb + k) : 0u;
#pragma unroll
    for (int k = 0; k < 16; ++k) S.w[k] = nw[k];
#pragma unroll
    for (int k = 0; k < 8; ++k) S.h[k] = B.chain[fb][k];
    S.nw = rem;
    S.total += 4ull * take;
    S.counter += take;
}

// nsq field elements into out; the whole block calls it.
__device__ void fs_fields(FsState &S, Batch &B, uint32_t nsq, uint32_t *out) {
    for (uint32_t done = 0; done < nsq;) {
        const uint32_t cnt = min(blockDim.x, nsq - done);
        if (threadIdx.x == 0) fs_chain(S, B, cnt);
        __syncthreads();
        if (threadIdx.x < cnt) out[done + threadIdx.x] = (uint32_t)fs_squeeze_at(S, B, threadIdx.x);
        __syncthreads();
        if (threadIdx.x == 0) fs_commit(S, B, cnt);
        __syncthreads();
        done += cnt;
    }
}

__device__ void load_state(FsState &S, const FsState *g) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(g);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&S);
    for (uint32_t i = threadIdx.x; i < sizeof(FsState) / 4; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}
__device__ void store_state(const FsState &S, FsState *g) {
    __syncthreads();
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&S);
    uint32_t *dst = reinterpret_cast<uint32_t *>(g);
    for (uint32_t i = threadIdx.x; i < sizeof(FsState) / 4; i += blockDim.x) dst[i] = src[i];
}

// The transcript step of a sumcheck kernel (FsTail), run by its last block
// to finish: every block has added its share of the triple at acc3; the
// last one reads the total, checks it against the enforced sum acc3[3] when
// asked, absorbs it and squeezes t.nsq challenges.  No block waits: a block
// that is not last returns.
// Every block reads the transcript state at its start (fs_tail_prefetch,
// one word per thread; nothing writes it before the last block does), so
// the last block does not wait for that read after learning it is last.
constexpr uint32_t kFsStateWords = sizeof(FsState) / 4;
static_assert(kFsStateWords <= 64, "the state is prefetched by the first threads of a block");
__device__ __forceinline__ uint32_t fs_tail_prefetch(const FsTail &t) {
    return t.fs && threadIdx.x < kFsStateWords ? reinterpret_cast<const uint32_t *>(t.fs)[threadIdx.x] : 0u;
}
__device__ void fs_tail_block(const FsTail &t, uint32_t *acc3, uint32_t pre) {
    __shared__ FsState S;
    __shared__ Batch B;
    __shared__ uint32_t tri[4];
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(t.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 4) tri[threadIdx.x] = atomicOr(acc3 + threadIdx.x, 0u);
    if (threadIdx.x < kFsStateWords) reinterpret_cast<uint32_t *>(&S)[threadIdx.x] = pre;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (t.check && (tri[0] ^ tri[1]) != tri[3]) S.err |= FS_ERR_SUMCHECK;
        fs_absorb(S, tri, 3);
        *t.ticket = 0;
    }
    __syncthreads();
    fs_fields(S, B, t.nsq, t.out);
    store_state(S, t.fs);
}

}  // namespace
}  // namespace fsd
}  // namespace lgk
