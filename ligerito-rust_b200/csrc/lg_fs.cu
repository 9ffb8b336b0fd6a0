// Fiat-Shamir transcript on the device: the prover's challenges, queries
// and Merkle opening lists come from here, so a proof runs as one stream
// of kernels without host round trips.
//
// The transcript (src/emulated_fs.rs:6-76) is a running SHA-256 (sha2
// 0.10.9, FIPS 180-4): absorb appends bytes; squeeze appends the LE u32
// counter, increments it and finalises a clone of the state; a field
// element is the low 32 bits of the digest's first 16 bytes read as a LE
// u128, a query the low 64 bits mod n.  get_distinct_queries rejects
// repeats and sorts.  Everything absorbed is whole u32s, so the pending
// message is kept as big-endian words.
//
// Absorbing is serial (one thread).  Squeezes are batched: squeeze i of a
// batch finalises the state after i+1 more counters, so one thread
// compresses the full blocks those counters complete (the only serial
// part), then every thread finalises its own clone in parallel.
#include <cstdint>

#include "lg_device.cuh"
#include "lg_fs.cuh"

namespace lgk {

namespace {

using namespace fsd;
using lgd::pdl_begin;

__global__ void k_fs_init(FsState *g, uint32_t seed) {
    pdl_begin();
    g += blockIdx.x;  // lockstep batch: one block per proof
    __shared__ FsState S;
    if (threadIdx.x == 0) {
        const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
        for (int k = 0; k < 8; ++k) S.h[k] = iv[k];
        S.nw = 0;
        S.total = 0;
        S.counter = 0;
        S.err = 0;
        S.pad = 0;
        fs_absorb(S, &seed, 1);  // FS::new(seed): the seed's LE bytes
    }
    store_state(S, g);
}

__global__ void k_fs_step(FsState *g, FsStep a, FsStrides st) {
    pdl_begin();
    {
        const uint32_t b = blockIdx.x;  // lockstep batch: one block per proof
        g += b;
        a.src += b * st.src;
        if (a.out) a.out += b * st.out;
        if (a.mirror) a.mirror += b * st.mirror;
    }
    __shared__ FsState S;
    __shared__ Batch B;
    __shared__ uint32_t stage[32];
    __shared__ uint32_t kw[kKwBlocks][64];
    load_state(S, g);
    const bool bad = threadIdx.x == 0 && a.check && (a.src[0] ^ a.src[1]) != a.src[3];
    // long runs (yr) with the message schedules in parallel
    if (a.nwords >= 64) fs_absorb_sched(S, a.src, a.nwords, kw, a.mirror);
    else fs_absorb_block(S, a.src, a.nwords, stage, 32, a.mirror);
    if (bad) S.err |= FS_ERR_SUMCHECK;
    __syncthreads();
    fs_fields(S, B, a.nsq, a.out);
    store_state(S, g);
}

// Exclusive prefix count of `flag` over the block (kQBlock threads) and
// the total; `scratch` holds kQBlock / 32 words.
__device__ uint32_t block_rank(bool flag, uint32_t *scratch, uint32_t *total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t m = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) scratch[warp] = __popc(m);
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t w = 0; w < kQBlock / 32; ++w) {
        const uint32_t c = scratch[w];
        before += w < warp ? c : 0;
        all += c;
    }
    __syncthreads();
    *total = all;
    return before + __popc(m & ((1u << lane) - 1));
}

// At most 2 kQBlock values (the queries taken and a batch) go into a set
// of kHash slots, so probing always ends within the table.
constexpr uint32_t kHash = 4 * kQBlock;
static_assert(kHash == 1024, "hash_insert takes 10 bits of the hash");
__device__ uint32_t hash_insert(unsigned long long *key, uint32_t *rank, uint64_t v, uint32_t r) {
    uint32_t h = ((uint32_t)(v ^ (v >> 31)) * 0x9E3779B1u) >> 22;  // 10 bits: kHash = 1024 slots
    for (uint32_t probe = 0; probe < kHash; ++probe) {
        const unsigned long long prev = atomicCAS(key + h, ~0ull, (unsigned long long)v);
        if (prev == ~0ull || prev == v) {
            atomicMin(rank + h, r);
            return h;
        }
        h = (h + 1) & (kHash - 1);
    }
    return kHash - 1;  // unreachable: the table is never more than half full
}

// The chain of a batch (see fs_chain) from schedules prepared by the block:
// thread t < full writes K + W of chain block t to kw[t], then thread 0
// runs only the rounds.  The whole block calls it.
__device__ void fs_chain_block(const FsState &S, Batch &B, uint32_t cnt, uint32_t (*kw)[64]) {
    const uint32_t full = (S.nw + cnt) / 16;
    if (threadIdx.x < full) {
        uint32_t blk[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) blk[k] = stream_word(S, 16 * threadIdx.x + k);
        sha_schedule_kw(blk, kw[threadIdx.x]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t st[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) B.chain[0][k] = st[k] = S.h[k];
        for (uint32_t f = 0; f < full; ++f) {
            sha_rounds_kw(st, kw[f]);
#pragma unroll
            for (int k = 0; k < 8; ++k) B.chain[f + 1][k] = st[k];
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kQBlock) k_fs_queries(FsState *g, FsQueries a, FsStrides st) {
    pdl_begin();
    {
        const uint32_t b = blockIdx.x;  // lockstep batch: one block per proof
        g += b;
        if (a.src) a.src += b * st.src;
        if (a.out) a.out += b * st.out;
        if (a.mirror) a.mirror += b * st.mirror;
        a.q += b * st.q;
        a.nodes += b * st.nodes;
        a.nnodes += b * st.nnodes;
    }
    __shared__ FsState S;
    __shared__ Batch B;
    __shared__ uint64_t acc[kQBlock];
    __shared__ unsigned long long hkey[kHash];
    __shared__ uint32_t hrank[kHash];
    __shared__ uint32_t lo32[kQBlock];
    __shared__ uint32_t scratch[kQBlock / 32];
    __shared__ uint32_t wcnt[64][kQBlock / 32], wmask[64][kQBlock / 32];
    __shared__ uint64_t sq[kQBlock];     // a batch's squeezes, by index
    __shared__ uint32_t order[kQBlock];  // squeeze index of each thread
    __shared__ uint32_t take_sh, batch_sh;
    __shared__ uint32_t kw[kMaxChain][64];
    const uint32_t tid = threadIdx.x;
    load_state(S, g);
    fs_absorb_block(S, a.src, a.nwords, lo32, kQBlock, a.mirror);
    const bool ok = a.n >= a.s && a.s >= 1 && a.s <= kQBlock;
    const uint64_t mask = a.n - 1;  // n is a power of two: % n is a mask
    uint32_t count = 0, batch = 0, take = 0;
    // get_distinct_queries in batches of squeezes; the round bound only
    // guards a state that cannot progress (n >= s always can)
    for (uint32_t round = 0; ok && count < a.s && round < 1024; ++round) {
        // the queries still needed, about twice the repeats expected among
        // them (need (need/2 + count) / n) plus 2 more, and the challenges
        // squeezed after them: the chain of full blocks a batch completes is
        // its serial part (~1.2 us a block), so the batch is kept tight; a
        // short batch just takes another round
        const uint32_t need = a.s - count;
        const uint64_t margin = ((uint64_t)need * (need + 2ull * count)) / a.n + 2;
        const uint64_t want = need + margin + a.nsq;
        batch = want < kQBlock ? (uint32_t)want : kQBlock;
        fs_chain_block(S, B, batch, kw);
        // A squeeze whose final data fills 14 or 15 words of its last block
        // needs a second compression for the padding; those squeezes go to
        // the first threads, so that only their warps run two compressions
        // (each warp of consecutive squeezes would otherwise hold some).
        {
            const bool two = tid < batch && ((S.nw + tid + 1) & 15) >= 14;
            uint32_t total2;
            const uint32_t r2 = block_rank(two, scratch, &total2);
            if (tid < batch) order[two ? r2 : total2 + (tid - r2)] = tid;
        }
        __syncthreads();
        if (tid < batch) {
            const uint32_t i = order[tid];
            sq[i] = fs_squeeze_at(S, B, i);
        }
        __syncthreads();
        uint64_t qv = 0;
        if (tid < batch) {
            const uint64_t lo = sq[tid];
            lo32[tid] = (uint32_t)lo;
            qv = lo & mask;
        }
        // Repeats: the queries taken so far (rank 0) and this batch's
        // squeezes (rank i + 1) go into a shared hash set that keeps each
        // value's smallest rank; a squeeze is new iff it holds its value's.
        for (uint32_t i = tid; i < kHash; i += blockDim.x) {
            hkey[i] = ~0ull;  // never a value: values are < n <= 2^63
            hrank[i] = ~0u;
        }
        __syncthreads();
        if (tid < count) hash_insert(hkey, hrank, acc[tid], 0);
        const uint32_t slot = tid < batch ? hash_insert(hkey, hrank, qv, tid + 1) : 0;
        __syncthreads();
        const bool dup = tid >= batch || hrank[slot] != tid + 1;
        uint32_t fresh;
        const uint32_t rank = block_rank(!dup, scratch, &fresh);
        if (!dup && rank < need) acc[count + rank] = qv;
        // squeezes consumed: the whole batch, or up to the one that
        // completes the set
        if (tid == 0) take_sh = batch;
        __syncthreads();
        if (fresh >= need && !dup && rank == need - 1) take_sh = tid + 1;
        __syncthreads();
        take = take_sh;
        count += min(fresh, need);
        // the challenges after the last query are the next squeezes of this
        // batch when it has them; commit past those too
        const uint32_t extra = count == a.s && take + a.nsq <= batch ? a.nsq : 0;
        if (tid < extra) a.out[tid] = lo32[take + tid];
        if (tid == 0) {
            fs_commit(S, B, take + extra);
            batch_sh = extra;
        }
        __syncthreads();
    }
    const uint32_t done_extra = ok && count == a.s ? batch_sh : 0;
    if (!ok || count < a.s) {
        if (tid == 0) {
            S.err |= FS_ERR_QUERIES;
            *a.nnodes = 0;
        }
        for (uint32_t i = tid; i < a.s && i < kQBlock; i += blockDim.x) a.q[i] = 0;
    } else {
        if (tid >= count) acc[tid] = ~0ull;
        __syncthreads();
        // bitonic sort of the kQBlock keys, one pair per thread per step
        for (uint32_t size = 2; size <= kQBlock; size <<= 1)
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                const uint32_t i = tid, j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const uint64_t x = acc[i], y = acc[j];
                    if ((x > y) == up) { acc[i] = y; acc[j] = x; }
                }
                __syncthreads();
            }
        if (tid < count) a.q[tid] = acc[tid];
        // Multi-proof siblings (merkle_tree::prove, src/merkle_tree.rs:62-111):
        // at layer d the present nodes are x = q >> d; the sibling x ^ 1 is
        // emitted, in order of x, unless it is present too.  Queries are
        // sorted, so the nodes equal to x form a run and x's sibling can only
        // be the run's neighbour: an odd x is settled at its run's first
        // query by the previous query, an even x at its run's last query by
        // the next one.  Thread i owns query i across all layers.
        const bool have = tid < count;
        const uint64_t qi = have ? acc[tid] : 0;
        const uint64_t qp = have && tid > 0 ? acc[tid - 1] : ~0ull;
        const uint64_t qn = have && tid + 1 < count ? acc[tid + 1] : ~0ull;
        const uint32_t lane = tid & 31, warp = tid >> 5;
        uint32_t nl = 0;
        while ((1ull << nl) < a.n) ++nl;
        auto emits = [&](uint32_t d, uint64_t &x) {
            x = qi >> d;
            if (!have) return false;
            const bool has_p = qp != ~0ull, has_n = qn != ~0ull;
            const uint64_t xp = qp >> d, xn = qn >> d;
            if (x & 1) return (!has_p || xp != x) && !(has_p && xp == (x ^ 1));
            return (!has_n || xn != x) && !(has_n && xn == (x ^ 1));
        };
        // Per-warp counts of every layer, then one scan gives each warp its
        // start in each layer (layers in order, threads in query order):
        // two barriers instead of two per layer.
        // (each layer's emit bit and warp mask are kept for the write pass)
        uint64_t x, emask = 0;
        for (uint32_t d = 0; d < nl; ++d) {
            const bool e = emits(d, x);
            emask |= (uint64_t)e << d;
            const uint32_t m = __ballot_sync(0xffffffffu, e);
            if (lane == 0) {
                wcnt[d][warp] = __popc(m);
                wmask[d][warp] = m;
            }
        }
        __syncthreads();
        if (warp == 0) {
            // lane l scans layers l and l + 32: in-layer warp offsets, then
            // a shuffle scan of the layer totals
            uint32_t tot[2] = {0, 0};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t d = lane + 32 * h;
                if (d < nl)
                    for (uint32_t w = 0; w < kQBlock / 32; ++w) {
                        const uint32_t c = wcnt[d][w];
                        wcnt[d][w] = tot[h];
                        tot[h] += c;
                    }
            }
            uint32_t inc[2] = {tot[0], tot[1]};
#pragma unroll
            for (int h = 0; h < 2; ++h)
                for (uint32_t o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, inc[h], o);
                    if (lane >= o) inc[h] += y;
                }
            const uint32_t all0 = __shfl_sync(0xffffffffu, inc[0], 31);
            const uint32_t start[2] = {inc[0] - tot[0], all0 + inc[1] - tot[1]};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t d = lane + 32 * h;
                if (d < nl)
                    for (uint32_t w = 0; w < kQBlock / 32; ++w) wcnt[d][w] += start[h];
            }
            if (lane == 31) take_sh = all0 + inc[1];
        }
        __syncthreads();
        uint64_t layer_off = 0, width = a.n;
        for (uint32_t d = 0; d < nl; ++d) {
            const bool e = (emask >> d) & 1;
            const uint32_t m = wmask[d][warp];
            const uint32_t pos = wcnt[d][warp] + __popc(m & ((1u << lane) - 1));
            if (e && pos < a.nodes_cap) a.nodes[pos] = layer_off + ((qi >> d) ^ 1);
            layer_off += width;
            width >>= 1;
        }
        const uint32_t nout = take_sh;
        if (tid == 0) {
            *a.nnodes = nout;
            if (nout > a.nodes_cap) S.err |= FS_ERR_QUERIES;
        }
    }
    __syncthreads();
    if (done_extra < a.nsq) fs_fields(S, B, a.nsq - done_extra, a.out + done_extra);
    store_state(S, g);
}

}  // namespace

cudaError_t fs_init(Launcher &L, FsState *d, uint32_t seed, uint32_t B) {
    if (B == 0 || B > 65535) return cudaErrorInvalidValue;
    LGK_LAUNCH(L, "fs_init", launch_k(k_fs_init, B, 32, 0, L.stream, d, seed));
    return cudaGetLastError();
}

cudaError_t fs_step(Launcher &L, FsState *d, const FsStep &a, uint32_t B, const FsStrides &st) {
    if (a.nwords > 1024 || (a.nwords && !a.src) || a.nsq > 256 || (a.nsq && !a.out) ||
        (a.check && (!a.src || a.nwords < 3)) || B == 0 || B > 65535)
        return cudaErrorInvalidValue;
    LGK_LAUNCH(L, "fs_step", launch_k(k_fs_step, B, 32, 0, L.stream, d, a, st));
    return cudaGetLastError();
}

cudaError_t fs_queries(Launcher &L, FsState *d, const FsQueries &a, uint32_t B, const FsStrides &st) {
    if (a.s == 0 || a.s > kQBlock || a.n == 0 || (a.n & (a.n - 1)) || a.nwords > 1024 || (a.nwords && !a.src) ||
        a.nsq > kQBlock || (a.nsq && !a.out) || !a.q || !a.nodes || !a.nnodes || B == 0 || B > 65535)
        return cudaErrorInvalidValue;
    LGK_LAUNCH(L, "fs_queries", launch_k(k_fs_queries, B, kQBlock, 0, L.stream, d, a, st));
    return cudaGetLastError();
}

}  // namespace lgk
