// Kernel launchers of liblgpu.  Each returns the launch's cudaError_t; all
// work goes to the Launcher's stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace lgk {

// Counts every kernel launch and, when timing is on, brackets each with a
// pair of CUDA events on the launching stream (resolved lazily).
// An FFT of up to 2^30 points runs in at most 6 passes of <= 6 stages; a
// pass has at most 63 node tables of 128 words.
constexpr uint32_t kMaxFftPasses = 6;
constexpr size_t kDtabWords = kMaxFftPasses * 63 * 128;
// D-table sets kept per context: one per FFT size a proof uses (its
// commitments), so a steady run of proofs builds none
constexpr uint32_t kDtabSlots = 4;

// A stage split of an FFT: np passes of ks[i] stages, the last one in tiles.
struct FftPlan {
    uint32_t np = 0;
    uint32_t ks[kMaxFftPasses] = {};
};
inline uint32_t plan_code(const FftPlan &p) {  // a compact key (3 bits a pass)
    uint32_t c = p.np;
    for (uint32_t i = 0; i < p.np && i < kMaxFftPasses; ++i) c = c * 8 + p.ks[i];
    return c;
}

struct Launcher {
    cudaStream_t stream = nullptr;
    int device = 0;
    // Autotuning (see tune_fft / tuned_fold_blocks): when set, the first call
    // of a shape times the candidates on scratch buffers and keeps the
    // fastest for the process; forced_plan overrides the split (tuning runs).
    bool autotune = false;
    const FftPlan *forced_plan = nullptr;
    int forced_fold_bps = 0;
    // device scratch of kDtabSlots x kDtabWords, owned by the context: sets
    // of the FFT passes' shared twiddle tables (fft_vectors), rebuilt in
    // stream order, each with the twiddle subtree it was built for and its
    // last use (the least recently used set is rebuilt first)
    uint32_t *dtab = nullptr;
    // device words, owned by the context and zero between launches: block
    // tickets of kernels whose last block to finish does the final step
    uint32_t *tickets = nullptr;
    struct DtabKey {
        const uint32_t *tw = nullptr;
        uint32_t log_len = 0, root_base = 0, plan = 0;
        bool operator==(const DtabKey &o) const {
            return tw == o.tw && log_len == o.log_len && root_base == o.root_base && plan == o.plan;
        }
    } dtab_key[kDtabSlots];
    uint64_t dtab_used[kDtabSlots] = {}, dtab_clock = 0;
    uint64_t launches = 0;
    bool timing = false;
    struct Pending { std::string name; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> free_events;
    std::map<std::string, std::pair<uint64_t, double>> stats;  // name -> (launches, ms)
    // Algorithmic work of the timed launches, by kernel name: compulsory HBM
    // bytes, GF(2^32) multiplications, BLAKE3 compressions.  A launcher
    // states the next launch's work with note(); end() books it.
    struct Work { double bytes = 0, mults = 0, comps = 0; };
    std::map<std::string, Work> work;
    Work next_work;
    void note(double bytes, double mults, double comps = 0) { next_work = {bytes, mults, comps}; }

    cudaEvent_t get_event();
    void begin(const char *name, cudaEvent_t *a);
    void end(const char *name, cudaEvent_t a);
    void resolve();  // requires the stream to be idle
    void release();
};

// Kernel launch with programmatic dependent launch: the kernel may begin
// launching while the previous kernel on the stream finishes; every kernel
// of this library starts with pdl_begin() (lg_device.cuh), which waits for
// the previous grid's completion before touching memory.  LG_PDL=0 in the
// environment turns it off.
bool pdl_enabled();
template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                     Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// A kernel launch on L's stream, counted and (when timing) bracketed.
#define LGK_LAUNCH(L, name, ...)   \
    do {                           \
        cudaEvent_t _ev = nullptr; \
        (L).begin(name, &_ev);     \
        __VA_ARGS__;               \
        (L).end(name, _ev);        \
    } while (0)

// --- autotuner -------------------------------------------------------------
// Choices measured on this device and kept for the process (all contexts):
// the FFT stage split per transform shape, and the fold grid.  Every choice
// computes the same values (the split only regroups the same butterflies),
// so tuning changes speed only.
struct TuneKey {
    int device;
    uint32_t log_len, nvec, Q;
    bool src, inverse;
    uint32_t kind;  // 0 FFT, 1 fold
    bool operator<(const TuneKey &o) const;
};
FftPlan default_fft_plan(uint32_t log_len);
bool tuned_fft_plan(const TuneKey &k, FftPlan *out);
cudaError_t tune_fft(Launcher &L, const TuneKey &k, uint32_t *data, const uint32_t *tw, uint64_t col_stride,
                     uint64_t q_stride, uint32_t root_base, const struct FftSrc *src, FftPlan *out);
// "log_len nvec Q src inv : k0 k1 ..." lines, and "fold log_len k : blocks/SM"
std::string tuned_choices();

// --- Reed-Solomon column encoding (src/reed_solomon.rs:104-113) ----------
// E (column-major, n columns of 4m): every quarter of column j receives
// poly[j*m + i] * pis[i]; the zero-padded 4m-point FFT's top two stages are
// copies, so quarter q then needs the m-point FFT under heap node 4+q.
cudaError_t rs_scale_spread(Launcher &L, const uint32_t *poly, const uint32_t *pis, uint32_t *E,
                            uint32_t log_m, uint32_t n);
// The same scaling without the spread: out[j*m + i] = poly[j*m + i] * pis[i]
// (n columns of m), for an FFT whose first pass reads all four quarters'
// input from it (FftSrc).
cudaError_t rs_scale(Launcher &L, const uint32_t *poly, const uint32_t *pis, uint32_t *out, uint32_t log_m,
                     uint32_t n);

// In-place additive FFT / IFFT (src/binary_fft.rs:109-206) of `nvec * Q`
// vectors of 2^log_len: vector (j, q) starts at data + j*col_stride +
// q*q_stride and uses the twiddle subtree under heap node root_base + q of
// `tw` (heap order, tw[idx-1]).
// The twiddle arrays must stay allocated and unchanged for the Launcher's
// lifetime (its cached pass tables are keyed by their address).
// passes: FFT_ALL, FFT_HEAD (every pass but the last), FFT_LAST (only the
// last; forward only) -- vectors are independent, so a caller may run the
// head passes on column groups as they arrive and the last pass on larger
// batches.
// src: where the first pass reads its input instead of data (vector (j, q)
// at src + j*col_stride + q*q_stride; q_stride 0 lets all Q subtrees start
// from one copy); the first pass must then be a strided pass (log_len > 6).
enum FftPasses { FFT_ALL = 0, FFT_HEAD = 1, FFT_LAST = 2 };
struct FftSrc {
    const uint32_t *p = nullptr;
    uint64_t col_stride = 0, q_stride = 0;
};
cudaError_t fft_vectors(Launcher &L, uint32_t *data, const uint32_t *tw, uint32_t log_len,
                        uint32_t nvec, uint64_t col_stride, uint32_t Q, uint64_t q_stride,
                        uint32_t root_base, bool inverse, FftPasses passes = FFT_ALL,
                        const FftSrc *src = nullptr);

// --- Merkle (src/merkle_tree.rs:4-60, leaves src/ligero.rs:53-68) --------
// Lockstep batches: several launchers take B proofs of one config at once,
// proof b in its own slice of each buffer (buffer + b * that buffer's
// stride, in elements), the proof index a grid dimension.  B = 1 with zero
// strides is a single proof.
constexpr uint32_t kMaxTickets = 64;  // Launcher::tickets words: the largest batch

// Leaf hash of every row of a column-major matrix (rows x ncols u32).
cudaError_t leaf_hashes(Launcher &L, const uint32_t *E, uint64_t rows, uint32_t ncols, uint32_t *out,
                        uint32_t B = 1, uint64_t e_stride = 0, uint64_t out_stride = 0);
// BLAKE3 blocks b0 .. b0+nb-1 (columns 16b .. 16b+15 each) of every leaf:
// chains from the value in out (the IV for b0 = 0) and leaves the chaining
// value there, the leaf hash after the last block.  Calls cover the blocks
// in order.
cudaError_t leaf_hash_block(Launcher &L, const uint32_t *E, uint64_t rows, uint32_t ncols, uint32_t b0,
                            uint32_t nb, uint32_t *out);
// All upper layers from the leaf layer at tree[0]; tree as 8-word nodes.
// Needs the Launcher's tickets.
cudaError_t merkle_upper(Launcher &L, uint32_t *tree, uint64_t num_leaves, uint32_t B = 1,
                         uint64_t tree_stride = 0);

// --- gathers for openings (src/ligero.rs:40-51, src/merkle_tree.rs:98) ---
// out = the nq opened rows (nq x ncols words), then count Merkle nodes (8
// words each; min(count, *d_count) of them when d_count is given)
struct GatherStrides { uint64_t E = 0, q = 0, tree = 0, nodes = 0, count = 0, out = 0; };
cudaError_t gather_opening(Launcher &L, const uint32_t *E, uint64_t rows, uint32_t ncols, const uint64_t *d_queries,
                           uint32_t nq, const uint32_t *tree, const uint64_t *d_node_index, uint32_t count,
                           const uint32_t *d_count, uint32_t *out, uint32_t B = 1,
                           const GatherStrides &st = GatherStrides{});

// --- multilinear folds (src/multilinear_poly.rs:66-87) -------------------
// partial_eval of the top k variables (1 <= k <= 6): out (M = 2^log_len >> k
// words) = sum_j eq(rs, j) * in[j*M + i], rs[0] for j's top bit; the k
// challenges on the host (rs) or the device (d_rs).
struct FoldStrides { uint64_t in = 0, out = 0, rs = 0; };
cudaError_t fold_eq(Launcher &L, const uint32_t *in, uint32_t *out, uint32_t log_len, uint32_t k,
                    const uint32_t *rs, const uint32_t *d_rs = nullptr, uint32_t B = 1,
                    const FoldStrides &st = FoldStrides{});

struct FsTail;  // a fused transcript step, below
// per-proof strides of the sumcheck kernels' buffers: f / g (the basis, or
// B and bi for axpy), the folded outputs fo / go, the triple acc, the
// challenge r (d_r / d_beta), and the fused transcript step's state (in
// states), ticket and output words
struct RoundStrides { uint64_t f = 0, g = 0, fo = 0, go = 0, acc = 0, r = 0, fs = 0, ticket = 0, out = 0; };

// --- sumcheck rounds (src/ligerito.rs:50-127, multilinear_poly.rs:90) -----
// acc3 (device, 3 words) is XOR-accumulated; the caller zeroes it.
cudaError_t eval013(Launcher &L, const uint32_t *f, const uint32_t *g, uint32_t log_len,
                    uint32_t *acc3, const FsTail *tail = nullptr, uint32_t B = 1,
                    const RoundStrides &st = RoundStrides{});
// f, B of 2^log_len folded by r (or *d_r) into fo, Bo (2^(log_len-1));
// triple of (fo, Bo)
cudaError_t fold_round(Launcher &L, const uint32_t *f, const uint32_t *B, uint32_t log_len,
                       uint32_t r, uint32_t *fo, uint32_t *Bo, uint32_t *acc3, const uint32_t *d_r = nullptr,
                       const FsTail *tail = nullptr, uint32_t NB = 1, const RoundStrides &st = RoundStrides{});
// B ^= beta * bi (beta or *d_beta)
cudaError_t axpy(Launcher &L, uint32_t *B, const uint32_t *bi, uint32_t log_len, uint32_t beta,
                 const uint32_t *d_beta = nullptr, uint32_t NB = 1, const RoundStrides &st = RoundStrides{});

// --- induce_sumcheck_poly basis (src/sumcheck_polys.rs:74-160) ------------
// basis[t] = sum_k apow[k] * prod_{bit i of t} S[k*n + i]; S = per-query
// subspace values (sks_at_x).  induce_basis writes all of out (2^n words);
// a plan with needs_zero set (none currently) wants out zeroed first.
// The enforced sum (the sum of the setup's per-query contributions) lands
// in d_sum (1 word).
struct InducePlan { uint32_t b; bool needs_zero; };  // b: low bits of t in Lo
// per-proof strides: opened rows, queries, subspace values, alpha powers
// (2 nq words), Lo / Hi vectors, basis out, enforced sum, challenges, alpha
struct InduceStrides {
    uint64_t rows = 0, q = 0, S = 0, apow = 0, lo = 0, hi = 0, out = 0, sum = 0, rs = 0, alpha = 0;
};
InducePlan induce_plan(uint32_t n, uint32_t nq);
cudaError_t induce_basis(Launcher &L, const InducePlan &p, const uint32_t *d_S, const uint32_t *d_apow,
                         uint32_t n, uint32_t nq, uint32_t *d_scratch_lo, uint32_t *d_scratch_hi,
                         uint32_t *out, uint32_t *d_sum, uint32_t B = 1, const InduceStrides &st = InduceStrides{});

// Per-query inputs of induce_basis from device-resident opened rows
// (nq x glen, nq <= 2^16): S (nq x n) and, in apow (2 nq words), the alpha
// powers and each query's contribution to the enforced sum.  gr and alpha
// from the host, or the Lagrange basis of log2(glen) device challenges
// d_rs and *d_alpha.
cudaError_t induce_setup(Launcher &L, const uint32_t *d_rows, uint32_t glen, const uint32_t *gr,
                         const uint64_t *d_q, uint32_t nq, uint32_t alpha, uint32_t n, const uint32_t *sks,
                         uint32_t *d_S, uint32_t *d_apow, const uint32_t *d_rs = nullptr,
                         const uint32_t *d_alpha = nullptr, uint32_t B = 1,
                         const InduceStrides &st = InduceStrides{});
// induce_setup and induce_basis with the setup and the prep in one launch
// (its last block sums the enforced sum; needs the Launcher's tickets, and
// otherwise runs the two calls).  d_S is used only by that fallback.
cudaError_t induce_fused(Launcher &L, const InducePlan &p, const uint32_t *d_rows, uint32_t glen, const uint32_t *gr,
                         const uint64_t *d_q, uint32_t nq, uint32_t alpha, uint32_t n, const uint32_t *sks,
                         uint32_t *d_S, uint32_t *d_apow, const uint32_t *d_rs, const uint32_t *d_alpha,
                         uint32_t *d_lo, uint32_t *d_hi, uint32_t *out, uint32_t *d_sum, uint32_t B = 1,
                         const InduceStrides &st = InduceStrides{});

cudaError_t splitmix(Launcher &L, uint64_t seed, uint32_t *out, uint64_t n);

// --- merkle_tree::verify of one opening (src/merkle_tree.rs:120-188) ------
// Well-formed inputs only (the caller checks): nq <= 256 sorted distinct
// queries, their rows (nq x ncols words, 1 <= ncols <= 256) and the 32-byte
// proof nodes the opening consumes (8 words each, in order).  out (9 words)
// = the last layer's first hash and the last layer's size.
cudaError_t opening_check(Launcher &L, const uint32_t *rows, uint32_t ncols, const uint64_t *q, uint32_t nq,
                          const uint32_t *proof, uint32_t depth, uint32_t *out);

// --- ligero_verify (src/ligero.rs:97-131) ----------------------------------
// Rows k < nrows at rows[row_off[k] .. row_off[k+1]), the Lagrange basis gr
// of the challenges (glen words), yr (2^nv words), the queries q and
// eval_sk_at_vks's first nv - 1 values; *bad (zeroed by the caller) becomes
// nonzero if any row's check fails.
struct ligero_sks { uint32_t v[32]; };
cudaError_t ligero_check(Launcher &L, const uint32_t *rows, const uint64_t *row_off, uint32_t nrows,
                         const uint32_t *gr, uint32_t glen, const uint32_t *yr, uint32_t nv, const uint64_t *q,
                         const uint32_t *sks, uint32_t *bad);

// --- BinaryElem128 (src/binary_field.rs:182-189) --------------------------
// out[i] = a[i] * b[i], n elements of two u64 limbs (low first), 16-byte
// aligned device arrays.
cudaError_t gf128_mul(Launcher &L, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t n);

// --- Fiat-Shamir transcript on the device (src/emulated_fs.rs:6-76) ------
// The running SHA-256 of the transcript: the host's lg::Transcript with the
// pending bytes kept as big-endian words (the transcript only ever absorbs
// whole u32s and 32-byte roots, so they stay word-aligned).
struct FsState {
    uint32_t h[8];
    uint32_t w[16];    // pending message words
    uint64_t total;    // bytes absorbed
    uint32_t nw;       // words pending in w
    uint32_t counter;  // squeezes so far
    uint32_t err;      // FS_ERR_* bits: a prover assertion failed
    uint32_t pad;
};
enum : uint32_t { FS_ERR_SUMCHECK = 1, FS_ERR_QUERIES = 2 };

// A transcript step fused into a sumcheck kernel (eval013, fold_round): its
// last block to finish absorbs the kernel's triple -- asserting first, when
// check is set, that triple[0] ^ triple[1] == triple[3] (the enforced sum)
// -- and squeezes nsq field elements into out.  ticket: a zeroed word the
// kernel counts finished blocks in (left zero again).
struct FsTail {
    FsState *fs = nullptr;
    uint32_t *ticket = nullptr;
    uint32_t check = 0;
    uint32_t nsq = 0;
    uint32_t *out = nullptr;
};

// Lockstep batches: B transcripts d[0..B), one block each; per-proof
// strides of the step / query arguments' buffers (in their elements).
struct FsStrides { uint64_t src = 0, out = 0, mirror = 0, q = 0, nodes = 0, nnodes = 0; };

// FS::new(seed)
cudaError_t fs_init(Launcher &L, FsState *d, uint32_t seed, uint32_t B = 1);
// If check: flag FS_ERR_SUMCHECK unless src[0] ^ src[1] == src[3] (a
// sumcheck triple and its enforced sum).  Then absorb nwords u32s of src
// (their LE bytes) and squeeze nsq field elements into out.
struct FsStep {
    const uint32_t *src = nullptr;
    uint32_t nwords = 0, check = 0;
    uint32_t nsq = 0;
    uint32_t *out = nullptr;
    uint32_t *mirror = nullptr;  // when set, also receives the absorbed words
};
cudaError_t fs_step(Launcher &L, FsState *d, const FsStep &a, uint32_t B = 1, const FsStrides &st = FsStrides{});
// Absorb nwords u32s of src; get_distinct_queries(n, s) sorted into q
// (s <= 256, n a power of two); the multi-proof siblings of those leaves
// in a tree of n leaves (merkle_tree::prove order) into nodes as node
// numbers, leaves first, count in *nnodes; then squeeze nsq field elements
// into out.  n < s flags FS_ERR_QUERIES (the reference loops forever).
struct FsQueries {
    const uint32_t *src = nullptr;
    uint32_t nwords = 0;
    uint64_t n = 0;
    uint32_t s = 0;
    uint64_t *q = nullptr;
    uint64_t *nodes = nullptr;
    uint32_t nodes_cap = 0;
    uint32_t *nnodes = nullptr;
    uint32_t nsq = 0;
    uint32_t *out = nullptr;
    uint32_t *mirror = nullptr;  // when set, also receives the absorbed words
};
cudaError_t fs_queries(Launcher &L, FsState *d, const FsQueries &a, uint32_t B = 1,
                       const FsStrides &st = FsStrides{});

}  // namespace lgk
