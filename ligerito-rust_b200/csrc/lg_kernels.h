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
struct Launcher {
    cudaStream_t stream = nullptr;
    uint64_t launches = 0;
    bool timing = false;
    struct Pending { std::string name; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> free_events;
    std::map<std::string, std::pair<uint64_t, double>> stats;  // name -> (launches, ms)

    cudaEvent_t get_event();
    void begin(const char *name, cudaEvent_t *a);
    void end(const char *name, cudaEvent_t a);
    void resolve();  // requires the stream to be idle
    void release();
};

// --- Reed-Solomon column encoding (src/reed_solomon.rs:104-113) ----------
// E (column-major, n columns of 4m): every quarter of column j receives
// poly[j*m + i] * pis[i]; the zero-padded 4m-point FFT's top two stages are
// copies, so quarter q then needs the m-point FFT under heap node 4+q.
cudaError_t rs_scale_spread(Launcher &L, const uint32_t *poly, const uint32_t *pis, uint32_t *E,
                            uint32_t log_m, uint32_t n);

// In-place additive FFT / IFFT (src/binary_fft.rs:109-206) of `nvec * Q`
// vectors of 2^log_len: vector (j, q) starts at data + j*col_stride +
// q*q_stride and uses the twiddle subtree under heap node root_base + q of
// `tw` (heap order, tw[idx-1]).
// passes: FFT_ALL, FFT_HEAD (every pass but the last), FFT_LAST (only the
// last; forward only) -- the head passes treat vectors independently, so a
// batch may run them in column groups and the last pass once for all.
enum FftPasses { FFT_ALL = 0, FFT_HEAD = 1, FFT_LAST = 2 };
cudaError_t fft_vectors(Launcher &L, uint32_t *data, const uint32_t *tw, uint32_t log_len,
                        uint32_t nvec, uint64_t col_stride, uint32_t Q, uint64_t q_stride,
                        uint32_t root_base, bool inverse, FftPasses passes = FFT_ALL);

// --- Merkle (src/merkle_tree.rs:4-60, leaves src/ligero.rs:53-68) --------
// Leaf hash of every row of a column-major matrix (rows x ncols u32).
cudaError_t leaf_hashes(Launcher &L, const uint32_t *E, uint64_t rows, uint32_t ncols, uint32_t *out);
// All upper layers from the leaf layer at tree[0]; tree as 8-word nodes.
cudaError_t merkle_upper(Launcher &L, uint32_t *tree, uint64_t num_leaves);

// --- gathers for openings (src/ligero.rs:40-51, src/merkle_tree.rs:98) ---
cudaError_t gather_rows(Launcher &L, const uint32_t *E, uint64_t rows, uint32_t ncols,
                        const uint64_t *d_queries, uint32_t nq, uint32_t *out);
cudaError_t gather_nodes(Launcher &L, const uint32_t *tree, const uint64_t *d_node_index,
                         uint32_t count, uint32_t *out);

// --- multilinear folds (src/multilinear_poly.rs:66-87) -------------------
// out[i] = sum_j gr[j] * in[j*M + i], M = 2^log_len >> k, 1 <= k <= 6.
cudaError_t fold_eq(Launcher &L, const uint32_t *in, uint32_t *out, uint32_t log_len, uint32_t k,
                    const uint32_t *gr);

// --- sumcheck rounds (src/ligerito.rs:50-127, multilinear_poly.rs:90) -----
// acc3 (device, 3 words) is XOR-accumulated; the caller zeroes it.
cudaError_t eval013(Launcher &L, const uint32_t *f, const uint32_t *g, uint32_t log_len,
                    uint32_t *acc3);
// f, B of 2^log_len folded by r into fo, Bo (2^(log_len-1)); triple of (fo, Bo)
cudaError_t fold_round(Launcher &L, const uint32_t *f, const uint32_t *B, uint32_t log_len,
                       uint32_t r, uint32_t *fo, uint32_t *Bo, uint32_t *acc3);
// B ^= beta * bi
cudaError_t axpy(Launcher &L, uint32_t *B, const uint32_t *bi, uint32_t log_len, uint32_t beta);

// --- induce_sumcheck_poly basis (src/sumcheck_polys.rs:74-160) ------------
// basis[t] = sum_k apow[k] * prod_{bit i of t} S[k*n + i]; S = per-query
// subspace values (sks_at_x).  out (2^n) must be zeroed when it returns
// needs_zero = true.
struct InducePlan { uint32_t b, qsplit; bool needs_zero; };
InducePlan induce_plan(uint32_t n, uint32_t nq);
cudaError_t induce_basis(Launcher &L, const InducePlan &p, const uint32_t *d_S, const uint32_t *d_apow,
                         uint32_t n, uint32_t nq, uint32_t *d_scratch_lo, uint32_t *d_scratch_hi,
                         uint32_t *out);

// Per-query inputs of induce_basis from device-resident opened rows
// (nq x glen): S (nq x n), apow (nq) and the enforced sum (1 word).
cudaError_t induce_setup(Launcher &L, const uint32_t *d_rows, uint32_t glen, const uint32_t *gr,
                         const uint64_t *d_q, uint32_t nq, uint32_t alpha, uint32_t n, const uint32_t *sks,
                         uint32_t *d_S, uint32_t *d_apow, uint32_t *d_sum);

cudaError_t splitmix(Launcher &L, uint64_t seed, uint32_t *out, uint64_t n);

}  // namespace lgk
