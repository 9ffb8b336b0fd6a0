// C ABI of liblgpu: context, device memory, the prover and verifier
// protocols (src/prover.rs, src/verifier.rs) driving the kernels of
// lg_kernels.cu, and the kernel-level entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ligerito_b200.h"
#include "lg_host.h"
#include "lg_kernels.h"

using lg::NodeRef;

struct lg_proof {
    lg::Proof p;
};

namespace {

struct Code {  // ReedSolomonEncoding::new(m, 4m) tables, src/reed_solomon.rs:49-64
    uint32_t *tw = nullptr;   // compute_twiddles(log m + 2): 4m - 1 words
    uint32_t *pis = nullptr;  // compute_pis(m, eval_sk_at_vks(m)): m words
};

// The code and twiddle tables depend only on the size, so every context on
// a device shares one copy (a server's workers would otherwise each build
// and hold their own).  They live while a context on the device does.
struct DeviceTables {
    int contexts = 0;
    uint64_t bytes = 0;
    std::map<uint32_t, Code> codes;        // by log_m
    std::map<uint32_t, uint32_t *> ffttw;  // by log_n, plain fft twiddles
};
std::mutex g_tables_mu;
std::map<int, DeviceTables> g_tables;

}  // namespace

struct lg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // host->device input copies overlapped with compute
    cudaEvent_t copy_ev[8] = {};
    lgk::Launcher L;
    uint64_t budget = 0, in_use = 0;
    std::string err;
    uint8_t *pinned = nullptr;  // staging for small synchronous transfers
    size_t pinned_cap = 0;
    // per-call bump arenas (reset at the start of each prove / verify)
    uint8_t *pin_arena = nullptr;
    size_t pin_cap = 0, pin_used = 0, pin_want = 0;  // pin_want: the arena a call wanted
    uint8_t *dev_arena = nullptr;
    size_t dev_cap = 0, dev_used = 0;
    // set only while lg_dump_intermediates runs
    lg_dump_cb dump_cb = nullptr;
    void *dump_user = nullptr;
};

namespace {

struct CudaFail {
    cudaError_t e;
};

void fail_if(lg_ctx *c, cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        c->err = std::string(what) + ": " + cudaGetErrorString(e);
        throw CudaFail{e};
    }
}
#define CK(c, expr) fail_if((c), (expr), #expr)

struct OutOfBudget {};
struct ProverAssert {};
struct VerifyPanic {};
struct BadConfig {};

// Stream-ordered device allocation from the device's pool, counted against
// the context's HBM budget.
struct DBuf {
    lg_ctx *c = nullptr;
    void *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(lg_ctx *ctx, size_t bytes) : c(ctx), n(bytes) {
        if (c->budget && c->in_use + bytes > c->budget) {
            c->err = "HBM budget exceeded";
            throw OutOfBudget{};
        }
        cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(bytes, 16), c->stream);
        if (e != cudaSuccess) {
            c->err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
            throw OutOfBudget{};
        }
        c->in_use += bytes;
    }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : c(o.c), p(o.p), n(o.n) { o.p = nullptr; }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) { reset(); c = o.c; p = o.p; n = o.n; o.p = nullptr; }
        return *this;
    }
    void reset() {
        if (p) { cudaFreeAsync(p, c->stream); c->in_use -= n; p = nullptr; }
    }
    ~DBuf() { reset(); }
    uint32_t *u32() const { return static_cast<uint32_t *>(p); }
};

uint8_t *pinned(lg_ctx *c, size_t bytes) {
    if (bytes > c->pinned_cap) {
        if (c->pinned) cudaFreeHost(c->pinned);
        c->pinned = nullptr;
        size_t cap = std::max<size_t>(bytes, 1 << 20);
        CK(c, cudaMallocHost((void **)&c->pinned, cap));
        c->pinned_cap = cap;
    }
    return c->pinned;
}

void sync(lg_ctx *c) { CK(c, cudaStreamSynchronize(c->stream)); }

// lg_dump_intermediates: hand the caller a host copy of `bytes` device
// bytes once the stream has produced them; nothing happens otherwise.
void dump_dev(lg_ctx *c, const char *name, uint32_t level, const void *d, size_t bytes) {
    if (!c->dump_cb) return;
    std::vector<uint8_t> h(bytes);
    sync(c);
    CK(c, cudaMemcpy(h.data(), d, bytes, cudaMemcpyDeviceToHost));
    c->dump_cb(c->dump_user, name, level, h.data(), bytes);
}
void dump_host(lg_ctx *c, const char *name, uint32_t level, const void *h, size_t bytes) {
    if (c->dump_cb) c->dump_cb(c->dump_user, name, level, h, bytes);
}

void d2h(lg_ctx *c, void *dst, const void *src, size_t bytes) {
    uint8_t *p = pinned(c, bytes);
    CK(c, cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    sync(c);
    std::memcpy(dst, p, bytes);
}

// The device's shared tables (created on first use, under the lock; the
// upload is synchronous, so a table is complete before any context sees it).
Code get_code(lg_ctx *c, uint32_t log_m) {
    std::lock_guard<std::mutex> lk(g_tables_mu);
    DeviceTables &t = g_tables[c->device];
    auto it = t.codes.find(log_m);
    if (it != t.codes.end()) return it->second;
    const uint64_t m = 1ull << log_m;
    std::vector<uint32_t> tw((4 * m) - 1), pis(m);
    lg::compute_twiddles(log_m + 2, tw.data());
    lg::compute_pis(m, lg::eval_sk_at_vks(m), pis.data());
    Code code;
    CK(c, cudaMalloc(&code.tw, tw.size() * 4));
    if (cudaMalloc(&code.pis, pis.size() * 4) != cudaSuccess) {
        cudaFree(code.tw);
        CK(c, cudaErrorMemoryAllocation);
    }
    cudaError_t e = cudaMemcpy(code.tw, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(code.pis, pis.data(), pis.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(code.tw);
        cudaFree(code.pis);
        CK(c, e);
    }
    t.bytes += (tw.size() + pis.size()) * 4;
    return t.codes[log_m] = code;
}

const uint32_t *get_fft_tw(lg_ctx *c, uint32_t log_n) {
    std::lock_guard<std::mutex> lk(g_tables_mu);
    DeviceTables &t = g_tables[c->device];
    auto it = t.ffttw.find(log_n);
    if (it != t.ffttw.end()) return it->second;
    std::vector<uint32_t> tw((1ull << log_n) - 1);
    lg::compute_twiddles(log_n, tw.data());
    uint32_t *d = nullptr;
    CK(c, cudaMalloc(&d, tw.size() * 4));
    cudaError_t e = cudaMemcpy(d, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        CK(c, e);
    }
    t.bytes += tw.size() * 4;
    return t.ffttw[log_n] = d;
}

// ------------------------------------------------------------- scratch
// Per-call scratch: small device buffers come from a bump arena, uploads
// and downloads go through a pinned bump arena without synchronising (a
// call that outgrows it gets extra pinned blocks, valid until the call
// ends, and the next call starts with an arena that size), and
// host-side results of downloads (openings) are materialised by finalizers
// after the call's last synchronisation.  Deferred downloads (of arena
// buffers, which live until the call ends) are only queued by flush(), so
// that the kernels between them run back to back and the copies go out
// while the host has other work.
struct Scratch {
    lg_ctx *c;
    std::vector<DBuf> dev_overflow;
    std::vector<uint8_t *> pin_overflow;
    std::vector<std::function<void()>> finalizers;
    struct Deferred { uint8_t *h; const void *d; size_t bytes; };
    std::vector<Deferred> deferred;
    static constexpr size_t kPin = 8u << 20, kDevArena = 32u << 20;
    explicit Scratch(lg_ctx *ctx) : c(ctx) {
        constexpr size_t kDev = kDevArena;
        if (c->pin_arena && c->pin_want > c->pin_cap) {  // the last call outgrew it; nothing is in flight
            cudaFreeHost(c->pin_arena);
            c->pin_arena = nullptr;
        }
        if (!c->pin_arena) {
            const size_t cap = std::max(kPin, (c->pin_want + (1u << 20) - 1) & ~size_t((1u << 20) - 1));
            CK(c, cudaMallocHost((void **)&c->pin_arena, cap));
            c->pin_cap = cap;
        }
        if (!c->dev_arena) {
            CK(c, cudaMalloc((void **)&c->dev_arena, kDev));
            c->dev_cap = kDev;
        }
        c->pin_used = 0;
        c->dev_used = 0;
    }
    void flush() {
        for (auto &x : deferred) CK(c, cudaMemcpyAsync(x.h, x.d, x.bytes, cudaMemcpyDeviceToHost, c->stream));
        deferred.clear();
    }
    // all pending transfers done, then hand the host copies over
    void finish() {
        flush();
        sync(c);
        for (auto &f : finalizers) f();
        finalizers.clear();
    }
    // Pinned host bytes valid until the call ends (earlier ones stay valid:
    // the arena is never reused or moved within a call).
    uint8_t *pin(size_t bytes) {
        bytes = (bytes + 63) & ~size_t(63);
        c->pin_want = std::max(c->pin_want, c->pin_used + bytes);
        if (c->pin_used + bytes > c->pin_cap) {
            uint8_t *p = nullptr;
            CK(c, cudaMallocHost((void **)&p, bytes));
            pin_overflow.push_back(p);
            c->pin_used += bytes;  // counted, so the next call's arena covers it
            return p;
        }
        uint8_t *p = c->pin_arena + c->pin_used;
        c->pin_used += bytes;
        return p;
    }
    ~Scratch() {
        if (pin_overflow.empty()) return;
        // copies into the extra blocks may still be in flight after an error
        cudaStreamSynchronize(c->stream);
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        for (uint8_t *p : pin_overflow) cudaFreeHost(p);
    }
    void *dev(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        if (c->dev_used + bytes <= c->dev_cap) {
            void *p = c->dev_arena + c->dev_used;
            c->dev_used += bytes;
            return p;
        }
        dev_overflow.emplace_back(c, bytes);
        return dev_overflow.back().p;
    }
    template <class T>
    T *upload(const T *src, size_t count) {  // async through pinned memory
        const size_t bytes = count * sizeof(T);
        uint8_t *h = pin(bytes);
        std::memcpy(h, src, bytes);
        T *d = static_cast<T *>(dev(bytes));
        CK(c, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream));
        return d;
    }
    template <class T>
    const T *download_later(const T *d, size_t count) {  // valid after finish()
        const size_t bytes = count * sizeof(T);
        uint8_t *h = pin(bytes);
        CK(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream));
        return reinterpret_cast<const T *>(h);
    }
    template <class T>
    const T *download_deferred(const T *d, size_t count) {  // valid after finish()
        const size_t bytes = count * sizeof(T);
        uint8_t *h = pin(bytes);
        deferred.push_back({h, d, bytes});
        return reinterpret_cast<const T *>(h);
    }
};

// ------------------------------------------------------------ commitment
struct Witness {  // RecursiveLigeroWitness, src/data_structures.rs:32-40
    DBuf E;       // column-major encoded matrix, cols x rows
    DBuf tree;    // all layers, leaves first, 8 words per node
    uint64_t rows = 0;
    uint32_t cols = 0;
    const uint32_t *root() const { return tree.u32() + 8 * (2 * rows - 2); }  // on the device
};

// encode_non_systematic (src/reed_solomon.rs:104-113) of n columns into E
// (column-major, 4m rows): the columns scaled by pis are written once to
// `scaled` (n columns of m words) and the first FFT pass of all four
// quarters reads them from there, instead of spreading four copies through
// HBM; codes short enough for a single FFT pass spread them.
void rs_encode(lg_ctx *c, const Code &code, const uint32_t *d_poly, uint32_t log_m, uint32_t n, uint32_t *E,
               uint64_t col_stride, uint32_t *scaled, lgk::FftPasses passes = lgk::FFT_ALL) {
    const uint64_t m = 1ull << log_m;
    if (log_m > 6) {
        CK(c, lgk::rs_scale(c->L, d_poly, code.pis, scaled, log_m, n));
        lgk::FftSrc src;
        src.p = scaled;
        src.col_stride = m;
        src.q_stride = 0;
        CK(c, lgk::fft_vectors(c->L, E, code.tw, log_m, n, col_stride, 4, m, 4, false, passes, &src));
    } else {
        CK(c, lgk::rs_scale_spread(c->L, d_poly, code.pis, E, log_m, n));
        CK(c, lgk::fft_vectors(c->L, E, code.tw, log_m, n, col_stride, 4, m, 4, false, passes));
    }
}

// ligero_commit (src/ligero.rs:70-95) into caller buffers
void commit_into(lg_ctx *c, const uint32_t *d_poly, uint32_t log_m, uint32_t n, uint32_t *E, uint32_t *tree) {
    const Code code = get_code(c, log_m);
    const uint64_t m = 1ull << log_m, rows = 4 * m;
    {
        DBuf scaled(c, log_m > 6 ? 4ull * n * m : 0);
        rs_encode(c, code, d_poly, log_m, n, E, rows, scaled.u32());
    }
    CK(c, lgk::leaf_hashes(c->L, E, rows, n, tree));
    CK(c, lgk::merkle_upper(c->L, tree, rows));
}

Witness commit(lg_ctx *c, const uint32_t *d_poly, uint32_t log_m, uint32_t n) {
    Witness w;
    w.rows = 4ull << log_m;
    w.cols = n;
    w.E = DBuf(c, w.rows * n * 4);
    w.tree = DBuf(c, (2 * w.rows - 1) * 32);
    commit_into(c, d_poly, log_m, n, w.E.u32(), w.tree.u32());
    return w;
}

// Hash units of the host-input commitment: 32 columns (two BLAKE3 blocks of
// every leaf) when there are at least 64, else 16 (one block).  The last
// FFT pass runs once per unit, and its table work per tile does not shrink
// with the columns, so a 16-column unit costs about as much GPU time per
// column as its copy takes and the compute falls behind the copy; 32
// keeps it ahead.
uint32_t host_hash_unit(uint32_t n) { return n >= 64 ? 32 : std::min<uint32_t>(16, n); }

// Copy groups of the host-input commitment (column counts, in order): the
// first unit arrives as 1/8, 1/8, 1/4, 1/2 of it (a 16-column unit as 1/4,
// 1/4, 1/2) so that compute starts after a few columns, the last as 1/2,
// 1/4, 1/4 (a 16-column unit as two halves) so that little work remains
// after the last bytes land, the units between whole.
std::vector<uint32_t> host_copy_groups(uint32_t n) {
    const uint32_t U = host_hash_unit(n), units = (n + U - 1) / U;
    std::vector<uint32_t> g;
    for (uint32_t u = 0; u < units; ++u) {
        const uint32_t cols = std::min(U, n - u * U);
        if (u == 0 && cols == 32) {
            g.insert(g.end(), {4, 4, 8, 16});
        } else if (u == 0 && cols >= 8 && cols % 4 == 0) {
            g.insert(g.end(), {cols / 4, cols / 4, cols / 2});
        } else if (u + 1 == units && cols == 32) {
            g.insert(g.end(), {16, 8, 8});
        } else if (u + 1 == units && cols >= 8 && cols % 2 == 0) {
            g.insert(g.end(), {cols / 2, cols / 2});
        } else {
            g.push_back(cols);
        }
    }
    return g;
}

// The first commitment of a proof whose polynomial is on the host: the
// columns travel in groups (host_copy_groups) on the copy stream; the
// compute stream waits for each group and, while the next is in flight,
// runs its scale-and-spread and the FFT passes but the last (columns are
// independent).  Each hash unit (host_hash_unit), once all its groups are
// in, gets the last FFT pass and its BLAKE3 blocks of every leaf: a leaf is
// the row's words in column order and 16 words are one BLAKE3 block, so
// columns 16b .. 16b+15 are block b of each leaf's chunk, chained through
// the leaf slots of the tree.  After the last unit only the upper tree
// remains.
Witness commit_from_host(lg_ctx *c, Scratch &sc, const uint32_t *h_poly, uint32_t *d_poly, uint32_t log_m,
                         uint32_t n) {
    const Code code = get_code(c, log_m);
    const uint64_t m = 1ull << log_m, rows = 4 * m;
    Witness w;
    w.rows = rows;
    w.cols = n;
    w.E = DBuf(c, rows * n * 4);
    w.tree = DBuf(c, (2 * rows - 1) * 32);
    cudaPointerAttributes attr{};
    const bool pinned_src = cudaPointerGetAttributes(&attr, h_poly) == cudaSuccess && attr.type == cudaMemoryTypeHost;
    cudaGetLastError();
    const std::vector<uint32_t> groups = host_copy_groups(n);
    const uint32_t U = host_hash_unit(n);
    DBuf scaled(c, log_m > 6 ? 4ull * n * m : 0);
    // staging for pageable input: two pinned chunks, reused after their copy
    constexpr size_t kChunk = 4u << 20;
    uint8_t *slot[2] = {nullptr, nullptr};
    bool slot_busy[2] = {false, false};
    int next_slot = 0;
    if (!pinned_src) { slot[0] = sc.pin(kChunk); slot[1] = sc.pin(kChunk); }
    // the copy stream must not start before work already queued on the
    // compute stream that may still read d_poly's memory
    CK(c, cudaEventRecord(c->copy_ev[7], c->stream));
    CK(c, cudaStreamWaitEvent(c->copy_stream, c->copy_ev[7], 0));
    uint32_t j0 = 0;
    for (size_t g = 0; g < groups.size(); ++g) {
        const uint32_t cols = groups[g];
        const uint8_t *src = reinterpret_cast<const uint8_t *>(h_poly + (uint64_t)j0 * m);
        uint8_t *dst = reinterpret_cast<uint8_t *>(d_poly + (uint64_t)j0 * m);
        const size_t bytes = (size_t)cols * m * 4;
        if (pinned_src) {
            CK(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->copy_stream));
        } else {
            for (size_t off = 0; off < bytes; off += kChunk) {
                const size_t nb = std::min(kChunk, bytes - off);
                const int k = next_slot;
                next_slot ^= 1;
                if (slot_busy[k]) CK(c, cudaEventSynchronize(c->copy_ev[4 + k]));
                std::memcpy(slot[k], src + off, nb);
                CK(c, cudaMemcpyAsync(dst + off, slot[k], nb, cudaMemcpyHostToDevice, c->copy_stream));
                CK(c, cudaEventRecord(c->copy_ev[4 + k], c->copy_stream));
                slot_busy[k] = true;
            }
        }
        CK(c, cudaEventRecord(c->copy_ev[g % 4], c->copy_stream));
        CK(c, cudaStreamWaitEvent(c->stream, c->copy_ev[g % 4], 0));
        uint32_t *Eg = w.E.u32() + (uint64_t)j0 * rows;
        rs_encode(c, code, d_poly + (uint64_t)j0 * m, log_m, cols, Eg, rows, scaled.u32() + (uint64_t)j0 * m,
                  lgk::FFT_HEAD);
        j0 += cols;
        if (j0 % U == 0 || j0 == n) {  // a hash unit is complete
            const uint32_t u = (j0 - 1) / U, ju = u * U, ucols = j0 - ju;
            CK(c, lgk::fft_vectors(c->L, w.E.u32() + (uint64_t)ju * rows, code.tw, log_m, ucols, rows, 4, m, 4, false,
                                   lgk::FFT_LAST));
            // the unit's BLAKE3 blocks of every leaf, chained after the earlier units'
            const uint32_t b0 = ju / 16, nb = (ucols + 15) / 16;
            CK(c, lgk::leaf_hash_block(c->L, w.E.u32(), rows, n, b0, nb, w.tree.u32()));
        }
    }
    CK(c, lgk::merkle_upper(c->L, w.tree.u32(), rows));
    return w;
}

// The same opening from host copies of the matrix (column-major, rows x
// cols) and of the tree (all layers, leaves first, 32 bytes per node).
void open_rows_host(const uint32_t *E, const uint8_t *tree, uint64_t rows, uint32_t cols,
                    const std::vector<uint64_t> &q, lg::Opening *out) {
    out->rows.data.resize(q.size() * cols);
    for (size_t k = 0; k < q.size(); ++k)
        for (uint32_t j = 0; j < cols; ++j) out->rows.data[k * cols + j] = E[(uint64_t)j * rows + q[k]];
    out->rows.off.resize(q.size() + 1);
    for (size_t k = 0; k <= q.size(); ++k) out->rows.off[k] = k * cols;
    std::vector<NodeRef> refs;
    lg::merkle_proof_nodes(q, rows, refs);
    uint64_t layer_off[64] = {0};
    for (uint32_t l = 1; l < 64; ++l) layer_off[l] = layer_off[l - 1] + (rows >> (l - 1));
    out->merkle.data.resize(32 * refs.size());
    for (size_t i = 0; i < refs.size(); ++i)
        std::memcpy(out->merkle.data.data() + 32 * i, tree + 32 * (layer_off[refs[i].layer] + refs[i].index), 32);
    out->merkle.off.resize(refs.size() + 1);
    for (size_t i = 0; i <= refs.size(); ++i) out->merkle.off[i] = 32 * i;
}

// extract_row for each query (src/ligero.rs:40-51) + merkle_tree::prove
// (src/merkle_tree.rs:98-111): device gathers, host copies materialised
// into `out` at sc.finish().  Returns the device copy of the opened rows
// (nq x cols) and of the queries.
std::pair<const uint32_t *, const uint64_t *> open_rows(lg_ctx *c, Scratch &sc, const Witness &w,
                                                        const std::vector<uint64_t> &q, lg::Opening *out) {
    std::vector<NodeRef> refs;
    lg::merkle_proof_nodes(q, w.rows, refs);
    const size_t nq = q.size(), nr = refs.size();
    std::vector<uint64_t> idx(nq + nr);
    std::copy(q.begin(), q.end(), idx.begin());
    uint64_t layer_off[64] = {0};
    for (uint32_t l = 1; l < 64; ++l) layer_off[l] = layer_off[l - 1] + (w.rows >> (l - 1));
    for (size_t i = 0; i < nr; ++i) idx[nq + i] = layer_off[refs[i].layer] + refs[i].index;
    const uint64_t *d_idx = sc.upload(idx.data(), idx.size());
    uint32_t *d_out = static_cast<uint32_t *>(sc.dev((nq * w.cols + nr * 8) * 4 + 16));
    CK(c, lgk::gather_opening(c->L, w.E.u32(), w.rows, w.cols, d_idx, (uint32_t)nq, w.tree.u32(), d_idx + nq,
                              (uint32_t)nr, nullptr, d_out));
    const uint32_t *h = sc.download_later(d_out, nq * w.cols + nr * 8);
    const uint32_t cols = w.cols;
    sc.finalizers.push_back([h, nq, nr, cols, out]() {
        out->rows.assign_fixed(h, nq, cols);
        out->merkle.assign_fixed(reinterpret_cast<const uint8_t *>(h + nq * cols), nr, 32);
    });
    return {d_out, d_idx};
}

// The same opening with the queries drawn by the device transcript:
// fs_queries absorbs `absorb` (a root, 32 bytes), draws the distinct sorted
// queries on w's rows and their multi-proof node list, then squeezes
// `nsq` challenges into out.  Returns the device copy of the opened rows
// and of the queries.
std::pair<const uint32_t *, const uint64_t *> open_rows_dev(lg_ctx *c, Scratch &sc, const Witness &w,
                                                            lgk::FsState *fs, const uint32_t *absorb, uint32_t nsq,
                                                            uint32_t *out, lg::Opening *op,
                                                            uint32_t *absorb_mirror = nullptr) {
    const uint32_t nq = LG_NUM_QUERIES;
    uint32_t depth = 0;
    while ((1ull << depth) < w.rows) ++depth;
    const uint32_t cap = nq * std::max<uint32_t>(depth, 1);
    uint64_t *d_q = static_cast<uint64_t *>(sc.dev(8ull * nq));
    uint64_t *d_nodes = static_cast<uint64_t *>(sc.dev(8ull * cap));
    uint32_t *d_out = static_cast<uint32_t *>(sc.dev((nq * w.cols + (size_t)cap * 8 + 1) * 4));
    uint32_t *d_cnt = d_out + nq * w.cols + (size_t)cap * 8;
    lgk::FsQueries a;
    a.src = absorb;
    a.nwords = 8;
    a.n = w.rows;
    a.s = nq;
    a.q = d_q;
    a.nodes = d_nodes;
    a.nodes_cap = cap;
    a.nnodes = d_cnt;
    a.nsq = nsq;
    a.out = out;
    a.mirror = absorb_mirror;
    CK(c, lgk::fs_queries(c->L, fs, a));
    CK(c, lgk::gather_opening(c->L, w.E.u32(), w.rows, w.cols, d_q, nq, w.tree.u32(), d_nodes, cap, d_cnt, d_out));
    const uint32_t *h = sc.download_deferred(d_out, nq * w.cols + (size_t)cap * 8 + 1);
    const uint32_t cols = w.cols;
    sc.finalizers.push_back([h, nq, cap, cols, op]() {
        op->rows.assign_fixed(h, nq, cols);
        const uint32_t nr = std::min(h[nq * cols + (size_t)cap * 8], cap);
        op->merkle.assign_fixed(reinterpret_cast<const uint8_t *>(h + nq * cols), nr, 32);
    });
    return {d_out, d_q};
}

// induce_sumcheck_poly_parallel (src/sumcheck_polys.rs:74-160) entirely on
// the device from device-resident rows (nq x 2^nch) and queries; the
// enforced sum lands in d_sum (1 word).
// The challenges (vch, alpha) come from the host, or from the device as
// d_vch / d_alpha.
void induce_dev(lg_ctx *c, Scratch &sc, uint32_t n, const uint32_t *d_rows, uint32_t nq, const uint32_t *vch,
                uint32_t nch, const uint64_t *d_q, uint32_t alpha, uint32_t *d_out, uint32_t *d_sum,
                const uint32_t *d_vch = nullptr, const uint32_t *d_alpha = nullptr) {
    std::vector<uint32_t> gr = d_vch ? std::vector<uint32_t>() : lg::lagrange_basis(vch, nch);
    std::vector<uint32_t> sks = lg::eval_sk_at_vks(1ull << n);
    lgk::InducePlan plan = lgk::induce_plan(n, nq);
    uint32_t *d_S = static_cast<uint32_t *>(sc.dev(4ull * nq * std::max<uint32_t>(n, 1)));
    uint32_t *d_apow = static_cast<uint32_t *>(sc.dev(8ull * nq));
    uint32_t *d_lo = static_cast<uint32_t *>(sc.dev(4ull * nq << plan.b));
    uint32_t *d_hi = static_cast<uint32_t *>(sc.dev(4ull * nq << (n - plan.b)));
    if (plan.needs_zero) CK(c, cudaMemsetAsync(d_out, 0, 4ull << n, c->stream));
    CK(c, lgk::induce_fused(c->L, plan, d_rows, 1u << nch, d_vch ? nullptr : gr.data(), d_q, nq, alpha, n,
                            sks.data(), d_S, d_apow, d_vch, d_alpha, d_lo, d_hi, d_out, d_sum));
}

// host rows / queries (verifier, kernel-level API) -> induce_dev
// The enforced sum arrives in pinned memory, valid after sc.finish().
const uint32_t *induce_host_rows_later(lg_ctx *c, Scratch &sc, uint32_t n, const uint32_t *rows, size_t nrows,
                                       const uint32_t *vch, uint32_t nch, const std::vector<uint64_t> &q,
                                       uint32_t alpha, uint32_t *d_out) {
    const uint32_t *d_rows = sc.upload(rows, nrows << nch);
    const uint64_t *d_q = sc.upload(q.data(), q.size());
    uint32_t *d_sum = static_cast<uint32_t *>(sc.dev(16));
    induce_dev(c, sc, n, d_rows, (uint32_t)nrows, vch, nch, d_q, alpha, d_out, d_sum);
    return sc.download_later(d_sum, 1);
}
uint32_t induce_host_rows(lg_ctx *c, Scratch &sc, uint32_t n, const uint32_t *rows, size_t nrows,
                          const uint32_t *vch, uint32_t nch, const std::vector<uint64_t> &q, uint32_t alpha,
                          uint32_t *d_out) {
    const uint32_t *h = induce_host_rows_later(c, sc, n, rows, nrows, vch, nch, q, alpha, d_out);
    sync(c);
    return *h;
}

// partial_eval by any number of challenges (host rs, or device d_rs),
// chunks of <= 6 per launch
void partial_eval_dev(lg_ctx *c, const uint32_t *d_in, uint32_t log_len, const uint32_t *rs, uint32_t k,
                      uint32_t *d_out, const uint32_t *d_rs = nullptr) {
    DBuf tmp[2];
    const uint32_t *src = d_in;
    uint32_t cur = log_len, done = 0, which = 0;
    while (done < k) {
        const uint32_t kk = std::min<uint32_t>(6, k - done);
        uint32_t *dst;
        if (done + kk == k) dst = d_out;
        else {
            tmp[which] = DBuf(c, 4ull << (cur - kk));
            dst = tmp[which].u32();
        }
        CK(c, lgk::fold_eq(c->L, src, dst, cur, kk, d_rs ? nullptr : rs + done, d_rs ? d_rs + done : nullptr));
        src = dst;
        which ^= 1;
        cur -= kk;
        done += kk;
    }
}

void absorb3(lg::Transcript &fs, const std::array<uint32_t, 3> &s) { fs.absorb_u32s(s.data(), 3); }

// ------------------------------------------------------------------ prover
// prover (src/prover.rs:15-199).  The transcript runs on the device
// (lg_fs.cu) up to yr: each challenge is squeezed into device memory
// right after what it depends on is absorbed, and the kernels read it from
// there, so the whole proof is queued without a host round trip.  yr is
// then downloaded with the transcript state and the host finishes the
// transcript (absorbing yr is long serial hashing) and the last opening.
// Roots, sumcheck triples and openings are downloaded asynchronously and
// materialised at the end; a failed prover assertion flagged on the device
// (src/ligerito.rs:35,52, get_distinct_queries) raises ProverAssert there.
void prove_impl(lg_ctx *c, Scratch &sc, const lg_config &cfg, const uint32_t *d_poly, uint64_t len, lg::Proof &P,
                const uint32_t *h_poly = nullptr) {
    const uint32_t steps = cfg.recursive_steps;
    uint32_t nrounds = 0;
    for (uint32_t i = 0; i < steps; ++i) nrounds += cfg.ks[i];
    const uint32_t ntri = 1 + nrounds + (steps - 1);  // sumcheck triples, in transcript order
    auto *fs = static_cast<lgk::FsState *>(sc.dev(sizeof(lgk::FsState)));
    uint32_t *chal = static_cast<uint32_t *>(sc.dev(4ull * (cfg.initial_k + nrounds + 3 * steps + 4)));
    // s0, s1, s2, enforced sum per triple, then the fused steps' block ticket
    uint32_t *tri = static_cast<uint32_t *>(sc.dev(16ull * ntri + 16));
    uint32_t *ticket = tri + 4 * ntri;
    uint32_t nchal = 0, ntri_used = 0;
    auto next_chal = [&](uint32_t n) { uint32_t *p = chal + nchal; nchal += n; return p; };
    auto next_tri = [&]() { return tri + 4 * ntri_used++; };
    CK(c, cudaMemsetAsync(tri, 0, 16ull * ntri + 16, c->stream));
    CK(c, lgk::fs_init(c->L, fs, LG_FS_SEED));
    // A root reaches the host from the arena copy that the transcript
    // kernel absorbing it writes (the tree itself may be freed before the
    // deferred copies are queued).
    auto root_later = [&](std::vector<uint8_t> *dst) {
        uint32_t *mirror = static_cast<uint32_t *>(sc.dev(32));
        const uint32_t *h = sc.download_deferred(mirror, 8);
        sc.finalizers.push_back([h, dst]() {
            const uint8_t *b = reinterpret_cast<const uint8_t *>(h);
            dst->assign(b, b + 32);
        });
        return mirror;
    };
    auto tail = [&](bool check, uint32_t nsq, uint32_t *out) {
        lgk::FsTail a;
        a.fs = fs;
        a.ticket = ticket;
        a.check = check;
        a.nsq = nsq;
        a.out = out;
        return a;
    };
    auto step = [&](const uint32_t *src, uint32_t nwords, bool check, uint32_t nsq, uint32_t *out,
                    uint32_t *mirror) {
        lgk::FsStep a;
        a.mirror = mirror;
        a.src = src;
        a.nwords = nwords;
        a.check = check;
        a.nsq = nsq;
        a.out = out;
        CK(c, lgk::fs_step(c->L, fs, a));
    };
    // lg_dump_intermediates only (no-ops otherwise)
    auto dump_commit = [&](uint32_t level, uint32_t log_m, const Witness &w) {
        if (!c->dump_cb) return;
        const Code code = get_code(c, log_m);
        dump_dev(c, "twiddles", level, code.tw, 4 * ((4ull << log_m) - 1));
        dump_dev(c, "pis", level, code.pis, 4ull << log_m);
        dump_dev(c, "encoded", level, w.E.p, 4ull * w.rows * w.cols);
        dump_dev(c, "tree", level, w.tree.p, 32ull * (2 * w.rows - 1));
    };
    auto dump_opening = [&](uint32_t level, const std::pair<const uint32_t *, const uint64_t *> &op, uint32_t cols,
                            const uint32_t *d_alpha) {
        dump_dev(c, "queries", level, op.second, 8ull * LG_NUM_QUERIES);
        dump_dev(c, "opened_rows", level, op.first, 4ull * LG_NUM_QUERIES * cols);
        dump_dev(c, "alpha", level, d_alpha, 4);
    };
    auto dump_triple = [&](const uint32_t *t) { dump_dev(c, "triple", (uint32_t)((t - tri) / 4), t, 12); };
    uint32_t round_no = 0;

    Witness w0 = h_poly ? commit_from_host(c, sc, h_poly, const_cast<uint32_t *>(d_poly), cfg.initial_log_m,
                                           1u << cfg.initial_log_n)
                        : commit(c, d_poly, cfg.initial_log_m, 1u << cfg.initial_log_n);  // :32-37
    dump_commit(0, cfg.initial_log_m, w0);
    uint32_t *root_m = root_later(&P.initial_root);
    P.recursive_roots.resize(steps);
    P.recursive.resize(steps - 1);  // openings are filled in by pointer later
    const uint32_t *pe0 = next_chal(cfg.initial_k);
    step(w0.root(), 8, false, cfg.initial_k, const_cast<uint32_t *>(pe0), root_m);  // :48-50
    uint32_t fv = cfg.initial_log_m;  // log2 |f|
    DBuf f(c, 4ull << fv);
    partial_eval_dev(c, d_poly, cfg.initial_log_m + cfg.initial_log_n, nullptr, cfg.initial_k, f.u32(), pe0);  // :52-53
    dump_dev(c, "fold_challenges", 0, pe0, 4ull * cfg.initial_k);
    dump_dev(c, "folded", 0, f.p, 4ull << fv);

    Witness wprev = commit(c, f.u32(), cfg.log_m[0], 1u << cfg.log_n[0]);  // :55-60
    dump_commit(1, cfg.log_m[0], wprev);
    root_m = root_later(&P.recursive_roots[0]);
    uint32_t *alpha = next_chal(1);
    auto opened = open_rows_dev(c, sc, w0, fs, wprev.root(), 1, alpha, &P.initial, root_m);  // :64-76
    DBuf B(c, 4ull << fv);
    uint32_t *t = next_tri();
    induce_dev(c, sc, fv, opened.first, LG_NUM_QUERIES, nullptr, cfg.initial_k, opened.second, 0, B.u32(), t + 3, pe0,
               alpha);  // :78-85
    dump_opening(0, opened, w0.cols, alpha);
    dump_dev(c, "basis", 0, B.p, 4ull << fv);
    dump_dev(c, "enforced_sum", 0, t + 3, 4);
    w0.E.reset();
    w0.tree.reset();
    uint32_t *r = next_chal(1);
    // SumcheckProverInstance::new, then :93 (src/ligerito.rs:35) and the
    // first challenge of :97
    const lgk::FsTail t0 = tail(true, 1, r);
    CK(c, lgk::eval013(c->L, f.u32(), B.u32(), fv, t, &t0));
    dump_triple(t);

    DBuf f2(c, 4ull << (fv - 1)), B2(c, 4ull << (fv - 1));
    for (uint32_t i = 0; i < steps; ++i) {
        const uint32_t *rs = r;  // this step's ks[i] round challenges are consecutive
        // The last commitment is final here: a side stream brings its matrix
        // and tree to the host during this step's rounds, so the final
        // opening needs no second round trip (when they are small and the
        // pinned arena has room for them and the last downloads).
        const uint32_t *h_E = nullptr;
        const uint8_t *h_tree = nullptr;
        const size_t eb = 4ull * wprev.rows * wprev.cols, tb = 32ull * (2 * wprev.rows - 1);
        if (i == steps - 1 && eb + tb <= (4u << 20) &&
            c->pin_used + eb + tb + (4ull << fv) + (1u << 16) <= c->pin_cap) {
            uint8_t *h = sc.pin(eb + tb);
            h_E = reinterpret_cast<const uint32_t *>(h);
            h_tree = h + eb;
            CK(c, cudaEventRecord(c->copy_ev[6], c->stream));
            CK(c, cudaStreamWaitEvent(c->copy_stream, c->copy_ev[6], 0));
            CK(c, cudaMemcpyAsync(h, wprev.E.p, eb, cudaMemcpyDeviceToHost, c->copy_stream));
            CK(c, cudaMemcpyAsync(h + eb, wprev.tree.p, tb, cudaMemcpyDeviceToHost, c->copy_stream));
            CK(c, cudaEventRecord(c->copy_ev[6], c->copy_stream));
        }
        for (uint32_t k = 0; k < cfg.ks[i]; ++k) {  // :97-102
            t = next_tri();
            const bool more = k + 1 < cfg.ks[i];
            uint32_t *rn = more ? next_chal(1) : nullptr;
            const lgk::FsTail tk = tail(false, more ? 1 : 0, rn);
            CK(c, lgk::fold_round(c->L, f.u32(), B.u32(), fv, 0, f2.u32(), B2.u32(), t, r, &tk));
            std::swap(f, f2);
            std::swap(B, B2);
            fv -= 1;
            if (c->dump_cb) {
                dump_dev(c, "round_challenge", round_no, r, 4);
                dump_dev(c, "round_f", round_no, f.p, 4ull << fv);
                dump_dev(c, "round_basis", round_no, B.p, 4ull << fv);
                dump_triple(t);
            }
            ++round_no;
            r = rn;
        }
        if (i == steps - 1) {  // :104-143
            P.yr.resize(1ull << fv);
            const uint32_t *hy = sc.download_later(f.u32(), 1ull << fv);
            const lgk::FsState *hs = sc.download_later(fs, 1);
            const uint32_t *ht = sc.download_later(tri, 4ull * ntri);
            if (h_E) CK(c, cudaStreamWaitEvent(c->stream, c->copy_ev[6], 0));
            // wait for these three only; the deferred downloads (roots,
            // openings) go out now, while the host finishes the transcript
            sync(c);
            sc.flush();
            std::memcpy(P.yr.data(), hy, 4ull << fv);
            for (uint32_t j = 0; j < ntri; ++j) P.transcript.push_back({ht[4 * j], ht[4 * j + 1], ht[4 * j + 2]});
            if (hs->err) throw ProverAssert{};
            lg::Transcript fsh(LG_FS_SEED);
            std::memcpy(fsh.h.h, hs->h, sizeof hs->h);
            for (uint32_t k = 0; k < hs->nw && k < 16; ++k)
                for (int b = 0; b < 4; ++b) fsh.h.buf[4 * k + b] = (uint8_t)(hs->w[k] >> (24 - 8 * b));
            fsh.h.total = hs->total;
            fsh.h.n = 4 * hs->nw;
            fsh.counter = hs->counter;
            fsh.absorb_u32s(P.yr.data(), P.yr.size());
            std::vector<uint64_t> q;
            if (!fsh.get_distinct_queries(wprev.rows, LG_NUM_QUERIES, q)) throw ProverAssert{};
            dump_host(c, "yr", steps, P.yr.data(), 4 * P.yr.size());
            dump_host(c, "queries", steps, q.data(), 8 * q.size());
            if (h_E) open_rows_host(h_E, h_tree, wprev.rows, wprev.cols, q, &P.final_);
            else open_rows(c, sc, wprev, q, &P.final_);
            return;
        }
        Witness wn = commit(c, f.u32(), cfg.log_m[i + 1], 1u << cfg.log_n[i + 1]);  // :145-155
        dump_commit(i + 2, cfg.log_m[i + 1], wn);
        root_m = root_later(&P.recursive_roots[i + 1]);
        uint32_t *al = next_chal(1);
        auto op = open_rows_dev(c, sc, wprev, fs, wn.root(), 1, al, &P.recursive[i], root_m);  // :156-172
        DBuf bi(c, 4ull << fv);
        t = next_tri();
        induce_dev(c, sc, fv, op.first, LG_NUM_QUERIES, nullptr, cfg.ks[i], op.second, 0, bi.u32(), t + 3, rs, al);
        dump_opening(i + 1, op, wprev.cols, al);
        dump_dev(c, "basis", i + 1, bi.p, 4ull << fv);
        dump_dev(c, "enforced_sum", i + 1, t + 3, 4);
        // introduce_new, :187-193 (src/ligerito.rs:52): the glue challenge,
        // then the next step's first round challenge
        uint32_t *beta = next_chal(2);
        const lgk::FsTail ti = tail(true, 2, beta);
        CK(c, lgk::eval013(c->L, f.u32(), bi.u32(), fv, t, &ti));
        dump_triple(t);
        r = beta + 1;
        CK(c, lgk::axpy(c->L, B.u32(), bi.u32(), fv, 0, beta));  // glue
        dump_dev(c, "beta", i + 1, beta, 4);
        dump_dev(c, "basis_sum", i + 1, B.p, 4ull << fv);
        wprev = std::move(wn);
    }
    throw ProverAssert{};  // :198
}

// ------------------------------------------------------ lockstep batches
// B proofs of one config in lockstep: each kernel launch of the prover
// above takes all B proofs at once (the proof index is a grid dimension),
// proof b in its own slice of every buffer, so that small proofs fill the
// GPU and the launch and transcript latencies are paid once per batch.
// The B polynomials are contiguous on the device (proof b at
// d_polys + b * len); the columns of a commitment are independent, so the
// B encodings are one matrix of B * n columns.  Each proof is the bytes
// prove_impl gives alone.
struct BatchWitness {
    DBuf E, tree;
    uint64_t rows = 0;
    uint32_t cols = 0, B = 0;
    uint64_t e_stride() const { return rows * cols; }       // words per proof
    uint64_t t_stride() const { return 8 * (2 * rows - 1); } // words per proof
    const uint32_t *root() const { return tree.u32() + 8 * (2 * rows - 2); }  // proof 0's
};

BatchWitness commit_batch(lg_ctx *c, const uint32_t *d_polys, uint32_t log_m, uint32_t n, uint32_t B) {
    const Code code = get_code(c, log_m);
    BatchWitness w;
    w.rows = 4ull << log_m;
    w.cols = n;
    w.B = B;
    w.E = DBuf(c, 4ull * B * w.e_stride());
    w.tree = DBuf(c, 4ull * B * w.t_stride());
    {
        DBuf scaled(c, log_m > 6 ? 4ull * B * n << log_m : 0);
        rs_encode(c, code, d_polys, log_m, B * n, w.E.u32(), w.rows, scaled.u32());
    }
    CK(c, lgk::leaf_hashes(c->L, w.E.u32(), w.rows, n, w.tree.u32(), B, w.e_stride(), w.t_stride()));
    CK(c, lgk::merkle_upper(c->L, w.tree.u32(), w.rows, B, w.t_stride()));
    return w;
}

// open_rows_dev for the B proofs: fs_queries absorbs each proof's `absorb`
// (8 words, proof b at absorb + b * absorb_stride; nothing when absorb is
// null) and draws its queries and
// node list; one gather opens all.  Returns the device copy of the opened
// rows (proof b at rows + b * stride) and of the queries (nq per proof).
struct BatchOpened {
    const uint32_t *rows;
    uint64_t stride;
    const uint64_t *q;
};
BatchOpened open_rows_batch(lg_ctx *c, Scratch &sc, const BatchWitness &w, lgk::FsState *fs, const uint32_t *absorb,
                            uint64_t absorb_stride, uint32_t nsq, uint32_t *out, uint64_t out_stride,
                            const std::vector<lg::Opening *> &ops, uint32_t *mirror) {
    const uint32_t nq = LG_NUM_QUERIES, B = w.B;
    uint32_t depth = 0;
    while ((1ull << depth) < w.rows) ++depth;
    const uint32_t cap = nq * std::max<uint32_t>(depth, 1);
    const uint64_t os = ((uint64_t)nq * w.cols + (uint64_t)cap * 8 + 1 + 3) & ~3ull;  // words per proof
    uint64_t *d_q = static_cast<uint64_t *>(sc.dev(8ull * nq * B));
    uint64_t *d_nodes = static_cast<uint64_t *>(sc.dev(8ull * cap * B));
    uint32_t *d_out = static_cast<uint32_t *>(sc.dev(4ull * os * B));
    uint32_t *d_cnt = d_out + (uint64_t)nq * w.cols + (uint64_t)cap * 8;
    lgk::FsQueries a;
    a.src = absorb;
    a.nwords = absorb ? 8 : 0;
    a.n = w.rows;
    a.s = nq;
    a.q = d_q;
    a.nodes = d_nodes;
    a.nodes_cap = cap;
    a.nnodes = d_cnt;
    a.nsq = nsq;
    a.out = out;
    a.mirror = mirror;
    lgk::FsStrides fst;
    fst.src = absorb_stride;
    fst.out = out_stride;
    fst.mirror = 8;
    fst.q = nq;
    fst.nodes = cap;
    fst.nnodes = os;
    CK(c, lgk::fs_queries(c->L, fs, a, B, fst));
    lgk::GatherStrides gst;
    gst.E = w.e_stride();
    gst.q = nq;
    gst.tree = w.t_stride();
    gst.nodes = cap;
    gst.count = os;
    gst.out = os;
    CK(c, lgk::gather_opening(c->L, w.E.u32(), w.rows, w.cols, d_q, nq, w.tree.u32(), d_nodes, cap, d_cnt, d_out, B,
                              gst));
    const uint32_t *h = sc.download_deferred(d_out, os * B);
    const uint32_t cols = w.cols;
    sc.finalizers.push_back([h, nq, cap, cols, os, ops]() {
        for (size_t b = 0; b < ops.size(); ++b) {
            const uint32_t *hb = h + b * os;
            ops[b]->rows.assign_fixed(hb, nq, cols);
            const uint32_t nr = std::min(hb[(uint64_t)nq * cols + (uint64_t)cap * 8], cap);
            ops[b]->merkle.assign_fixed(reinterpret_cast<const uint8_t *>(hb + (uint64_t)nq * cols), nr, 32);
        }
    });
    return {d_out, os, d_q};
}

// induce_dev for the B proofs: rows (nq x 2^nch each, proof b at
// d_rows + b * rows_stride), queries (nq each), basis out (2^n each), the
// enforced sums (d_sum + b * sum_stride) and the device challenges (vch,
// alpha: + b * chal_stride).
void induce_batch(lg_ctx *c, Scratch &sc, uint32_t n, const uint32_t *d_rows, uint64_t rows_stride, uint32_t nq,
                  uint32_t nch, const uint64_t *d_q, uint32_t *d_out, uint32_t *d_sum, uint64_t sum_stride,
                  const uint32_t *d_vch, const uint32_t *d_alpha, uint64_t chal_stride, uint32_t B) {
    std::vector<uint32_t> sks = lg::eval_sk_at_vks(1ull << n);
    const lgk::InducePlan plan = lgk::induce_plan(n, nq);
    lgk::InduceStrides st;
    st.rows = rows_stride;
    st.q = nq;
    st.S = (uint64_t)nq * std::max<uint32_t>(n, 1);
    st.apow = 2ull * nq;
    st.lo = (uint64_t)nq << plan.b;
    st.hi = (uint64_t)nq << (n - plan.b);
    st.out = 1ull << n;
    st.sum = sum_stride;
    st.rs = chal_stride;
    st.alpha = chal_stride;
    uint32_t *d_S = static_cast<uint32_t *>(sc.dev(4ull * st.S * B));
    uint32_t *d_apow = static_cast<uint32_t *>(sc.dev(4ull * st.apow * B));
    uint32_t *d_lo = static_cast<uint32_t *>(sc.dev(4ull * st.lo * B));
    uint32_t *d_hi = static_cast<uint32_t *>(sc.dev(4ull * st.hi * B));
    if (plan.needs_zero) CK(c, cudaMemsetAsync(d_out, 0, (4ull << n) * B, c->stream));
    CK(c, lgk::induce_fused(c->L, plan, d_rows, 1u << nch, nullptr, d_q, nq, 0, n, sks.data(), d_S, d_apow, d_vch,
                            d_alpha, d_lo, d_hi, d_out, d_sum, B, st));
}

// partial_eval_dev for the B proofs (inputs in_stride apart, outputs and
// intermediates packed, challenges rs_stride apart)
void partial_eval_batch(lg_ctx *c, const uint32_t *d_in, uint64_t in_stride, uint32_t log_len, uint32_t k,
                        uint32_t *d_out, const uint32_t *d_rs, uint64_t rs_stride, uint32_t B) {
    DBuf tmp[2];
    const uint32_t *src = d_in;
    uint64_t src_stride = in_stride;
    uint32_t cur = log_len, done = 0, which = 0;
    while (done < k) {
        const uint32_t kk = std::min<uint32_t>(6, k - done);
        uint32_t *dst;
        if (done + kk == k) dst = d_out;
        else {
            tmp[which] = DBuf(c, (4ull << (cur - kk)) * B);
            dst = tmp[which].u32();
        }
        lgk::FoldStrides st;
        st.in = src_stride;
        st.out = 1ull << (cur - kk);
        st.rs = rs_stride;
        CK(c, lgk::fold_eq(c->L, src, dst, cur, kk, nullptr, d_rs + done, B, st));
        src = dst;
        src_stride = st.out;
        which ^= 1;
        cur -= kk;
        done += kk;
    }
}

// prove_impl for B proofs of cfg in lockstep.  P[b] receives proof b;
// bad[b] is set when proof b's prover assertion fails (its P[b] is then
// incomplete).
void prove_batch_impl(lg_ctx *c, Scratch &sc, const lg_config &cfg, const uint32_t *d_polys, uint64_t len,
                      uint32_t B, const std::vector<lg::Proof *> &P, std::vector<char> &bad) {
    if (B == 0 || B > lgk::kMaxTickets || P.size() != B) throw BadConfig{};
    bad.assign(B, 0);
    const uint32_t steps = cfg.recursive_steps;
    uint32_t nrounds = 0;
    for (uint32_t i = 0; i < steps; ++i) nrounds += cfg.ks[i];
    const uint32_t ntri = 1 + nrounds + (steps - 1);
    // per-proof strides (words): challenges, then triples + the fused
    // steps' ticket
    const uint64_t CH = (cfg.initial_k + nrounds + 3 * steps + 4 + 3) & ~3u, TR = 4ull * ntri + 4;
    auto *fs = static_cast<lgk::FsState *>(sc.dev(sizeof(lgk::FsState) * B));
    uint32_t *chal = static_cast<uint32_t *>(sc.dev(4ull * CH * B));
    uint32_t *tri = static_cast<uint32_t *>(sc.dev(4ull * TR * B));
    uint32_t nchal = 0, ntri_used = 0;
    auto next_chal = [&](uint32_t n) { uint32_t *p = chal + nchal; nchal += n; return p; };
    auto next_tri = [&]() { return tri + 4 * ntri_used++; };
    CK(c, cudaMemsetAsync(tri, 0, 4ull * TR * B, c->stream));
    CK(c, lgk::fs_init(c->L, fs, LG_FS_SEED, B));
    auto root_later = [&](std::vector<std::vector<uint8_t> *> dst) {
        uint32_t *mirror = static_cast<uint32_t *>(sc.dev(32ull * B));
        const uint32_t *h = sc.download_deferred(mirror, 8ull * B);
        sc.finalizers.push_back([h, dst]() {
            for (size_t b = 0; b < dst.size(); ++b) {
                const uint8_t *p = reinterpret_cast<const uint8_t *>(h + 8 * b);
                dst[b]->assign(p, p + 32);
            }
        });
        return mirror;
    };
    auto each = [&](auto get) {
        std::vector<decltype(get(P[0]))> v;
        for (auto *p : P) v.push_back(get(p));
        return v;
    };
    auto tail = [&](bool check, uint32_t nsq, uint32_t *out) {
        lgk::FsTail a;
        a.fs = fs;
        a.ticket = tri + 4 * ntri;
        a.check = check;
        a.nsq = nsq;
        a.out = out;
        return a;
    };
    auto rstr = [&](uint32_t fv) {
        lgk::RoundStrides st;
        st.f = st.g = 1ull << fv;
        st.fo = st.go = 1ull << (fv - 1);
        st.acc = TR;
        st.r = CH;
        st.fs = 1;
        st.ticket = TR;
        st.out = CH;
        return st;
    };
    const uint32_t nq = LG_NUM_QUERIES;

    for (auto *p : P) {
        p->recursive_roots.resize(steps);
        p->recursive.resize(steps - 1);
    }
    BatchWitness w0 = commit_batch(c, d_polys, cfg.initial_log_m, 1u << cfg.initial_log_n, B);  // :32-37
    uint32_t *root_m = root_later(each([](lg::Proof *p) { return &p->initial_root; }));
    const uint32_t *pe0 = next_chal(cfg.initial_k);
    {
        lgk::FsStep a;
        a.src = w0.root();
        a.nwords = 8;
        a.nsq = cfg.initial_k;
        a.out = const_cast<uint32_t *>(pe0);
        a.mirror = root_m;
        lgk::FsStrides st;
        st.src = w0.t_stride();
        st.out = CH;
        st.mirror = 8;
        CK(c, lgk::fs_step(c->L, fs, a, B, st));  // :48-50
    }
    uint32_t fv = cfg.initial_log_m;
    DBuf f(c, (4ull << fv) * B);
    partial_eval_batch(c, d_polys, len, cfg.initial_log_m + cfg.initial_log_n, cfg.initial_k, f.u32(), pe0, CH,
                       B);  // :52-53

    BatchWitness wprev = commit_batch(c, f.u32(), cfg.log_m[0], 1u << cfg.log_n[0], B);  // :55-60
    root_m = root_later(each([](lg::Proof *p) { return &p->recursive_roots[0]; }));
    uint32_t *alpha = next_chal(1);
    BatchOpened op = open_rows_batch(c, sc, w0, fs, wprev.root(), wprev.t_stride(), 1, alpha, CH,
                                     each([](lg::Proof *p) { return &p->initial; }), root_m);  // :64-76
    DBuf Bv(c, (4ull << fv) * B);
    uint32_t *t = next_tri();
    induce_batch(c, sc, fv, op.rows, op.stride, nq, cfg.initial_k, op.q, Bv.u32(), t + 3, TR, pe0, alpha, CH,
                 B);  // :78-85
    w0.E.reset();
    w0.tree.reset();
    uint32_t *r = next_chal(1);
    const lgk::FsTail t0 = tail(true, 1, r);
    CK(c, lgk::eval013(c->L, f.u32(), Bv.u32(), fv, t, &t0, B, rstr(fv)));

    DBuf f2(c, (4ull << (fv - 1)) * B), B2(c, (4ull << (fv - 1)) * B);
    for (uint32_t i = 0; i < steps; ++i) {
        const uint32_t *rs = r;
        for (uint32_t k = 0; k < cfg.ks[i]; ++k) {  // :97-102
            t = next_tri();
            const bool more = k + 1 < cfg.ks[i];
            uint32_t *rn = more ? next_chal(1) : nullptr;
            const lgk::FsTail tk = tail(false, more ? 1 : 0, rn);
            CK(c, lgk::fold_round(c->L, f.u32(), Bv.u32(), fv, 0, f2.u32(), B2.u32(), t, r, &tk, B, rstr(fv)));
            std::swap(f, f2);
            std::swap(Bv, B2);
            fv -= 1;
            r = rn;
        }
        if (i == steps - 1) {  // :104-143
            // The rest of each transcript runs on the device as well (one
            // block per proof, all at once): absorb yr, draw the final
            // queries and their node list, and one gather opens every
            // proof -- no host round trip inside the batch.
            const uint64_t ny = 1ull << fv;
            for (uint64_t off = 0; off < ny; off += 1024) {
                lgk::FsStep a;
                a.src = f.u32() + off;
                a.nwords = (uint32_t)std::min<uint64_t>(1024, ny - off);
                lgk::FsStrides st;
                st.src = ny;
                CK(c, lgk::fs_step(c->L, fs, a, B, st));
            }
            open_rows_batch(c, sc, wprev, fs, nullptr, 0, 0, nullptr, 0,
                            each([](lg::Proof *p) { return &p->final_; }), nullptr);
            // (f is freed when this returns: its copy is queued now)
            const uint32_t *hy = sc.download_later(f.u32(), ny * B);
            const lgk::FsState *hs = sc.download_deferred(fs, B);
            const uint32_t *ht = sc.download_deferred(tri, TR * B);
            std::vector<char> *flags = &bad;
            sc.finalizers.push_back([hy, hs, ht, ny, ntri, TR, P, flags]() {
                for (size_t b = 0; b < P.size(); ++b) {
                    lg::Proof &pb = *P[b];
                    pb.yr.assign(hy + b * ny, hy + (b + 1) * ny);
                    for (uint32_t j = 0; j < ntri; ++j) {
                        const uint32_t *x = ht + b * TR + 4 * j;
                        pb.transcript.push_back({x[0], x[1], x[2]});
                    }
                    (*flags)[b] = hs[b].err != 0;  // a prover assertion failed on the device
                }
            });
            return;
        }
        BatchWitness wn = commit_batch(c, f.u32(), cfg.log_m[i + 1], 1u << cfg.log_n[i + 1], B);  // :145-155
        const uint32_t ip1 = i + 1, ii = i;
        root_m = root_later(each([ip1](lg::Proof *p) { return &p->recursive_roots[ip1]; }));
        uint32_t *al = next_chal(1);
        BatchOpened o = open_rows_batch(c, sc, wprev, fs, wn.root(), wn.t_stride(), 1, al, CH,
                                        each([ii](lg::Proof *p) { return &p->recursive[ii]; }), root_m);  // :156-172
        DBuf bi(c, (4ull << fv) * B);
        t = next_tri();
        induce_batch(c, sc, fv, o.rows, o.stride, nq, cfg.ks[i], o.q, bi.u32(), t + 3, TR, rs, al, CH, B);
        uint32_t *beta = next_chal(2);
        const lgk::FsTail ti = tail(true, 2, beta);
        CK(c, lgk::eval013(c->L, f.u32(), bi.u32(), fv, t, &ti, B, rstr(fv)));
        r = beta + 1;
        lgk::RoundStrides ax = rstr(fv);
        CK(c, lgk::axpy(c->L, Bv.u32(), bi.u32(), fv, 0, beta, B, ax));  // glue
        wprev = std::move(wn);
    }
    throw ProverAssert{};  // :198
}

// ---------------------------------------------------------------- verifier
struct Quad { uint32_t a, b, c; };  // QuadraticPoly, src/sumcheck.rs:38-65
Quad quad_from_evals(uint32_t at0, uint32_t at1, uint32_t atx) {  // :67-81, x = 3
    const uint32_t x = 3;
    static const uint32_t inv_den = lg::gf_inv(lg::gf_mul(x, x) ^ x);
    const uint32_t num = atx ^ at0 ^ lg::gf_mul(x, at1 ^ at0);
    const uint32_t a = lg::gf_mul(num, inv_den);
    return {a, at1 ^ at0 ^ a, at0};
}
uint32_t eval_quad(const Quad &p, uint32_t r) { return lg::gf_mul(lg::gf_mul(p.a, r), r) ^ lg::gf_mul(p.b, r) ^ p.c; }

// merkle_tree::verify of an opening (leaf bytes = LE words of each row)
bool opening_ok_host(const std::vector<uint8_t> &root, const lg::Opening &o, size_t depth,
                     const std::vector<uint64_t> &q) {
    if (o.rows.size() < q.size()) return false;  // layer index panic
    std::vector<std::array<uint8_t, 32>> layer(q.size());
    std::vector<uint8_t> buf;
    for (size_t i = 0; i < q.size(); ++i) {
        buf.resize(4 * o.rows.len(i));
        for (size_t j = 0; j < o.rows.len(i); ++j) {
            uint32_t v = o.rows.ptr(i)[j];
            buf[4 * j] = (uint8_t)v; buf[4 * j + 1] = (uint8_t)(v >> 8);
            buf[4 * j + 2] = (uint8_t)(v >> 16); buf[4 * j + 3] = (uint8_t)(v >> 24);
        }
        lg::blake3_hash(buf.data(), buf.size(), layer[i].data());
    }
    bool ok = false;
    if (!lg::merkle_verify(root.data(), root.size(), o.merkle, depth, layer, q, &ok)) return false;
    return ok;
}

// The same check on the device when the opening is well formed (the first
// nq rows of one length, 1..256 words; sorted distinct queries inside the
// tree; every proof node the opening consumes present and 32 bytes), which
// are exactly the cases where the host walk neither panics nor meets a
// sibling of another length.  Anything else takes the host walk.
// Checks whose failure is a verifier panic wherever it is found are queued
// on the device as the verifier goes and decided by finalizers at the next
// synchronisation (sc.finish(), which throws their panic).  Nothing the
// verifier computes depends on them, so deciding them late gives the same
// outcome as the reference's early panics.
void check_opening(lg_ctx *c, Scratch &sc, const std::vector<uint8_t> &root, const lg::Opening &o, size_t depth,
                   const std::vector<uint64_t> &q) {
    const size_t nq = q.size();
    bool fast = nq >= 1 && nq <= 256 && o.rows.size() >= nq && depth >= 1 && depth <= 63;
    const size_t ncols = fast ? o.rows.len(0) : 0;
    for (size_t i = 0; fast && i < nq; ++i)
        fast = o.rows.len(i) == ncols && (i == 0 || q[i] > q[i - 1]) && (q[i] >> depth) == 0;
    fast = fast && ncols >= 1 && ncols <= 256;
    std::vector<NodeRef> refs;
    if (fast) {
        lg::merkle_proof_nodes(q, 1ull << depth, refs);
        fast = o.merkle.size() >= refs.size();
        for (size_t j = 0; fast && j < refs.size(); ++j) fast = o.merkle.len(j) == 32;
    }
    if (!fast) {
        if (!opening_ok_host(root, o, depth, q)) throw VerifyPanic{};
        return;
    }
    const uint32_t *d_rows = sc.upload(o.rows.data.data(), nq * ncols);
    const uint64_t *d_q = sc.upload(q.data(), nq);
    const uint32_t *d_proof = refs.empty() ? nullptr
                                           : sc.upload(reinterpret_cast<const uint32_t *>(o.merkle.data.data()),
                                                       8 * refs.size());
    uint32_t *d_out = static_cast<uint32_t *>(sc.dev(9 * 4));
    CK(c, lgk::opening_check(c->L, d_rows, (uint32_t)ncols, d_q, (uint32_t)nq, d_proof, (uint32_t)depth, d_out));
    const uint32_t *h = sc.download_later(d_out, 9);
    const std::vector<uint8_t> *rp = &root;
    sc.finalizers.push_back([h, rp]() {
        if (!(h[8] == 1 && rp->size() == 32 && std::memcmp(h, rp->data(), 32) == 0)) throw VerifyPanic{};
    });
}

std::vector<uint32_t> dense(const lg::Opening &o, size_t want_rows, size_t want_len) {
    if (o.rows.size() != want_rows) throw VerifyPanic{};  // assert_eq (src/sumcheck_polys.rs:98)
    std::vector<uint32_t> r(want_rows * want_len);
    for (size_t k = 0; k < want_rows; ++k) {
        if (o.rows.len(k) != want_len) throw VerifyPanic{};  // :97
        std::copy(o.rows.ptr(k), o.rows.ptr(k) + want_len, r.begin() + k * want_len);
    }
    return r;
}

// ligero_verify (src/ligero.rs:97-131); rows zip against gr (truncation)
void ligero_verify_host(const std::vector<uint64_t> &q, const lg::Opening &o, const std::vector<uint32_t> &yr,
                        const std::vector<uint32_t> &ch) {
    std::vector<uint32_t> gr = lg::lagrange_basis(ch.data(), ch.size());
    const size_t ylen = yr.size();
    if (ylen == 0 || (ylen & (ylen - 1))) throw VerifyPanic{};
    uint32_t nv = 0;
    while ((1ull << nv) < ylen) ++nv;
    std::vector<uint32_t> sks = lg::eval_sk_at_vks(ylen), basis(ylen), sx(nv + 1);
    if (o.rows.size() > q.size()) throw VerifyPanic{};
    for (size_t i = 0; i < o.rows.size(); ++i) {
        uint32_t dot = 0;
        const size_t zl = std::min(o.rows.len(i), gr.size());
        for (size_t j = 0; j < zl; ++j) dot ^= lg::gf_mul(o.rows.ptr(i)[j], gr[j]);
        if (q[i] > 0xFFFFFFFFull) throw VerifyPanic{};
        sx[0] = (uint32_t)q[i];
        for (uint32_t t = 1; t < nv; ++t) sx[t] = lg::next_s(sx[t - 1], sks[t - 1]);
        basis[0] = 1;
        for (uint32_t t = 0; t < nv; ++t) {
            const size_t cur = 1ull << t;
            for (size_t j = 0; j < cur; ++j) basis[cur + j] = lg::gf_mul(sx[t], basis[j]);
        }
        uint32_t e = 0;
        for (size_t j = 0; j < ylen; ++j) e ^= lg::gf_mul(yr[j], basis[j]);
        if (e != dot) throw VerifyPanic{};
    }
}

// The same check with the per-row work on the device: every panic that
// does not depend on the field values is decided on the host first, then
// one block per opened row compares <row, gr> with <yr, basis>.
void ligero_verify_dev(lg_ctx *c, Scratch &sc, const std::vector<uint64_t> &q, const lg::Opening &o,
                       const std::vector<uint32_t> &yr, const std::vector<uint32_t> &ch) {
    const size_t ylen = yr.size();
    if (ylen == 0 || (ylen & (ylen - 1))) throw VerifyPanic{};
    uint32_t nv = 0;
    while ((1ull << nv) < ylen) ++nv;
    if (nv > 31) return ligero_verify_host(q, o, yr, ch);
    const size_t nrows = o.rows.size();
    if (nrows > q.size()) throw VerifyPanic{};
    for (size_t i = 0; i < nrows; ++i)
        if (q[i] > 0xFFFFFFFFull) throw VerifyPanic{};
    if (nrows == 0) return;
    const std::vector<uint32_t> gr = lg::lagrange_basis(ch.data(), ch.size());
    const std::vector<uint32_t> sks = lg::eval_sk_at_vks(ylen);
    const uint32_t *d_rows = sc.upload(o.rows.data.data(), o.rows.data.size());
    const uint64_t *d_off = sc.upload(o.rows.off.data(), o.rows.off.size());
    const uint32_t *d_gr = sc.upload(gr.data(), gr.size());
    const uint32_t *d_yr = sc.upload(yr.data(), ylen);
    const uint64_t *d_q = sc.upload(q.data(), nrows);
    uint32_t *d_bad = static_cast<uint32_t *>(sc.dev(4));
    CK(c, cudaMemsetAsync(d_bad, 0, 4, c->stream));
    CK(c, lgk::ligero_check(c->L, d_rows, d_off, (uint32_t)nrows, d_gr, (uint32_t)gr.size(), d_yr, nv, d_q,
                            sks.data(), d_bad));
    const uint32_t *h = sc.download_later(d_bad, 1);
    sc.finalizers.push_back([h]() {
        if (*h != 0) throw VerifyPanic{};
    });
}

bool verify_impl(lg_ctx *c, Scratch &sc, const lg_config &cfg, const lg::Proof &P) {
    const size_t s = LG_NUM_QUERIES;
    const uint32_t log_inv_rate = 2;  // src/verifier.rs:26
    lg::Transcript fs(LG_FS_SEED);
    fs.absorb(P.initial_root.data(), P.initial_root.size());  // :27
    std::vector<uint32_t> pe0(cfg.initial_k);
    for (auto &r : pe0) r = fs.get_field();  // :29
    if (P.recursive_roots.empty()) throw VerifyPanic{};
    fs.absorb(P.recursive_roots[0].data(), P.recursive_roots[0].size());  // :30
    size_t depth = cfg.initial_log_m + log_inv_rate;
    std::vector<uint64_t> q;
    if (!fs.get_distinct_queries(1ull << depth, s, q)) throw VerifyPanic{};
    check_opening(c, sc, P.initial_root, P.initial, depth, q);  // :42-49
    const uint32_t alpha = fs.get_field();
    std::vector<uint32_t> rows = dense(P.initial, s, 1ull << cfg.initial_k);
    std::vector<DBuf> basis;
    std::vector<uint32_t> bvars, sep;
    basis.emplace_back(c, 4ull << cfg.initial_log_m);
    bvars.push_back(cfg.initial_log_m);
    sep.push_back(1);
    const uint32_t *h1 = induce_host_rows_later(c, sc, cfg.initial_log_m, rows.data(), s, pe0.data(),
                                                cfg.initial_k, q, alpha, basis.back().u32());  // :53-60
    // SumcheckVerifierInstance::new (src/ligerito.rs:172-192)
    size_t rd = 0;
    auto read_tr = [&]() {
        if (rd >= P.transcript.size()) throw VerifyPanic{};
        return P.transcript[rd++];
    };
    std::array<uint32_t, 3> g = read_tr();
    {
        const uint32_t e = g[0] ^ g[1];
        sc.finalizers.push_back([h1, e]() {
            if (*h1 != e) throw VerifyPanic{};
        });
    }
    Quad running = quad_from_evals(g[0], g[1], g[2]);
    absorb3(fs, g);  // :67
    std::vector<uint32_t> ris;
    for (uint32_t i = 0; i < cfg.recursive_steps; ++i) {
        std::vector<uint32_t> rs;
        for (uint32_t t = 0; t < cfg.ks[i]; ++t) {  // :70-76, fold :201-210
            const uint32_t r = fs.get_field();
            ris.push_back(r);
            const uint32_t sum = eval_quad(running, r);
            g = read_tr();
            if ((g[0] ^ g[1]) != sum) throw VerifyPanic{};
            running = quad_from_evals(g[0], g[1], g[2]);
            absorb3(fs, g);
            rs.push_back(r);
        }
        if (i >= P.recursive_roots.size()) throw VerifyPanic{};
        const std::vector<uint8_t> &root = P.recursive_roots[i];
        if (i == cfg.recursive_steps - 1) {  // :78-120
            fs.absorb_u32s(P.yr.data(), P.yr.size());
            depth = cfg.log_m[i] + log_inv_rate;
            if (!fs.get_distinct_queries(1ull << depth, s, q)) throw VerifyPanic{};
            check_opening(c, sc, root, P.final_, depth, q);
            ligero_verify_dev(c, sc, q, P.final_, P.yr, rs);
            const uint32_t final_r = fs.get_field();  // :114
            const size_t yl = P.yr.size();
            if (yl < 2) throw VerifyPanic{};
            std::vector<uint32_t> fe(yl / 2);
            for (size_t j = 0; j < yl / 2; ++j)
                fe[j] = P.yr[j] ^ lg::gf_mul(final_r, P.yr[j] ^ P.yr[yl / 2 + j]);
            // verify_partial (src/ligerito.rs:282-295)
            uint32_t k = 0;
            while ((1ull << k) < fe.size()) ++k;
            const uint32_t sum = eval_quad(running, final_r);
            ris.push_back(final_r);
            std::vector<uint32_t> acc(fe.size(), 0);
            std::vector<const uint32_t *> parts;
            for (size_t bi = 0; bi < basis.size(); ++bi) {  // evaluate_basis_polys_partially :257-280
                const uint32_t nv = bvars[bi];
                size_t npts, first;
                if (bi == 0) { npts = ris.size(); first = 0; }
                else {
                    if (nv < k || nv - k > ris.size()) throw VerifyPanic{};
                    npts = nv - k;
                    first = ris.size() - npts;
                }
                if (npts == 0 || npts > nv || (1ull << (nv - npts)) != fe.size()) throw VerifyPanic{};
                DBuf d(c, 4ull << (nv - npts));
                partial_eval_dev(c, basis[bi].u32(), nv, ris.data() + first, (uint32_t)npts, d.u32());
                parts.push_back(sc.download_later(d.u32(), fe.size()));
            }
            sc.finish();  // also decides the queued checks
            for (size_t bi = 0; bi < parts.size(); ++bi)
                for (size_t j = 0; j < acc.size(); ++j)
                    acc[j] ^= bi == 0 ? parts[bi][j] : lg::gf_mul(sep[bi], parts[bi][j]);
            uint32_t dot = 0;
            for (size_t j = 0; j < fe.size(); ++j) dot ^= lg::gf_mul(fe[j], acc[j]);
            return dot == sum;
        }
        if (i + 1 >= P.recursive_roots.size() || i >= P.recursive.size()) throw VerifyPanic{};
        fs.absorb(P.recursive_roots[i + 1].data(), P.recursive_roots[i + 1].size());  // :122
        depth = cfg.log_m[i] + log_inv_rate;
        if (!fs.get_distinct_queries(1ull << depth, s, q)) throw VerifyPanic{};  // :126
        check_opening(c, sc, root, P.recursive[i], depth, q);
        const uint32_t al = fs.get_field();  // :345
        std::vector<uint32_t> rr = dense(P.recursive[i], s, 1ull << cfg.ks[i]);
        basis.emplace_back(c, 4ull << cfg.log_m[i]);
        bvars.push_back(cfg.log_m[i]);
        const uint32_t *h = induce_host_rows_later(c, sc, cfg.log_m[i], rr.data(), s, rs.data(), cfg.ks[i], q, al,
                                                   basis.back().u32());
        g = read_tr();  // introduce_new (src/ligerito.rs:212-220)
        {
            const uint32_t e = g[0] ^ g[1];
            sc.finalizers.push_back([h, e]() {
                if (*h != e) throw VerifyPanic{};
            });
        }
        Quad to_glue = quad_from_evals(g[0], g[1], g[2]);
        absorb3(fs, g);
        const uint32_t beta = fs.get_field();  // :358
        sep.push_back(beta);                   // glue (src/ligerito.rs:222-232)
        running.a ^= lg::gf_mul(beta, to_glue.a);
        running.b ^= lg::gf_mul(beta, to_glue.b);
        running.c ^= lg::gf_mul(beta, to_glue.c);
    }
    throw VerifyPanic{};  // :362
}

template <class F>
lg_status guarded(lg_ctx *c, F &&f) {
    // A call that stops early may leave copies in flight into the context's
    // pinned and device arenas; the next call reuses those from the start,
    // so wait for both streams first (errors already reported are ignored).
    auto drain = [c]() {
        if (!c) return;
        cudaStreamSynchronize(c->stream);
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        cudaGetLastError();
    };
    try {
        f();
        return LG_OK;
    } catch (const CudaFail &) {
        drain();
        return LG_ERR_CUDA;
    } catch (const OutOfBudget &) {
        drain();
        return LG_ERR_OUT_OF_MEMORY;
    } catch (const ProverAssert &) {
        drain();
        if (c) c->err = "prover assertion failed";
        return LG_ERR_PROVER_ASSERT;
    } catch (const VerifyPanic &) {
        drain();
        if (c) c->err = "verifier panic";
        return LG_ERR_VERIFY_PANIC;
    } catch (const BadConfig &) {
        drain();
        return LG_ERR_INVALID_CONFIG;
    } catch (const std::bad_alloc &) {
        drain();
        if (c) c->err = "host allocation failed";
        return LG_ERR_OUT_OF_MEMORY;
    }
}

}  // namespace

// =================================================================== C ABI
extern "C" {

const char *lg_status_string(lg_status s) {
    switch (s) {
        case LG_OK: return "ok";
        case LG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case LG_ERR_INVALID_CONFIG: return "invalid config";
        case LG_ERR_OUT_OF_MEMORY: return "out of memory";
        case LG_ERR_CUDA: return "CUDA error";
        case LG_ERR_VERIFY_PANIC: return "verifier panic";
        case LG_ERR_PROVER_ASSERT: return "prover assertion failed";
        case LG_ERR_NO_DEVICE: return "no CUDA device";
        case LG_ERR_MALFORMED_PROOF: return "malformed proof";
        case LG_ERR_EXCEEDS_STATIC_SCRATCH: return "sizes exceed the fixed scratch of an allocation-free call";
        case LG_ERR_TIMEOUT: return "timed out";
    }
    return "unknown status";
}

uint32_t lg_abi_version(void) { return LG_ABI_VERSION; }

lg_status lg_hardcoded_config_20(lg_config *out) {
    if (!out) return LG_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->recursive_steps = 1;  // src/config.rs:19-28
    out->initial_log_m = 14;
    out->initial_log_n = 6;
    out->initial_k = 6;
    out->log_m[0] = 10;
    out->log_n[0] = 4;
    out->ks[0] = 4;
    return LG_OK;
}

lg_status lg_hardcoded_config_24(lg_config *out) {
    if (!out) return LG_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->recursive_steps = 2;  // src/config.rs:82-93
    out->initial_log_m = 18;
    out->initial_log_n = 6;
    out->initial_k = 6;
    out->log_m[0] = 14; out->log_n[0] = 4; out->ks[0] = 4;
    out->log_m[1] = 10; out->log_n[1] = 4; out->ks[1] = 4;
    return LG_OK;
}

lg_status lg_config_make(uint32_t L, lg_config *out) {
    if (!out || L < 16 || L > 30) return LG_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->initial_log_m = L - 6;
    out->initial_log_n = 6;
    out->initial_k = 6;
    uint32_t d = L - 6, s = 0;
    while (d - 4 >= 10 && s < LG_MAX_STEPS) {
        out->log_m[s] = d - 4; out->log_n[s] = 4; out->ks[s] = 4;
        ++s;
        d -= 4;
    }
    if (s == 0) { out->log_m[0] = L - 10; out->log_n[0] = 4; out->ks[0] = 4; s = 1; }
    out->recursive_steps = s;
    return LG_OK;
}

lg_status lg_config_validate(const lg_config *cfg, uint64_t poly_len) {
    if (!cfg) return LG_ERR_INVALID_ARGUMENT;
    return lg::config_check(*cfg, poly_len);
}

// Text form of a config (the fields of ProverConfig, src/config.rs:6-67),
// one "key = values" per line, '#' to the end of a line is a comment:
//   recursive_steps = 2
//   initial_dims = 262144 64     (rows, columns of the first matrix)
//   initial_k = 6
//   dims = 16384 16, 1024 16     (one "rows columns" pair per step)
//   ks = 4 4
// Every dimension is a power of two.
lg_status lg_config_parse(const char *text, lg_config *out) {
    if (!text || !out) return LG_ERR_INVALID_ARGUMENT;
    lg_config c{};
    bool seen[5] = {false, false, false, false, false};
    std::vector<uint64_t> dims;
    std::vector<uint64_t> ks;
    auto log2_exact = [](uint64_t v, uint32_t *lg) {
        if (v == 0 || (v & (v - 1))) return false;
        uint32_t l = 0;
        while ((1ull << l) < v) ++l;
        *lg = l;
        return true;
    };
    std::string all(text);
    size_t pos = 0;
    while (pos <= all.size()) {
        size_t eol = all.find('\n', pos);
        if (eol == std::string::npos) eol = all.size();
        std::string line = all.substr(pos, eol - pos);
        pos = eol + 1;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        const size_t eq = line.find('=');
        std::string key = line.substr(0, eq == std::string::npos ? line.size() : eq);
        key.erase(0, key.find_first_not_of(" \t\r"));
        key.erase(key.find_last_not_of(" \t\r") + 1);
        if (key.empty() && eq == std::string::npos) continue;  // blank line
        if (eq == std::string::npos) return LG_ERR_INVALID_CONFIG;
        std::vector<uint64_t> vals;
        std::string rest = line.substr(eq + 1);
        for (char &ch : rest)
            if (ch == ',') ch = ' ';
        const char *p = rest.c_str();
        while (*p) {
            while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
            if (!*p) break;
            if (*p < '0' || *p > '9') return LG_ERR_INVALID_CONFIG;
            char *end = nullptr;
            const unsigned long long v = std::strtoull(p, &end, 10);
            if (end == p) return LG_ERR_INVALID_CONFIG;
            vals.push_back(v);
            p = end;
        }
        const char *keys[5] = {"recursive_steps", "initial_dims", "initial_k", "dims", "ks"};
        int k = -1;
        for (int i = 0; i < 5; ++i)
            if (key == keys[i]) k = i;
        if (k < 0 || seen[k]) return LG_ERR_INVALID_CONFIG;
        seen[k] = true;
        if (k == 0 || k == 2) {
            if (vals.size() != 1 || vals[0] > 0xFFFFFFFFull) return LG_ERR_INVALID_CONFIG;
            (k == 0 ? c.recursive_steps : c.initial_k) = (uint32_t)vals[0];
        } else if (k == 1) {
            if (vals.size() != 2 || !log2_exact(vals[0], &c.initial_log_m) || !log2_exact(vals[1], &c.initial_log_n))
                return LG_ERR_INVALID_CONFIG;
        } else if (k == 3) {
            dims = vals;
        } else {
            ks = vals;
        }
    }
    for (bool b : seen)
        if (!b) return LG_ERR_INVALID_CONFIG;
    if (c.recursive_steps < 1 || c.recursive_steps > LG_MAX_STEPS || dims.size() != 2ull * c.recursive_steps ||
        ks.size() != c.recursive_steps)
        return LG_ERR_INVALID_CONFIG;
    for (uint32_t i = 0; i < c.recursive_steps; ++i) {
        if (!log2_exact(dims[2 * i], &c.log_m[i]) || !log2_exact(dims[2 * i + 1], &c.log_n[i]) ||
            ks[i] > 0xFFFFFFFFull)
            return LG_ERR_INVALID_CONFIG;
        c.ks[i] = (uint32_t)ks[i];
    }
    *out = c;
    return LG_OK;
}

lg_status lg_config_format(const lg_config *cfg, char *buf, uint64_t *len) {
    if (!cfg || !len || cfg->recursive_steps < 1 || cfg->recursive_steps > LG_MAX_STEPS || cfg->initial_log_m > 63 ||
        cfg->initial_log_n > 63)
        return LG_ERR_INVALID_ARGUMENT;
    std::string s = "recursive_steps = " + std::to_string(cfg->recursive_steps) + "\n";
    s += "initial_dims = " + std::to_string(1ull << cfg->initial_log_m) + " " +
         std::to_string(1ull << cfg->initial_log_n) + "\n";
    s += "initial_k = " + std::to_string(cfg->initial_k) + "\n";
    s += "dims =";
    for (uint32_t i = 0; i < cfg->recursive_steps; ++i) {
        if (cfg->log_m[i] > 63 || cfg->log_n[i] > 63) return LG_ERR_INVALID_ARGUMENT;
        s += (i ? ", " : " ") + std::to_string(1ull << cfg->log_m[i]) + " " + std::to_string(1ull << cfg->log_n[i]);
    }
    s += "\nks =";
    for (uint32_t i = 0; i < cfg->recursive_steps; ++i) s += " " + std::to_string(cfg->ks[i]);
    s += "\n";
    const uint64_t need = s.size() + 1;  // with the terminating NUL
    if (!buf || *len < need) {
        const bool ask = !buf;
        *len = need;
        return ask ? LG_OK : LG_ERR_INVALID_ARGUMENT;
    }
    std::memcpy(buf, s.c_str(), need);
    *len = need;
    return LG_OK;
}

lg_status lg_ctx_create(int device, uint64_t budget, lg_ctx **out) {
    if (!out) return LG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return LG_ERR_NO_DEVICE; }
    if (device < 0 || device >= n) return LG_ERR_INVALID_ARGUMENT;
    auto *c = new (std::nothrow) lg_ctx;
    if (!c) return LG_ERR_OUT_OF_MEMORY;
    c->device = device;
    c->budget = budget;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess) {
        delete c;
        return LG_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return LG_ERR_CUDA;
    }
    if (cudaMalloc((void **)&c->L.dtab, lgk::kDtabSlots * lgk::kDtabWords * 4) != cudaSuccess ||
        cudaMalloc((void **)&c->L.tickets, 256) != cudaSuccess || cudaMemset(c->L.tickets, 0, 256) != cudaSuccess) {
        cudaGetLastError();
        if (c->L.dtab) cudaFree(c->L.dtab);
        if (c->L.tickets) cudaFree(c->L.tickets);
        cudaStreamDestroy(c->copy_stream);
        cudaStreamDestroy(c->stream);
        delete c;
        return LG_ERR_OUT_OF_MEMORY;
    }
    for (auto &e : c->copy_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    c->L.stream = c->stream;
    c->L.device = device;
    {
        const char *e = std::getenv("LG_AUTOTUNE");
        c->L.autotune = e && e[0] == '1';
    }
    {
        std::lock_guard<std::mutex> lk(g_tables_mu);
        ++g_tables[device].contexts;
    }
    *out = c;
    return LG_OK;
}

void lg_ctx_destroy(lg_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    {
        std::lock_guard<std::mutex> lk(g_tables_mu);
        auto it = g_tables.find(c->device);
        if (it != g_tables.end() && --it->second.contexts <= 0) {
            for (auto &kv : it->second.codes) { cudaFree(kv.second.tw); cudaFree(kv.second.pis); }
            for (auto &kv : it->second.ffttw) cudaFree(kv.second);
            g_tables.erase(it);
        }
    }
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->pin_arena) cudaFreeHost(c->pin_arena);
    if (c->dev_arena) cudaFree(c->dev_arena);
    if (c->L.dtab) cudaFree(c->L.dtab);
    if (c->L.tickets) cudaFree(c->L.tickets);
    c->L.release();
    for (auto e : c->copy_ev) if (e) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    cudaStreamDestroy(c->stream);
    delete c;
}

const char *lg_ctx_last_error(const lg_ctx *c) { return c ? c->err.c_str() : "null context"; }
void *lg_ctx_stream(lg_ctx *c) { return c ? (void *)c->stream : nullptr; }
lg_status lg_ctx_synchronize(lg_ctx *c) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] { sync(c); });
}
uint64_t lg_ctx_launch_count(const lg_ctx *c) { return c ? c->L.launches : 0; }
lg_status lg_ctx_set_autotune(lg_ctx *c, int on) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    c->L.autotune = on != 0;
    return LG_OK;
}
lg_status lg_tuned_choices(char *buf, uint64_t *len) {
    if (!len) return LG_ERR_INVALID_ARGUMENT;
    const std::string s = lgk::tuned_choices();
    if (!buf) { *len = s.size() + 1; return LG_OK; }
    if (*len < s.size() + 1) { *len = s.size() + 1; return LG_ERR_INVALID_ARGUMENT; }
    std::memcpy(buf, s.c_str(), s.size() + 1);
    *len = s.size() + 1;
    return LG_OK;
}
lg_status lg_ctx_set_kernel_timing(lg_ctx *c, int on) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    c->L.timing = on != 0;
    return LG_OK;
}
lg_status lg_ctx_kernel_stats(lg_ctx *c, uint32_t index, char *name, size_t cap, uint64_t *launches, double *ms) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    lg_status st = guarded(c, [&] { sync(c); c->L.resolve(); });
    if (st != LG_OK) return st;
    if (index >= c->L.stats.size()) return LG_ERR_INVALID_ARGUMENT;
    auto it = c->L.stats.begin();
    std::advance(it, index);
    if (name && cap) { std::snprintf(name, cap, "%s", it->first.c_str()); }
    if (launches) *launches = it->second.first;
    if (ms) *ms = it->second.second;
    return LG_OK;
}
lg_status lg_ctx_kernel_work(lg_ctx *c, uint32_t index, double *bytes, double *mults, double *comps) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    lg_status st = guarded(c, [&] { sync(c); c->L.resolve(); });
    if (st != LG_OK) return st;
    if (index >= c->L.stats.size()) return LG_ERR_INVALID_ARGUMENT;
    auto it = c->L.stats.begin();
    std::advance(it, index);
    const auto w = c->L.work.find(it->first);
    const lgk::Launcher::Work none{};
    const lgk::Launcher::Work &x = w == c->L.work.end() ? none : w->second;
    if (bytes) *bytes = x.bytes;
    if (mults) *mults = x.mults;
    if (comps) *comps = x.comps;
    return LG_OK;
}
lg_status lg_ctx_reset_kernel_stats(lg_ctx *c) {
    if (!c) return LG_ERR_INVALID_ARGUMENT;
    lg_status st = guarded(c, [&] { sync(c); c->L.resolve(); });
    c->L.stats.clear();
    c->L.work.clear();
    return st;
}
uint64_t lg_ctx_device_bytes_in_use(const lg_ctx *c) { return c ? c->in_use : 0; }
uint64_t lg_ctx_device_bytes_cached(const lg_ctx *c) {
    return c ? lgk::kDtabSlots * lgk::kDtabWords * 4 + Scratch::kDevArena : 0;
}
uint64_t lg_device_table_bytes(int device) {
    std::lock_guard<std::mutex> lk(g_tables_mu);
    auto it = g_tables.find(device);
    return it == g_tables.end() ? 0 : it->second.bytes;
}

lg_status lg_prove(lg_ctx *c, const lg_config *cfg, const uint32_t *poly, uint64_t len, int on_device,
                   lg_proof **out) {
    if (!c || !cfg || !poly || !out) return LG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    lg_status st = lg::config_check(*cfg, len);
    if (st != LG_OK) return st;
    auto *res = new (std::nothrow) lg_proof;
    if (!res) return LG_ERR_OUT_OF_MEMORY;
    st = guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        Scratch sc(c);
        if (on_device) {
            prove_impl(c, sc, *cfg, poly, len, res->p);
        } else {
            DBuf d(c, len * 4);
            prove_impl(c, sc, *cfg, d.u32(), len, res->p, poly);
        }
        sc.finish();
    });
    if (st != LG_OK) { delete res; return st; }
    *out = res;
    return LG_OK;
}

lg_status lg_dump_intermediates(lg_ctx *c, const lg_config *cfg, const uint32_t *poly, uint64_t len, int on_device,
                                lg_dump_cb cb, void *user, lg_proof **out) {
    if (!c || !cb) return LG_ERR_INVALID_ARGUMENT;
    struct Hook {  // cleared however lg_prove returns
        lg_ctx *c;
        ~Hook() { c->dump_cb = nullptr; c->dump_user = nullptr; }
    } hook{c};
    c->dump_cb = cb;
    c->dump_user = user;
    return lg_prove(c, cfg, poly, len, on_device, out);
}

lg_status lg_prove_lockstep(lg_ctx *c, const lg_config *cfg, const uint32_t *const *polys, uint64_t len,
                            uint32_t count, int on_device, lg_proof **out) {
    if (!c || !cfg || !polys || !out) return LG_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) {
        out[i] = nullptr;
        if (!polys[i]) return LG_ERR_INVALID_ARGUMENT;
    }
    lg_status st = lg::config_check(*cfg, len);
    if (st != LG_OK) return st;
    lg_status first = LG_OK;
    for (uint32_t s0 = 0; s0 < count; s0 += lgk::kMaxTickets) {
        const uint32_t B = std::min<uint32_t>(lgk::kMaxTickets, count - s0);
        std::vector<lg_proof *> res(B, nullptr);
        std::vector<char> bad;
        for (auto &r : res) {
            r = new (std::nothrow) lg_proof;
            if (!r) {
                for (auto *x : res) delete x;
                return first != LG_OK ? first : LG_ERR_OUT_OF_MEMORY;
            }
        }
        st = guarded(c, [&] {
            CK(c, cudaSetDevice(c->device));
            Scratch sc(c);
            if (B == 1) {  // alone, the single-proof path is faster
                bad.assign(1, 0);
                if (on_device) prove_impl(c, sc, *cfg, polys[s0], len, res[0]->p);
                else {
                    DBuf one(c, len * 4);
                    prove_impl(c, sc, *cfg, one.u32(), len, res[0]->p, polys[s0]);
                }
                sc.finish();
                return;
            }
            // the inputs as one contiguous run, copied together unless
            // they already are
            bool contiguous = on_device != 0;
            for (uint32_t b = 1; b < B && contiguous; ++b) contiguous = polys[s0 + b] == polys[s0] + b * len;
            DBuf in;
            const uint32_t *d = polys[s0];
            if (!contiguous) {
                in = DBuf(c, 4 * len * B);
                for (uint32_t b = 0; b < B; ++b)
                    CK(c, cudaMemcpyAsync(in.u32() + b * len, polys[s0 + b], 4 * len,
                                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
                d = in.u32();
            }
            std::vector<lg::Proof *> P(B);
            for (uint32_t b = 0; b < B; ++b) P[b] = &res[b]->p;
            prove_batch_impl(c, sc, *cfg, d, len, B, P, bad);
            sc.finish();
        });
        for (uint32_t b = 0; b < B; ++b) {
            if (st == LG_OK && !bad[b]) {
                out[s0 + b] = res[b];
            } else {
                delete res[b];
                if (st == LG_OK) {
                    c->err = "prover assertion failed";
                    if (first == LG_OK) first = LG_ERR_PROVER_ASSERT;
                }
            }
        }
        if (st != LG_OK && first == LG_OK) first = st;
    }
    return first;
}

lg_status lg_verify(lg_ctx *c, const lg_config *cfg, const lg_proof *proof, int *accepted) {
    if (!c || !cfg || !proof || !accepted) return LG_ERR_INVALID_ARGUMENT;
    *accepted = 0;
    if (cfg->recursive_steps < 1 || cfg->recursive_steps > LG_MAX_STEPS || cfg->initial_k > 8 ||
        cfg->initial_log_m > 26)
        return LG_ERR_INVALID_CONFIG;
    for (uint32_t i = 0; i < cfg->recursive_steps; ++i)
        if (cfg->ks[i] > 8 || cfg->log_m[i] > 26) return LG_ERR_INVALID_CONFIG;
    bool ok = false;
    lg_status st = guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        Scratch sc(c);
        ok = verify_impl(c, sc, *cfg, proof->p);
        sc.finish();
    });
    if (st == LG_OK) *accepted = ok ? 1 : 0;
    return st;
}

lg_status lg_proof_serialize(const lg_proof *p, uint8_t *buf, uint64_t *len) {
    if (!p || !len) return LG_ERR_INVALID_ARGUMENT;
    const size_t need = lg::serialized_size(p->p);
    if (!buf || *len < need) {
        const bool ask = !buf;
        *len = need;
        return ask ? LG_OK : LG_ERR_INVALID_ARGUMENT;
    }
    std::vector<uint8_t> b = lg::serialize(p->p);
    std::memcpy(buf, b.data(), b.size());
    *len = b.size();
    return LG_OK;
}

lg_status lg_verify_bytes(lg_ctx *c, const lg_config *cfg, const uint8_t *proof, uint64_t len, int *accepted) {
    if (!c || !cfg || !proof || !accepted) return LG_ERR_INVALID_ARGUMENT;
    *accepted = 0;
    lg_proof p;
    if (!lg::deserialize(proof, len, p.p)) return LG_ERR_MALFORMED_PROOF;
    return lg_verify(c, cfg, &p, accepted);
}
lg_status lg_proof_deserialize(const uint8_t *buf, uint64_t len, lg_proof **out) {
    if (!buf || !out) return LG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto *p = new (std::nothrow) lg_proof;
    if (!p) return LG_ERR_OUT_OF_MEMORY;
    if (!lg::deserialize(buf, len, p->p)) { delete p; return LG_ERR_MALFORMED_PROOF; }
    *out = p;
    return LG_OK;
}

void lg_proof_free(lg_proof *p) { delete p; }

lg_status lg_proof_size(const lg_proof *p, uint64_t *bytes) {
    if (!p || !bytes) return LG_ERR_INVALID_ARGUMENT;
    *bytes = lg::proof_size(p->p);
    return LG_OK;
}

lg_status lg_compute_twiddles(uint32_t log_n, uint32_t *out) {
    if (!out || log_n < 1 || log_n > 30) return LG_ERR_INVALID_ARGUMENT;
    lg::compute_twiddles(log_n, out);
    return LG_OK;
}

static lg_status fft_common(lg_ctx *c, uint32_t *d, uint32_t log_n, uint64_t batch, bool inv) {
    if (!c || !d || log_n < 1 || log_n > 30 || batch == 0 || batch > 0xFFFFFFFFull) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        const uint32_t *tw = get_fft_tw(c, log_n);
        CK(c, lgk::fft_vectors(c->L, d, tw, log_n, (uint32_t)batch, 1ull << log_n, 1, 0, 1, inv));
        sync(c);
    });
}
lg_status lg_fft(lg_ctx *c, uint32_t *d, uint32_t log_n, uint64_t batch) { return fft_common(c, d, log_n, batch, false); }
lg_status lg_ifft(lg_ctx *c, uint32_t *d, uint32_t log_n, uint64_t batch) { return fft_common(c, d, log_n, batch, true); }

lg_status lg_rs_encode_cols(lg_ctx *c, const uint32_t *d_poly, uint32_t log_m, uint32_t n, uint32_t *d_enc) {
    if (!c || !d_poly || !d_enc || log_m < 1 || log_m > 26 || n == 0) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        const Code code = get_code(c, log_m);
        DBuf scaled(c, log_m > 6 ? 4ull * n << log_m : 0);
        rs_encode(c, code, d_poly, log_m, n, d_enc, 4ull << log_m, scaled.u32());
        sync(c);
    });
}

lg_status lg_ligero_commit(lg_ctx *c, const uint32_t *d_poly, uint32_t log_m, uint32_t n, uint32_t *d_enc,
                           uint8_t *d_tree, uint8_t *root) {
    if (!c || !d_poly || !d_enc || !d_tree || log_m < 1 || log_m > 26 || n == 0 || n > 256)
        return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        commit_into(c, d_poly, log_m, n, d_enc, reinterpret_cast<uint32_t *>(d_tree));
        const uint64_t rows = 4ull << log_m;
        if (root) d2h(c, root, d_tree + 32 * (2 * rows - 2), 32);
        sync(c);
    });
}

lg_status lg_partial_eval(lg_ctx *c, const uint32_t *d_evals, uint32_t log_len, const uint32_t *rs, uint32_t k,
                          uint32_t *d_out) {
    if (!c || !d_evals || !rs || !d_out || k == 0 || k > log_len || log_len > 34) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        partial_eval_dev(c, d_evals, log_len, rs, k, d_out);
        sync(c);
    });
}

lg_status lg_eval_013_product(lg_ctx *c, const uint32_t *d_f, const uint32_t *d_g, uint32_t log_len, uint32_t out[3]) {
    if (!c || !d_f || !d_g || !out || log_len < 1 || log_len > 34) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        DBuf acc(c, 16);
        CK(c, cudaMemsetAsync(acc.p, 0, 12, c->stream));
        CK(c, lgk::eval013(c->L, d_f, d_g, log_len, acc.u32()));
        d2h(c, out, acc.p, 12);
    });
}

lg_status lg_induce_sumcheck_poly(lg_ctx *c, uint32_t n, const uint32_t *rows, uint32_t nrows, const uint32_t *vch,
                                  uint32_t nch, const uint64_t *queries, uint32_t alpha, uint32_t *d_out,
                                  uint32_t *enforced_sum) {
    if (!c || !rows || !vch || !queries || !d_out || !enforced_sum || nch == 0 || nch > 8 || n > 28 || nrows == 0)
        return LG_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < nrows; ++k)
        if (queries[k] > 0xFFFFFFFFull) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        std::vector<uint64_t> q(queries, queries + nrows);
        Scratch sc(c);
        *enforced_sum = induce_host_rows(c, sc, n, rows, nrows, vch, nch, q, alpha, d_out);
        sc.finish();
    });
}

struct lg_transcript {
    lg::Transcript t;
    explicit lg_transcript(uint32_t seed) : t(seed) {}
};

lg_status lg_transcript_new(uint32_t seed, lg_transcript **out) {
    if (!out) return LG_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) lg_transcript(seed);
    return *out ? LG_OK : LG_ERR_OUT_OF_MEMORY;
}
void lg_transcript_free(lg_transcript *t) { delete t; }
lg_status lg_transcript_absorb(lg_transcript *t, const uint8_t *b, uint64_t len) {
    if (!t || (!b && len)) return LG_ERR_INVALID_ARGUMENT;
    t->t.absorb(b, len);
    return LG_OK;
}
lg_status lg_transcript_squeeze(lg_transcript *t, uint64_t out[2]) {
    if (!t || !out) return LG_ERR_INVALID_ARGUMENT;
    auto v = t->t.squeeze();
    out[0] = v[0];
    out[1] = v[1];
    return LG_OK;
}
lg_status lg_transcript_get_field(lg_transcript *t, uint32_t *out) {
    if (!t || !out) return LG_ERR_INVALID_ARGUMENT;
    *out = t->t.get_field();
    return LG_OK;
}
lg_status lg_transcript_get_query(lg_transcript *t, uint64_t n, uint64_t *out) {
    if (!t || !out || n == 0) return LG_ERR_INVALID_ARGUMENT;
    *out = t->t.get_query(n);
    return LG_OK;
}
lg_status lg_transcript_get_distinct_queries(lg_transcript *t, uint64_t n, uint64_t s, uint64_t *out) {
    if (!t || (!out && s)) return LG_ERR_INVALID_ARGUMENT;
    std::vector<uint64_t> q;
    if (!t->t.get_distinct_queries(n, s, q)) return LG_ERR_INVALID_ARGUMENT;
    std::copy(q.begin(), q.end(), out);
    return LG_OK;
}

lg_status lg_merkle_verify(const uint8_t *root, const uint8_t *proof, uint64_t n_sib, uint64_t depth,
                           const uint8_t *leaves, const uint64_t *off, const uint64_t *queries, uint64_t nq,
                           int *ok) {
    if (!root || !ok || (!proof && n_sib) || (nq && (!leaves || !off || !queries)) || depth > 64)
        return LG_ERR_INVALID_ARGUMENT;
    std::vector<std::array<uint8_t, 32>> layer(nq);
    for (uint64_t i = 0; i < nq; ++i) lg::blake3_hash(leaves + off[i], off[i + 1] - off[i], layer[i].data());
    lg::ByteList sib;
    sib.assign_fixed(proof, n_sib, 32);
    bool good = false;
    if (!lg::merkle_verify(root, 32, sib, depth, layer, std::vector<uint64_t>(queries, queries + nq), &good)) {
        *ok = 0;
        return LG_ERR_VERIFY_PANIC;
    }
    *ok = good ? 1 : 0;
    return LG_OK;
}

lg_status lg_fill_splitmix(lg_ctx *c, uint64_t seed, uint32_t *d_out, uint64_t n) {
    if (!c || !d_out) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        CK(c, lgk::splitmix(c->L, seed, d_out, n));
        sync(c);
    });
}

lg_status lg_gf128_mul(lg_ctx *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, uint64_t n) {
    if (!c || (n && (!d_a || !d_b || !d_out))) return LG_ERR_INVALID_ARGUMENT;
    if ((uintptr_t)d_a % 16 || (uintptr_t)d_b % 16 || (uintptr_t)d_out % 16) return LG_ERR_INVALID_ARGUMENT;
    return guarded(c, [&] {
        CK(c, cudaSetDevice(c->device));
        CK(c, lgk::gf128_mul(c->L, d_a, d_b, d_out, n));
        sync(c);
    });
}

void lg_fill_splitmix_host(uint64_t seed, uint32_t *out, uint64_t n) {
    if (out) lg::splitmix_fill(seed, out, n, 0);
}

}  // extern "C"
