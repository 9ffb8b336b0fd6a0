// lg_induce_sumcheck_poly_noalloc: the induced sumcheck basis without any
// device allocation, for callers that cannot allocate device memory.
//
// Who needs this: a caller whose device memory is entirely owned by another
// allocator (a host framework that reserves the GPU's memory up front and
// hands out slices of it), or a latency-critical path that must not call
// cudaMalloc / cudaFree because those can synchronise the whole device.
// Such a caller can pass its own input and output buffers, but the regular
// entry point also needs scratch space (per-query subspace values, alpha
// powers and the two expansion tables of the basis), which it takes from a
// context that allocates.  Here that scratch is one fixed array in device
// memory.  It sits in this file's own code module, which the CUDA runtime
// loads lazily: the first call on a device loads the module, reserving the
// array on that device (a driver allocation), and every GPU that has loaded
// it keeps it until the process exits.  Callers make one warm-up call per
// device at start-up; later calls allocate nothing.
//
// Queries are read as 32-bit row indices on the device (the regular entry
// point rejects larger values on the host; here they stay on the device,
// so values of 2^32 and more give undefined results).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/ligerito_b200.h"
#include "lg_host.h"
#include "lg_kernels.h"

namespace {

constexpr uint32_t kScratchWords = LG_NOALLOC_SCRATCH_BYTES / 4;

// The scratch itself.  Host code must not pass its name to a kernel (on the
// host it only stands in for the symbol); it takes the device address from
// cudaGetSymbolAddress once per device.
static __device__ __align__(256) uint32_t g_induce_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
uint32_t *g_scratch_ptr[kMaxDevices];
cudaError_t g_scratch_err[kMaxDevices];

// First use on a device, with that device current: resolve the array's
// device address.  This happens inside the first call on each device, so
// that call should come before any stream capture.
uint32_t *scratch_for_current_device(cudaError_t *err) {
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= kMaxDevices) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::call_once(g_once[dev], [dev] {
        void *p = nullptr;
        g_scratch_err[dev] = cudaGetSymbolAddress(&p, g_induce_scratch);
        g_scratch_ptr[dev] = static_cast<uint32_t *>(p);
    });
    *err = g_scratch_err[dev];
    return *err == cudaSuccess ? g_scratch_ptr[dev] : nullptr;
}

uint64_t round256(uint64_t words) { return (words + 63) & ~uint64_t(63); }

}  // namespace

extern "C" lg_status lg_induce_sumcheck_poly_noalloc(void *stream, uint32_t n, const uint32_t *d_rows,
                                                     uint32_t nrows, const uint32_t *v_challenges, uint32_t nch,
                                                     const uint64_t *d_queries, uint32_t alpha,
                                                     uint32_t *d_basis_out, uint32_t *d_enforced_sum) {
    if (!d_rows || !v_challenges || !d_queries || !d_basis_out || !d_enforced_sum || nch == 0 || nch > 8 ||
        nrows == 0 || n > 28)
        return LG_ERR_INVALID_ARGUMENT;
    const lgk::InducePlan plan = lgk::induce_plan(n, nrows);
    const uint64_t w_S = round256((uint64_t)nrows * (n ? n : 1));
    const uint64_t w_apow = round256(2ull * nrows);
    const uint64_t w_lo = round256((uint64_t)nrows << plan.b);
    const uint64_t w_hi = round256((uint64_t)nrows << (n - plan.b));
    if (nrows > 256 || n > 20 || w_S + w_apow + w_lo + w_hi > kScratchWords) return LG_ERR_EXCEEDS_STATIC_SCRATCH;

    cudaError_t err;
    uint32_t *scratch = scratch_for_current_device(&err);
    if (!scratch) return LG_ERR_CUDA;
    uint32_t *d_S = scratch, *d_apow = d_S + w_S, *d_lo = d_apow + w_apow, *d_hi = d_lo + w_lo;

    // Lagrange basis of the challenges and s_k(v_k) on the stack: nothing
    // here allocates, on the device or the host.
    uint32_t gr[256], tmp[256], sks[32], layer[32];
    gr[0] = 1u ^ v_challenges[0];
    gr[1] = v_challenges[0];
    for (uint32_t i = 1, len = 2; i < nch; ++i, len *= 2) {
        const uint32_t r = v_challenges[i], rp1 = 1u ^ r;
        for (uint32_t j = 0; j < len; ++j) {
            tmp[2 * j] = lg::gf_mul(gr[j], rp1);
            tmp[2 * j + 1] = lg::gf_mul(gr[j], r);
        }
        for (uint32_t j = 0; j < 2 * len; ++j) gr[j] = tmp[j];
    }
    sks[0] = 1;
    for (uint32_t i = 1; i <= n; ++i) layer[i - 1] = 1u << i;
    for (uint32_t i = 1, cur = n; i <= n; ++i, --cur) {
        for (uint32_t j = 1; j <= cur; ++j) {
            if (j == 1) sks[i] = lg::gf_mul(layer[0], layer[0]) ^ lg::gf_mul(sks[i - 1], layer[0]);
            else layer[j - 2] = lg::gf_mul(layer[j - 1], layer[j - 1]) ^ lg::gf_mul(sks[i - 1], layer[j - 1]);
        }
    }

    lgk::Launcher L;
    L.stream = static_cast<cudaStream_t>(stream);
    err = lgk::induce_setup(L, d_rows, 1u << nch, gr, d_queries, nrows, alpha, n, sks, d_S, d_apow);
    // The output is accumulated across query groups when the plan splits
    // them, so it must start at zero; the scratch regions are fully written
    // before they are read and need no clearing.
    if (err == cudaSuccess && plan.needs_zero) err = cudaMemsetAsync(d_basis_out, 0, 4ull << n, L.stream);
    if (err == cudaSuccess)
        err = lgk::induce_basis(L, plan, d_S, d_apow, n, nrows, d_lo, d_hi, d_basis_out, d_enforced_sum);
    return err == cudaSuccess ? LG_OK : LG_ERR_CUDA;
}
