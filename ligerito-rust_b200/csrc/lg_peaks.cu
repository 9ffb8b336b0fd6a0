// Integer-pipe and shared-memory peak rates of the current device, measured
// by throughput microkernels.  They are the denominators of the integer
// rooflines: the hot kernels of this library are bound by integer logic
// (GF(2^32) table products, BLAKE3) and shared-memory table lookups, not by
// HBM, and no vendor figure for those rates exists for this part.
//
// Each kernel runs 8 independent dependency chains per thread (enough to
// hide the pipes' latency at full occupancy) of one instruction kind,
// written as inline PTX with runtime operands so that nothing folds.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ligerito_b200.h"

namespace {

constexpr int kIters = 2048;  // loop trips per thread, 8 chains x 4 ops each

template <int KIND>
__device__ __forceinline__ void step(uint32_t (&x)[8], uint32_t m) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t y = x[(i + 1) & 7], z = x[(i + 3) & 7];
        if (KIND == LG_PIPE_LOP3) {
            asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[i]) : "r"(y), "r"(z));
        } else if (KIND == LG_PIPE_IADD) {
            asm volatile("add.u32 %0, %0, %1;" : "+r"(x[i]) : "r"(y));
        } else if (KIND == LG_PIPE_PRMT) {
            asm volatile("prmt.b32 %0, %0, %1, 0x6521;" : "+r"(x[i]) : "r"(y));
        } else if (KIND == LG_PIPE_SHF) {
            asm volatile("shf.r.wrap.b32 %0, %0, %1, 7;" : "+r"(x[i]) : "r"(y));
        } else if (KIND == LG_PIPE_IMAD) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(y));
        } else if (KIND == LG_PIPE_IMAD_HI) {
            asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(y));
        } else if (KIND == LG_PIPE_LOP3_IMAD) {  // one of each per chain step
            asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;\n\tmad.lo.u32 %0, %0, %3, %1;"
                         : "+r"(x[i]) : "r"(y), "r"(z), "r"(m));
        }
    }
}

// ops issued per chain step, for the rate
__host__ __device__ constexpr int ops_per_step(int kind) {
    return kind == LG_PIPE_LOP3_IMAD ? 2 : 1;
}

template <int KIND>
__global__ void __launch_bounds__(256) k_pipe(uint32_t m, uint32_t *out) {
    uint32_t x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 0x9E3779B9u + i * 0x85EBCA6Bu + blockIdx.x;
#pragma unroll 1
    for (int it = 0; it < kIters; ++it) {
        step<KIND>(x, m);
        step<KIND>(x, m);
        step<KIND>(x, m);
        step<KIND>(x, m);
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r ^= x[i];
    if (r == 0x12345678u) out[0] = r;  // keeps the chains live
}

// Conflict-free shared-memory loads: every lane of a warp reads a distinct
// bank of one row, 8 independent chains whose addresses depend on the
// previous value (like a table lookup).  Rate = warp-level loads, i.e.
// shared-memory wavefronts.
__global__ void __launch_bounds__(256) k_lds(uint32_t m, uint32_t *out) {
    __shared__ uint32_t tab[8][32];
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) tab[i >> 5][i & 31] = i & 31;  // entry = its own bank
    __syncthreads();
    uint32_t x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = lane;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(&tab[0][0]);
#pragma unroll 1
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                // x stays the lane's bank; m == 0 at run time, so the row stays i
                asm volatile("ld.shared.u32 %0, [%1];" : "=r"(x[i]) : "r"(base + 128u * (uint32_t)i + 4u * (x[i] ^ m)));
            }
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r += x[i];
    if (r == 0x12345678u) out[0] = r;
}

template <class K>
float time_kernel(K kernel, int blocks, uint32_t m, uint32_t *out, cudaEvent_t a, cudaEvent_t b) {
    kernel<<<blocks, 256>>>(m, out);  // warm-up
    cudaEventRecord(a);
    kernel<<<blocks, 256>>>(m, out);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace

extern "C" lg_status lg_measure_pipe_peaks(int device, double *rates, uint32_t count) {
    if (!rates || count == 0) return LG_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return LG_ERR_NO_DEVICE;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return LG_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8;  // 2048 resident threads per SM
    uint32_t *out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    lg_status st = LG_OK;
    if (cudaMalloc(&out, 16) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
        cudaEventCreate(&b) != cudaSuccess) {
        st = LG_ERR_CUDA;
    } else {
        const double lane_steps = (double)blocks * 256 * kIters * 4 * 8;  // chain steps over all lanes
        for (uint32_t k = 0; k < count && k < LG_PIPE_COUNT; ++k) {
            float ms = 0.f;
            switch (k) {
                case LG_PIPE_LOP3: ms = time_kernel(k_pipe<LG_PIPE_LOP3>, blocks, 3u, out, a, b); break;
                case LG_PIPE_IADD: ms = time_kernel(k_pipe<LG_PIPE_IADD>, blocks, 3u, out, a, b); break;
                case LG_PIPE_PRMT: ms = time_kernel(k_pipe<LG_PIPE_PRMT>, blocks, 3u, out, a, b); break;
                case LG_PIPE_SHF: ms = time_kernel(k_pipe<LG_PIPE_SHF>, blocks, 3u, out, a, b); break;
                case LG_PIPE_IMAD: ms = time_kernel(k_pipe<LG_PIPE_IMAD>, blocks, 3u, out, a, b); break;
                case LG_PIPE_IMAD_HI: ms = time_kernel(k_pipe<LG_PIPE_IMAD_HI>, blocks, 3u, out, a, b); break;
                case LG_PIPE_LOP3_IMAD: ms = time_kernel(k_pipe<LG_PIPE_LOP3_IMAD>, blocks, 3u, out, a, b); break;
                case LG_PIPE_LDS: ms = time_kernel(k_lds, blocks, 0u, out, a, b); break;
            }
            const double ops = k == LG_PIPE_LDS ? lane_steps / 32.0 : lane_steps * ops_per_step((int)k);
            rates[k] = ms > 0.f ? ops / (ms * 1e-3) : 0.0;
        }
        if (cudaGetLastError() != cudaSuccess) st = LG_ERR_CUDA;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (out) cudaFree(out);
    cudaSetDevice(prev);
    return st;
}
