// prism_residual_norms_noalloc: true residual norms ||b_c - A x_c||_2 and
// ||b_c||_2 for k right-hand sides, computed without allocating anything.
//
// Who needs it.  Every other device entry point of this library works out of
// buffers that a handle allocates with cudaMalloc.  Some callers cannot let a
// library do that: a host framework that has already handed all device memory
// to its own pool allocator (cudaMalloc would fail or fight the pool), a
// process running at the edge of device memory that still has to check its
// solution, or an inner loop on a latency-sensitive stream, where
// cudaMalloc/cudaFree would synchronize the device and stall every other
// stream.  For them this entry point takes only caller-owned device pointers
// and keeps its reduction scratch in one statically sized __device__ array of
// this file, so no call allocates host or device memory.
//
// The scratch.  g_noalloc_scratch holds, per device, the block partials of a
// deterministic "last block finishes" reduction (kNaBlocks blocks x 2 values
// for each of at most kNaMaxCols columns: 151,552 bytes) followed by one
// ticket word in its own 256-byte slot.  The partials need no initial value;
// the ticket must be zero when a launch starts, so every call clears it with
// a 4-byte cudaMemsetAsync on its stream before the launch (a memset, not an
// allocation), whatever an earlier, possibly failed, launch left there; the
// last block of every completed launch also sets it back to zero.  Because
// the scratch is one array per device, two calls on the same device that may
// run at the same time (different streams with no ordering between them, or
// different host threads) race on it and give wrong results: order such calls
// on one stream or with events.
//
// On success a call allocates nothing, host or device.  A failing call
// formats its message in a stack buffer and stores it for prism_last_error(),
// which may take host memory for the text.
//
// Set-up.  The first call on a device, with that device current, resolves the
// scratch address once with cudaGetSymbolAddress (under a mutex) and caches it
// in an atomic per-device slot; later calls read the slot without taking the
// mutex.  Make that first call before any stream capture begins on the
// calling thread.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/prism_solve.h"
#include "device_common.cuh"

namespace prism {
// Stores msg as the calling thread's prism_last_error() text (cleared for
// PRISM_OK) and returns status; defined in capi.cu.
int record_error(int status, const char* msg);
}

namespace {

constexpr int kNaThreads = 256;                  // threads per block
constexpr int kNaG = 8;                          // lanes per CSR row (same row split as the SpMV)
constexpr int kNaBlocks = 592;                   // at most 148 SMs x 4 blocks
constexpr int kNaMaxCols = 16;                   // right-hand sides per call
constexpr int kNaVals = 2 * kNaMaxCols;          // per block: (sum r^2, sum b^2) per column
constexpr int kNaPartialDoubles = kNaBlocks * kNaVals;
constexpr int kNaTicketDoubles = 32;             // 256-byte slot for the ticket word
constexpr int kNaMaxDevices = 64;

static_assert((kNaPartialDoubles * sizeof(double)) % 256 == 0, "ticket slot must stay 256-byte aligned");

// 151,808 bytes per device: partials, then the ticket (first 4 bytes of the last slot).
static __device__ __align__(256) double g_noalloc_scratch[kNaPartialDoubles + kNaTicketDoubles];

int na_fail(int status, const char* fmt, unsigned long long a = 0, unsigned long long b = 0) {
    char msg[256];
    std::snprintf(msg, sizeof msg, fmt, a, b);
    return prism::record_error(status, msg);
}

int na_cuda_fail(const char* what, cudaError_t e) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "prism_residual_norms_noalloc: %s: %s", what, cudaGetErrorString(e));
    return prism::record_error(PRISM_ERR_CUDA, msg);
}

std::mutex g_setup_mu;
std::atomic<void*> g_scratch_ptr[kNaMaxDevices] = {};

// The scratch address on `device`, which the caller has made current; resolved
// once per device (the only call that takes the mutex), then read lock-free.
int scratch_for(int device, double** out) {
    void* p = g_scratch_ptr[device].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        p = g_scratch_ptr[device].load(std::memory_order_relaxed);
        if (!p) {
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return na_cuda_fail("cudaGetSymbolAddress of the scratch", e);
            g_scratch_ptr[device].store(p, std::memory_order_release);
        }
    }
    *out = static_cast<double*>(p);
    return PRISM_OK;
}

template <int NV>
__device__ __forceinline__ void na_block_sum(double (&v)[NV], double* smem /* [NV * 32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) smem[q * 32 + wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = lane < nw ? smem[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[q] = s;  // valid in warp 0
        }
    }
    __syncthreads();
}

// r_c = b_c - A x_c row by row (kNaG lanes per row, the row's nonzeros read
// once for all k columns), sums of r^2 and b^2 per column reduced in a fixed
// order: the same grid gives bitwise identical norms run after run.
__global__ void __launch_bounds__(kNaThreads) k_residual_norms_noalloc(
    uint32_t n, const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b, uint32_t k,
    uint64_t ld, double* __restrict__ partial, unsigned* __restrict__ ticket, double* __restrict__ norms) {
    __shared__ double smem[kNaVals * 32];
    __shared__ bool last;
    const int lane = threadIdx.x & (kNaG - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / kNaG;
    const uint32_t gid = (blockIdx.x * blockDim.x + threadIdx.x) / kNaG;
    const uint32_t sub = (threadIdx.x & 31) / kNaG;
    double acc[kNaVals];
#pragma unroll
    for (int q = 0; q < kNaVals; ++q) acc[q] = 0.0;
    // warp-uniform trip count: the full-mask shuffles below see all 32 lanes; 64-bit
    // so that the stride cannot wrap past 2^32 for n close to it
    for (uint64_t row0 = (uint64_t)(gid - sub); row0 < n; row0 += groups) {
        const uint64_t row = row0 + sub;
        double s[kNaMaxCols];
#pragma unroll
        for (int c = 0; c < kNaMaxCols; ++c) s[c] = 0.0;
        if (row < n) {
            const uint32_t beg = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
            for (uint32_t e = beg + lane; e < end; e += kNaG) {
                const double v = __ldg(val + e);
                const uint64_t j = __ldg(col + e);
#pragma unroll
                for (int c = 0; c < kNaMaxCols; ++c)
                    if (c < (int)k) s[c] += v * __ldg(x + (uint64_t)c * ld + j);
            }
        }
#pragma unroll
        for (int c = 0; c < kNaMaxCols; ++c) {
            if (c < (int)k) {
                const double y = prism::group_sum<kNaG>(s[c]);
                if (lane == 0 && row < n) {
                    const double bi = __ldg(b + (uint64_t)c * ld + row);
                    const double r = bi - y;
                    acc[2 * c] += r * r;
                    acc[2 * c + 1] += bi * bi;
                }
            }
        }
    }
    na_block_sum<kNaVals>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kNaVals; ++q)
            if (q < 2 * (int)k) partial[blockIdx.x * kNaVals + q] = acc[q];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double tot[kNaVals];
#pragma unroll
    for (int q = 0; q < kNaVals; ++q) tot[q] = 0.0;
    for (unsigned blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x) {
#pragma unroll
        for (int q = 0; q < kNaVals; ++q)
            if (q < 2 * (int)k) tot[q] += __ldcg(partial + blk * kNaVals + q);
    }
    na_block_sum<kNaVals>(tot, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < kNaMaxCols; ++c) {
            if (c < (int)k) {
                norms[2 * c] = sqrt(tot[2 * c]);
                norms[2 * c + 1] = sqrt(tot[2 * c + 1]);
            }
        }
        *ticket = 0u;  // re-armed for the next launch
    }
}

}  // namespace

extern "C" int32_t prism_residual_norms_noalloc(int32_t device, uint32_t n, const uint32_t* rowptr_d,
                                                const uint32_t* col_d, const double* val_d, const double* x_d,
                                                const double* b_d, uint32_t k, uint64_t ld, double* norms_d,
                                                void* stream) {
    try {
        int count = 0;
        cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess) return na_cuda_fail("cudaGetDeviceCount", e);
        if (device < 0 || device >= count || device >= kNaMaxDevices)
            return na_fail(PRISM_ERR_ARG, "prism_residual_norms_noalloc: device %llu out of range (%llu devices)",
                           (unsigned long long)device, (unsigned long long)count);
        if (n == 0) return na_fail(PRISM_ERR_ARG, "prism_residual_norms_noalloc: n must be > 0");
        if (k == 0 || k > (uint32_t)kNaMaxCols)
            return na_fail(PRISM_ERR_ARG,
                           "prism_residual_norms_noalloc: k = %llu right-hand sides; its fixed scratch holds 1 to %llu",
                           k, kNaMaxCols);
        if (k > 1 && ld < n)
            return na_fail(PRISM_ERR_ARG, "prism_residual_norms_noalloc: leading dimension %llu < n = %llu", ld, n);
        if (!rowptr_d || !col_d || !val_d || !x_d || !b_d || !norms_d)
            return na_fail(PRISM_ERR_ARG, "prism_residual_norms_noalloc: null device pointer");

        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return na_cuda_fail("cudaSetDevice", e);
        double* scratch = nullptr;
        int rc = scratch_for(device, &scratch);
        if (rc == PRISM_OK) {
            const uint64_t want = ((uint64_t)n * kNaG + kNaThreads - 1) / kNaThreads;
            const int grid = (int)(want < (uint64_t)kNaBlocks ? want : (uint64_t)kNaBlocks);
            unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNaPartialDoubles);
            e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), static_cast<cudaStream_t>(stream));
            if (e != cudaSuccess) {
                rc = na_cuda_fail("clearing the scratch ticket", e);
            } else {
                k_residual_norms_noalloc<<<grid, kNaThreads, 0, static_cast<cudaStream_t>(stream)>>>(
                    n, rowptr_d, col_d, val_d, x_d, b_d, k, k > 1 ? ld : (uint64_t)n, scratch, ticket, norms_d);
                prism::launch_counter().fetch_add(1, std::memory_order_relaxed);
                e = cudaGetLastError();
                rc = e != cudaSuccess ? na_cuda_fail("launch", e) : prism::record_error(PRISM_OK, "");
            }
        }
        if (prev >= 0 && prev != device) cudaSetDevice(prev);
        return rc;
    } catch (...) {
        return na_fail(PRISM_ERR_ARG, "prism_residual_norms_noalloc: unexpected error");
    }
}
