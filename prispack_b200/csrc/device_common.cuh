// Device-side plumbing shared by the solve-phase kernels: error handling,
// owning device buffers, launch accounting and small PTX helpers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace prism {

// Error carried up to the C ABI, where it becomes a prism_status + message.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define PRISM_CUDA(call)                                                                          \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            throw ::prism::Error(2, std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

// Count of kernel launches issued by this library (reported through the ABI).
std::atomic<uint64_t>& launch_counter();

#define PRISM_LAUNCHED()                                                                          \
    do {                                                                                          \
        ::prism::launch_counter().fetch_add(1, std::memory_order_relaxed);                        \
        cudaError_t e_ = cudaGetLastError();                                                      \
        if (e_ != cudaSuccess)                                                                    \
            throw ::prism::Error(2, std::string("kernel launch: ") + cudaGetErrorString(e_));     \
    } while (0)

template <typename T>
class DevBuf {
  public:
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p_, count * sizeof(T));
        if (e != cudaSuccess) {
            p_ = nullptr;
            throw Error(8, std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) + " B): " + cudaGetErrorString(e));
        }
        n_ = count;
    }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    void upload(const T* host, size_t count, cudaStream_t s) {
        if (count > n_) alloc(count);
        if (count) PRISM_CUDA(cudaMemcpyAsync(p_, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }

  private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

constexpr int kBlock = 256;

// Scratch of one deterministic grid reduction (see grid_reduce in kernels.cuh).
struct ReduceSlot {
    double* partial;      // [gridDim.x * NV]
    unsigned* ticket;     // one counter, 0 between launches
    double* out;          // [NV]
};

// ---- PTX helpers -------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const void* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(void* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

}  // namespace prism
