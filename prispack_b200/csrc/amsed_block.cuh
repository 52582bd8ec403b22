// Kernels of the AMSED / MSLR / GMSLR apply on a block of k <= 64 right-hand
// sides (AMSEDPrecondition::MInvSolve, AMSEDPrecondition.cpp:1976-2087, with
// levelCInvRecursiveSolve, :1494-1587, column by column).  Block vectors are
// interleaved, X[row * k + c], as in the block solves of batched.cu.
//
// The low-rank correction x2 += W (H o (W^T xc)) (AMSEDPrecondition.cpp:
// 1557-1574; DenseMatrix::transposeVec / MatVec, DenseMatrix.cpp:208-267)
// becomes two matrix products once k columns share W:
//   T = H o (W^T Xc)     M = rank, N = k, K = rows of the C block
//   Y += W T             M = rows,  N = k, K = rank
// With FP32 factor values they run on the tensor cores (mma.sync m16n8k16,
// BF16 operands, FP32 accumulation); with FP64 values, in FP64 on the CUDA
// cores.  Both are HBM-bound at these shapes (about 12.8 flop per byte at rank
// 32 and k = 64, far below the tensor pipe's balance point), so the
// warp-level mma is enough to keep them at the memory roofline; the tensor
// cores matter here for the conversion-free FP32 accumulation, not for peak
// throughput.
//
// BF16 conversion: values are rounded to float, then to BF16 (round to nearest
// even); products are exact in FP32 and summed in FP32 in the mma's order.
#pragma once

#include <cuda_bf16.h>

#include "kernels.cuh"

namespace prism {

constexpr int kLrMaxK = 64;     // columns of a block
constexpr int kLrQGroup = 32;   // rank columns one pass of the BF16 product accumulates

// ---------------------------------------------------------------------------
// row permutation and sparse products on interleaved blocks
// ---------------------------------------------------------------------------
// out[i] = in[perm[i]] (scatter = 0) / out[perm[i]] = in[i] (scatter = 1), rows of k values
static __global__ void __launch_bounds__(kBlock) k_bk_permute(uint32_t n, uint32_t k, const uint32_t* __restrict__ perm,
                                                              const double* __restrict__ in, double* __restrict__ out,
                                                              int scatter) {
    const uint64_t total = (uint64_t)n * k;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = e / k, c = e - i * k;
        const uint64_t p = __ldg(perm + i);
        if (scatter) out[p * k + c] = in[e];
        else out[e] = in[p * k + c];
    }
}

// Y = M X (SUB = 0) or Y -= M X (SUB = 1) for a CSR M with nrows rows; warp per row,
// lane l for columns l and l + 32; entries summed in stored order per column
// (CSRMatrix::MatPVec / MatPVecWithoutClearOutVector, CSRMatrix.h:360-486).
template <int SUB>
static __global__ void __launch_bounds__(kBlock) k_bk_csr(uint32_t nrows, uint32_t k, const uint32_t* __restrict__ rowptr,
                                                          const uint32_t* __restrict__ col,
                                                          const double* __restrict__ val, const double* __restrict__ X,
                                                          double* __restrict__ Y) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool h0 = (uint32_t)lane < k, h1 = (uint32_t)lane + 32 < k;
    for (uint32_t row = warp; row < nrows; row += nwarps) {
        const uint32_t beg = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
        double s0 = 0.0, s1 = 0.0;
        for (uint32_t e0 = beg; e0 < end; e0 += 32) {
            uint32_t cc = 0;
            double aa = 0.0;
            if (e0 + lane < end) {
                cc = __ldg(col + e0 + lane);
                aa = __ldg(val + e0 + lane);
            }
            const int cnt = (int)min(32u, end - e0);
            for (int t = 0; t < cnt; ++t) {
                const uint64_t c = __shfl_sync(0xffffffffu, cc, t);
                const double a = __shfl_sync(0xffffffffu, aa, t);
                if (h0) s0 += a * __ldg(X + c * k + lane);
                if (h1) s1 += a * __ldg(X + c * k + lane + 32);
            }
        }
        const uint64_t o = (uint64_t)row * k;
        if (SUB) {
            if (h0) Y[o + lane] = Y[o + lane] + -1.0 * s0;
            if (h1) Y[o + lane + 32] = Y[o + lane + 32] + -1.0 * s1;
        } else {
            if (h0) Y[o + lane] = s0;
            if (h1) Y[o + lane + 32] = s1;
        }
    }
}

// y[e] -= a[e] over count values
static __global__ void __launch_bounds__(kBlock) k_bk_sub(uint64_t count, const double* __restrict__ a,
                                                          double* __restrict__ y) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (uint64_t)gridDim.x * blockDim.x)
        y[e] -= a[e];
}

// ---------------------------------------------------------------------------
// low-rank block products, FP64 (CUDA cores)
// ---------------------------------------------------------------------------
// Block partials of W^T X for rank columns q and block columns c: thread (g, c) with
// g = threadIdx.x / 64 sums q = g, g + 4, ... over the block's rows (grid-stride by
// blocks of 64 rows); the last block adds the partials in block order and scales by H.
static __global__ void __launch_bounds__(kBlock) k_lr_dots_f64(uint32_t nrem, uint32_t k, uint32_t r,
                                                               const double* __restrict__ W, const double* __restrict__ H,
                                                               const double* __restrict__ X, double* __restrict__ partial,
                                                               unsigned* __restrict__ ticket, double* __restrict__ T) {
    const uint32_t c = threadIdx.x & 63, g = threadIdx.x >> 6;
    for (uint32_t q0 = 0; q0 < r; q0 += 32) {
        double acc[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) acc[t] = 0.0;
        if (c < k) {
            for (uint32_t i0 = blockIdx.x * 64; i0 < nrem; i0 += gridDim.x * 64) {
                const uint32_t i1 = min(nrem, i0 + 64);
                for (uint32_t i = i0; i < i1; ++i) {
                    const double x = X[(uint64_t)i * k + c];
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        const uint32_t q = q0 + g + 4 * t;
                        if (q < r) acc[t] += W[(size_t)q * nrem + i] * x;
                    }
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const uint32_t q = q0 + g + 4 * t;
            if (q < r && c < k) partial[((size_t)blockIdx.x * r + q) * kLrMaxK + c] = acc[t];
        }
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (uint32_t e = threadIdx.x; e < r * kLrMaxK; e += blockDim.x) {
        const uint32_t q = e / kLrMaxK, cc = e % kLrMaxK;
        if (cc >= k) continue;
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(partial + ((size_t)b * r + q) * kLrMaxK + cc);
        T[(size_t)q * kLrMaxK + cc] = s * H[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0u;
}

// Y[i][c] += sum_q W[q][i] T[q][c], q in order (DenseMatrix::MatVec column order, then x2 += ...)
static __global__ void __launch_bounds__(kBlock) k_lr_add_f64(uint32_t nrem, uint32_t k, uint32_t r,
                                                              const double* __restrict__ W, const double* __restrict__ T,
                                                              double* __restrict__ Y) {
    const uint64_t total = (uint64_t)nrem * k;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(e / k), c = (uint32_t)(e - (uint64_t)i * k);
        double s = 0.0;
        for (uint32_t q = 0; q < r; ++q) s += W[(size_t)q * nrem + i] * T[(size_t)q * kLrMaxK + c];
        Y[e] += s;
    }
}

// ---------------------------------------------------------------------------
// low-rank block products, BF16 operands on the tensor cores (FP32 accumulate)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low half) = lo
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D += A(16x16, row) B(16x8, col): BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// T = H o (W^T X) for rank <= rpad (a multiple of 16) and k <= 64 columns.
// Wc: BF16, column-major rpad x ldw (ldw = rows rounded up to 16, zero padded), so that
// the A fragment (rows q, columns i) reads pairs of consecutive rows i.  Each warp takes
// 16-row slices of X (grid-stride) and accumulates a 32 x 64 tile (two q tiles, eight
// column tiles) per pass over X; the warps of a block add their tiles in warp order in
// shared memory, the blocks' tiles are added in block order by the last block.
static __global__ void __launch_bounds__(kBlock) k_lr_dots_tc(uint32_t nrem, uint32_t ldw, uint32_t k, uint32_t rpad,
                                                              const __nv_bfloat16* __restrict__ Wc,
                                                              const float* __restrict__ H, const double* __restrict__ X,
                                                              float* __restrict__ partial, unsigned* __restrict__ ticket,
                                                              float* __restrict__ T) {
    __shared__ float tile[kLrQGroup][kLrMaxK];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + wid, nwarps = gridDim.x * (blockDim.x >> 5);
    const uint32_t slices = ldw / 16;
    for (uint32_t q0 = 0; q0 < rpad; q0 += kLrQGroup) {
        const int qt = min((uint32_t)kLrQGroup, rpad - q0) / 16;  // q tiles this pass (1 or 2)
        float acc[2][8][4];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.f;
        for (uint32_t s = gwarp; s < slices; s += nwarps) {
            const uint32_t i0 = s * 16;
            uint32_t af[2][4];
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                if (m < qt) {
                    const __nv_bfloat16* w0 = Wc + (size_t)(q0 + 16 * m + gid) * ldw + i0 + 2 * tig;
                    const __nv_bfloat16* w1 = w0 + (size_t)8 * ldw;
                    af[m][0] = *reinterpret_cast<const uint32_t*>(w0);
                    af[m][1] = *reinterpret_cast<const uint32_t*>(w1);
                    af[m][2] = *reinterpret_cast<const uint32_t*>(w0 + 8);
                    af[m][3] = *reinterpret_cast<const uint32_t*>(w1 + 8);
                }
            }
            const uint32_t ra = i0 + 2 * tig, rb = ra + 8;  // the rows of this lane's B values
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const uint32_t c = 8 * nt + gid;
                float x[4] = {0.f, 0.f, 0.f, 0.f};
                if (c < k) {
                    if (ra < nrem) x[0] = (float)X[(uint64_t)ra * k + c];
                    if (ra + 1 < nrem) x[1] = (float)X[(uint64_t)(ra + 1) * k + c];
                    if (rb < nrem) x[2] = (float)X[(uint64_t)rb * k + c];
                    if (rb + 1 < nrem) x[3] = (float)X[(uint64_t)(rb + 1) * k + c];
                }
                const uint32_t b0 = pack_bf16(x[0], x[1]), b1 = pack_bf16(x[2], x[3]);
#pragma unroll
                for (int m = 0; m < 2; ++m)
                    if (m < qt) mma_bf16_16816(acc[m][nt], af[m], b0, b1);
            }
        }
        // the block's sum of the warps' tiles, warp by warp
        for (int e = threadIdx.x; e < kLrQGroup * kLrMaxK; e += blockDim.x) (&tile[0][0])[e] = 0.f;
        __syncthreads();
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            if (wid == w) {
#pragma unroll
                for (int m = 0; m < 2; ++m)
#pragma unroll
                    for (int nt = 0; nt < 8; ++nt) {
                        const int qa = 16 * m + gid, cb = 8 * nt + 2 * tig;
                        tile[qa][cb] += acc[m][nt][0];
                        tile[qa][cb + 1] += acc[m][nt][1];
                        tile[qa + 8][cb] += acc[m][nt][2];
                        tile[qa + 8][cb + 1] += acc[m][nt][3];
                    }
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < qt * 16 * kLrMaxK; e += blockDim.x)
            partial[((size_t)blockIdx.x * rpad + q0) * kLrMaxK + e] = (&tile[0][0])[e];
        __syncthreads();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (uint32_t e = threadIdx.x; e < rpad * kLrMaxK; e += blockDim.x) {
        float s = 0.f;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(partial + (size_t)b * rpad * kLrMaxK + e);
        T[e] = s * H[e / kLrMaxK];
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0u;
}

// Y += W T for rank <= rpad and k <= 64 columns.  Wr: BF16, row-major ldw x rpad (zero
// padded), so that the A fragment (rows i, columns q) reads pairs of consecutive q; T (FP32,
// rpad x 64) is rounded to BF16 once per block in shared memory.  Each warp computes a
// 16 x 64 tile of rows (grid-stride) and adds it to Y in FP64.
static __global__ void __launch_bounds__(kBlock) k_lr_add_tc(uint32_t nrem, uint32_t ldw, uint32_t k, uint32_t rpad,
                                                             const __nv_bfloat16* __restrict__ Wr,
                                                             const float* __restrict__ T, double* __restrict__ Y) {
    extern __shared__ __align__(16) uint32_t tb[];  // [rpad / 2][64]: BF16 pairs (q, q + 1) per column
    for (uint32_t e = threadIdx.x; e < (rpad / 2) * kLrMaxK; e += blockDim.x) {
        const uint32_t qp = e / kLrMaxK, c = e % kLrMaxK;
        tb[e] = pack_bf16(T[(size_t)(2 * qp) * kLrMaxK + c], T[(size_t)(2 * qp + 1) * kLrMaxK + c]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + wid, nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t s = gwarp; s < ldw / 16; s += nwarps) {
        const uint32_t i0 = s * 16;
        float acc[8][4];
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[b][e] = 0.f;
        for (uint32_t q0 = 0; q0 < rpad; q0 += 16) {
            const __nv_bfloat16* w0 = Wr + (size_t)(i0 + gid) * rpad + q0 + 2 * tig;
            const __nv_bfloat16* w1 = w0 + (size_t)8 * rpad;
            uint32_t af[4];
            af[0] = *reinterpret_cast<const uint32_t*>(w0);
            af[1] = *reinterpret_cast<const uint32_t*>(w1);
            af[2] = *reinterpret_cast<const uint32_t*>(w0 + 8);
            af[3] = *reinterpret_cast<const uint32_t*>(w1 + 8);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const uint32_t c = 8 * nt + gid;
                const uint32_t b0 = tb[(q0 / 2 + tig) * kLrMaxK + c];
                const uint32_t b1 = tb[(q0 / 2 + 4 + tig) * kLrMaxK + c];
                mma_bf16_16816(acc[nt], af, b0, b1);
            }
        }
        const uint32_t ra = i0 + gid, rb = ra + 8;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const uint32_t c = 8 * nt + 2 * tig;
            if (ra < nrem) {
                if (c < k) Y[(uint64_t)ra * k + c] += (double)acc[nt][0];
                if (c + 1 < k) Y[(uint64_t)ra * k + c + 1] += (double)acc[nt][1];
            }
            if (rb < nrem) {
                if (c < k) Y[(uint64_t)rb * k + c] += (double)acc[nt][2];
                if (c + 1 < k) Y[(uint64_t)rb * k + c + 1] += (double)acc[nt][3];
            }
        }
    }
}

}  // namespace prism
