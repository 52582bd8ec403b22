// Streamed round sweep: one triangular sweep (IncompleteCholesky /
// IncompleteLDLT / IncompleteLU MSolve*UsePtr, IncompleteCholesky.cpp:249-295,
// IncompleteLDLT.cpp:188-233, IncompleteLU.cpp:268-297) as one persistent
// CTA per SM, each owning a slab of contiguous rows (StreamLayout in
// host_setup.hpp describes the records).
//
// Why.  A sweep is a chain of dependency wavefronts (about 2,000 for the
// level-0 ILDLT factor of 3D Poisson 128^3), so its time is the number of
// wavefronts times the latency of one.  A slab computes its rows in rounds of
// up to 128 mutually independent rows, one thread per row, reading every
// dependency from a shared-memory value slot; the L2 stays off the chain: the
// slab's round records stream from HBM into a shared-memory ring by bulk
// copies (cp.async.bulk + mbarrier) well ahead of their rounds, and values of
// rows owned by other slabs ("halo" rows, always upstream: lower sweeps depend
// on lower rows only, upper sweeps on higher ones) are copied into their slots
// by prefetcher warps as soon as they are finished.
//
// What sits on the chain.  Of a row's ~25 dependencies only two or three
// ("late" entries) are rows of the round just before; the others ("early"
// entries) were computed two or more rounds earlier or are halo values.  So
// while round i is computed, each row thread also sums round i + 1's early
// entries, and round i + 1 then only adds its late entries: one round on the
// chain is a barrier, a few shared-memory loads and fused multiply-adds, the
// result and its store.  The record of round i + 2 is loaded into registers
// a round ahead of use, and the setup orders every row's entries so that the
// 32 (16 for 8-byte slots) rows one wavefront serves read distinct banks.
//
// Roles (256 threads, two warps per SM sub-partition):
//   warps 0..3    row threads: thread j computes row j of each round.  One
//                 iteration (after the barrier that ends round i - 1): load round
//                 i's late values; sum round i + 1's early entries; finish round
//                 i (late entries, result into its slot and into global memory);
//                 load round i + 2's record into registers; barrier (a named
//                 barrier with an OR reduction, so that all four warps take the
//                 same decision to leave).
//   warps 4..6    prefetchers: warp 4+k handles the halo of rounds k, k+3, ...:
//                 polls each halo row in global memory until it is finished,
//                 waits until the slot's previous value has had its last reader,
//                 writes the slot and raises the round's halo flag.  A row thread
//                 that finds round i + 1's flag down sums its early entries after
//                 the barrier instead, waiting for the flag there.
//   warp 7        producer: issues the bulk copies of the records into the ring
//                 in order, publishes how many have landed, and recycles the ring
//                 space of finished rounds.
//
// Finished values are published in global memory with the kPending encoding
// of k_sweep (the 8-byte word itself says whether it is finished); a prep
// kernel writes each row's right-hand side into its record and marks the
// output pending before the sweep.
//
// Progress: rounds of a slab depend only on earlier rounds of the slab and on
// upstream slabs, so the most upstream unfinished slab always progresses.  All
// CTAs are co-resident (cooperative launch, one per SM).  Every wait is a
// bounded poll (wait_ns); on expiry the kernel raises status 6 and tells the
// CTA to leave; the row warps leave together after their next barrier, and the
// producer waits (bounded, much longer than any copy takes) for its copies in
// flight before it returns.
#pragma once

#include <type_traits>

#include "host_setup.hpp"
#include "kernels.cuh"

namespace prism {


constexpr int kStrRowWarps = (int)kRoundRows / 32;     // row threads: one per row of a round
constexpr int kStrPrefetchWarps = 3;                   // warps kStrRowWarps .. kStrProducer - 1
constexpr int kStrProducer = kStrRowWarps + kStrPrefetchWarps;
constexpr int kStrThreads = 32 * (kStrProducer + 1);
constexpr uint32_t kStrMaxRounds = 64;                 // rounds in flight (ring table and halo flag slots)
// copy barriers, halo flags, ring offsets, words
constexpr uint32_t kStrFixedSmem = 64 * 8 + 64 * 4 + 64 * 4 + 32;
constexpr unsigned long long kStrDrainNs = 2000000000ull;  // bound of the final wait for copies in flight
static_assert(kStrThreads <= 1024, "warp roles");
static_assert(kStrFixedSmem % 16 == 0, "round table alignment");

// Dynamic shared memory of one CTA, in bytes from its start: copy barriers, halo flags,
// ring offsets and words (kStrFixedSmem), the round table (16 B per round), the value
// slots (rounded up to 128 B), then the ring.  The host sizes the launch with the same
// function.
struct StrSmem {
    uint32_t meta, xs, ring, total;
};
PRISM_HD inline StrSmem stream_smem(uint32_t meta_slots, uint32_t slots, uint32_t slot_bytes, uint32_t ring_bytes) {
    StrSmem m;
    m.meta = kStrFixedSmem;
    m.xs = m.meta + 16u * meta_slots;
    m.ring = m.xs + ((slots * slot_bytes + 127u) & ~127u);
    m.total = m.ring + ring_bytes;
    return m;
}

struct StreamArgs {
    const unsigned char* blob;
    const uint4* meta;            // per round: {offset / 16, bytes, nr | Eg << 8 | Kg << 16 | halo << 24, 0}
    const uint32_t* cta_round;    // num_ctas + 1
    const uint32_t* slab_start;   // num_ctas + 1: CTA b owns rows [slab_start[b], slab_start[b+1])
    const uint32_t* halo_ptr;     // rounds + 1
    const uint32_t* halo_row;     // per halo copy: row
    const uint32_t* halo_sw;      // per halo copy: slot | wait << 16
    uint32_t n, ring_bytes, meta_slots, slots;
    double* out;
    int* status;
    unsigned long long wait_ns;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t ld_acquire_shared_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_shared_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_addr(p)), "r"(v) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test_parity(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// global -> shared bulk copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Barrier 1 over the row threads with an OR reduction: every row thread gets the
// same answer, so all of them leave at the same barrier or none does.
__device__ __forceinline__ bool row_barrier_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(kStrRowWarps * 32)
        : "memory");
    return r != 0;
}

// Correctly rounded arithmetic in the sweep's type, never contracted.
__device__ __forceinline__ float acc_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double acc_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float acc_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double acc_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float acc_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double acc_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float acc_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double acc_mul(double a, double b) { return __dmul_rn(a, b); }

// four coefficients of one entry group (16-byte aligned)
template <typename Low>
__device__ __forceinline__ void load_coef4(const unsigned char* p, Low (&c)[4]) {
    if constexpr (sizeof(Low) == 4) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        c[0] = v.x;
        c[1] = v.y;
        c[2] = v.z;
        c[3] = v.w;
    } else {
        const double2 v0 = *reinterpret_cast<const double2*>(p);
        const double2 v1 = *reinterpret_cast<const double2*>(p + 16);
        c[0] = v0.x;
        c[1] = v0.y;
        c[2] = v1.x;
        c[3] = v1.y;
    }
}

// Value loads of a round's first EG early entry groups (slots: 4 x u16 per group), all
// issued before any is used.
template <int EG, int EGR, typename Acc>
__device__ __forceinline__ void gather_groups(const Acc* xs, const uint32_t (&es)[EGR][2], Acc (&x)[EGR][4]) {
#pragma unroll
    for (int g = 0; g < EG; ++g) {
        x[g][0] = xs[es[g][0] & 0xFFFFu];
        x[g][1] = xs[es[g][0] >> 16];
        x[g][2] = xs[es[g][1] & 0xFFFFu];
        x[g][3] = xs[es[g][1] >> 16];
    }
}
// c_i += coefficient * value over early positions 4g + i of the first EG groups
template <int EG, int EGR, typename Acc, typename Low>
__device__ __forceinline__ void fma_groups(const Low (&ec)[EGR][4], const Acc (&x)[EGR][4], Acc (&c)[4]) {
#pragma unroll
    for (int g = 0; g < EG; ++g) {
#pragma unroll
        for (int i = 0; i < 4; ++i) c[i] = acc_fma((Acc)ec[g][i], x[g][i], c[i]);
    }
}

// Prep: each row's right-hand side into its record (in the sweep's type), the output
// marked pending.  Safe for in == out (each row is read, then written, by one thread).
template <typename Acc>
static __global__ void __launch_bounds__(kBlock) k_stream_prep(uint32_t n, const uint32_t* __restrict__ in_slot,
                                                               const double* in, Acc* __restrict__ blob,
                                                               unsigned long long* out) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double v = in[r];
        blob[__ldg(in_slot + r)] = (Acc)v;
        out[r] = kPending;
    }
}

// Low: factor value type; Acc: the arithmetic type of the sweep (double; float for the
// single-precision apply, whose value slots, products and sums are float and whose
// results are widened to double).
template <typename Low, int OP, typename Acc>
static __global__ void __launch_bounds__(kStrThreads, 1) k_sweep_stream(const StreamArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* tma_bar = reinterpret_cast<uint64_t*>(sm);                       // [64] record copies
    uint32_t* hflag = reinterpret_cast<uint32_t*>(sm + 64 * 8);                // [64] round q's halo in: q + 1
    uint32_t* ring_off = hflag + 64;                                           // [64]
    uint32_t* words = ring_off + 64;                                           // landed, rounds done, abort
    const StrSmem lay = stream_smem(a.meta_slots, a.slots, (uint32_t)sizeof(Acc), a.ring_bytes);
    uint4* meta_s = reinterpret_cast<uint4*>(sm + lay.meta);                   // [meta_slots]
    Acc* xs = reinterpret_cast<Acc*>(sm + lay.xs);                             // [slots]; zero slots first
    unsigned char* ring = sm + lay.ring;
    constexpr uint32_t vb = sizeof(Low), ab = sizeof(Acc);
    constexpr uint32_t NZ = ab == 4 ? 32u : 16u;
    const uint32_t b = blockIdx.x;
    const uint32_t rb = a.slab_start[b];
    const uint32_t g0 = a.cta_round[b];
    const uint32_t R = a.cta_round[b + 1] - g0;

    for (uint32_t i = threadIdx.x; i < R; i += blockDim.x) meta_s[i] = __ldg(a.meta + g0 + i);
    for (uint32_t i = threadIdx.x; i < NZ; i += blockDim.x) xs[i] = (Acc)0;
    for (uint32_t i = threadIdx.x; i < kStrMaxRounds; i += blockDim.x) hflag[i] = 0;
    if (threadIdx.x == 0) {
        words[0] = 0;  // records landed
        words[1] = 0;  // rounds done
        words[2] = 0;  // abort
        for (uint32_t i = 0; i < kStrMaxRounds; ++i) mbar_init(tma_bar + i, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (R == 0) return;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* status = a.status;
    const unsigned long long wait_ns = a.wait_ns;
    volatile uint32_t* vwords = words;
    // bounded-wait helper: true (and the CTA told to leave) after wait_ns without success
    auto give_up = [&](unsigned& spins, unsigned long long t0) {
        if ((++spins & 15u) != 0u) return false;
        if (vwords[2] != 0 || ld_relaxed_s32(status) != 0 || globaltimer_ns() - t0 > wait_ns) {
            atomicCAS(status, 0, 6);
            vwords[2] = 1;
            return true;
        }
        return false;
    };
    // bounded wait until rounds done >= need (polling warps sleep between polls)
    auto wait_done = [&](uint32_t need) {
        if (ld_acquire_shared_u32(words + 1) >= need) return true;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_shared_u32(words + 1) < need) {
            __nanosleep(32);
            if (give_up(spins, t0)) return false;
        }
        return true;
    };

    if (warp == kStrProducer) {
        // ------------------------------------------------------------------ producer
        if (lane != 0) return;
        uint32_t issued = 0, landed = 0, freed = 0, head = 0;
        unsigned long long t_event = globaltimer_ns();
        unsigned spins = 0;
        bool failed = false;
        while (landed < R) {
            bool event = false;
            const uint32_t done = ld_acquire_shared_u32(words + 1);  // rounds done: their records are free
            while (freed < landed && freed < done) {
                ++freed;
                event = true;
            }
            // ring: live records [freed, issued) occupy [tail, head) circularly
            const uint32_t tail = freed < issued ? ring_off[freed % kStrMaxRounds] : head;
            while (issued < R && issued - freed < kStrMaxRounds && vwords[2] == 0) {
                const uint4 m = meta_s[issued];
                const uint32_t bytes = m.y;
                uint32_t off;
                if (issued == freed) {
                    off = 0;
                    if (bytes > a.ring_bytes) break;  // rejected by the host; never reached
                } else if (head > tail) {
                    if (head + bytes <= a.ring_bytes) off = head;
                    else if (bytes <= tail) off = 0;
                    else break;
                } else {
                    if (head + bytes <= tail) off = head;
                    else break;
                }
                ring_off[issued % kStrMaxRounds] = off;
                uint64_t* bar = tma_bar + issued % kStrMaxRounds;
                // the readers of a released region finished before its refill
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive_expect_tx(bar, bytes);
                bulk_copy_g2s(ring + off, a.blob + (size_t)m.x * 16, bytes, bar);
                head = off + bytes;
                ++issued;
                event = true;
            }
            const uint32_t before = landed;
            while (landed < issued && mbar_test_parity(tma_bar + landed % kStrMaxRounds, (landed / kStrMaxRounds) & 1u))
                ++landed;
            if (landed != before) {
                st_release_shared_u32(words, landed);
                event = true;
            }
            if (event) {
                t_event = globaltimer_ns();
                spins = 0;
            } else {
                __nanosleep(spins < 16 ? 64 : 256);  // polling warps leave issue slots to the row threads
                if (give_up(spins, t_event)) {
                    failed = true;
                    break;
                }
            }
        }
        if (failed) {
            // no new copy was issued after the failure; wait for those in flight so that none
            // is still writing into this CTA's shared memory when it exits
            const unsigned long long t0 = globaltimer_ns();
            while (landed < issued && globaltimer_ns() - t0 < kStrDrainNs) {
                if (mbar_test_parity(tma_bar + landed % kStrMaxRounds, (landed / kStrMaxRounds) & 1u)) ++landed;
                else __nanosleep(256);
            }
        }
        return;
    }

    if (warp >= kStrRowWarps) {
        // ------------------------------------------------------------------ prefetchers
        // Warp k copies in the halo of rounds k, k + 3, ... and raises each round's flag.
        // Round q's halo is read while round q - 1 is computed (rounds done = q - 1); each
        // slot's wait (<= q - 2) lets the copy happen a round before that.
        for (uint32_t q = (uint32_t)(warp - kStrRowWarps); q < R; q += kStrPrefetchWarps) {
            if ((meta_s[q].z >> 24) == 0u) continue;
            const uint32_t x0 = __ldg(a.halo_ptr + g0 + q), x1 = __ldg(a.halo_ptr + g0 + q + 1);
            bool ok = true;
            for (uint32_t xb = x0; xb < x1; xb += 64) {
                // two halo rows per lane in flight at once
                unsigned long long v[2];
                uint32_t idx[2], row[2], sw[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    idx[u] = xb + (uint32_t)lane + 32u * u;
                    row[u] = idx[u] < x1 ? __ldg(a.halo_row + idx[u]) : 0u;
                    sw[u] = idx[u] < x1 ? __ldg(a.halo_sw + idx[u]) : 0u;
                    v[u] = idx[u] < x1 ? ld_relaxed_u64(a.out + row[u]) : 0ull;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (idx[u] >= x1 || !ok) continue;
                    if (v[u] == kPending) {
                        const double* p = a.out + row[u];
                        ok = spin_ready([&] { return ld_relaxed_u64(p); }, v[u], status, wait_ns);
                        if (!ok) break;
                    }
                    if (!wait_done(sw[u] >> 16)) {
                        ok = false;
                        break;
                    }
                    xs[sw[u] & 0xFFFFu] = (Acc)__longlong_as_double((long long)v[u]);
                }
            }
            if (!__all_sync(0xFFFFFFFFu, ok)) {
                if (lane == 0) {
                    atomicCAS(status, 0, 6);
                    vwords[2] = 1;
                }
                return;
            }
            __syncwarp();
            if (lane == 0) {
                // the flag's slot last served round q - 64, whose readers are done with it
                // once round q - 63 is done
                if (!wait_done(q >= 63 ? q - 63 : 0)) return;
                st_release_shared_u32(hflag + q % kStrMaxRounds, q + 1);
            }
        }
        return;
    }

    // ---------------------------------------------------------------------- row threads
    const uint32_t j = threadIdx.x;
    constexpr int EGR = (int)stream_early_groups(ab);  // early entry groups in registers (every round has them)
    // One round as a row thread holds it: fields, the first group of late entries and,
    // once summed, its early part P.
    struct Fld {
        Acc vin, dg, P;
        uint32_t lo, shape, base;
        uint32_t ls0, ls1;
        Low lc[4];
    };
    uint32_t es[EGR][2];  // early slots of the round whose early part comes next (4 x u16 per group)
    Low ec[EGR][4];       // and their coefficients
    auto nr_of = [](uint32_t shape) { return shape & 0xFFu; };
    auto eg_of = [](uint32_t shape) { return (shape >> 8) & 0xFFu; };
    auto kg_of = [](uint32_t shape) { return (shape >> 16) & 0xFFu; };
    auto rec_of = [&](const Fld& F) {
        return round_rec(nr_of(F.shape), eg_of(F.shape), kg_of(F.shape), vb, ab);
    };
    auto load_fields = [&](uint32_t q, Fld& F) {
        const uint4 m = meta_s[q];
        F.shape = m.z;
        F.base = ring_off[q % kStrMaxRounds];
        F.P = (Acc)0;
        if (j >= nr_of(m.z)) return;
        const RoundRec rec = rec_of(F);
        const unsigned char* base = ring + F.base;
        if constexpr (ab == 4) {
            const uint4 f = *reinterpret_cast<const uint4*>(base + rec.fld + 16u * j);
            F.vin = __uint_as_float(f.x);
            F.dg = __uint_as_float(f.y);
            F.lo = f.z;
        } else {
            const double2 f = *reinterpret_cast<const double2*>(base + rec.fld + 16u * j);
            F.vin = f.x;
            F.dg = f.y;
            F.lo = *reinterpret_cast<const uint32_t*>(base + rec.lo + 4u * j);
        }
        const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.ls + 8u * j);  // late group 0
        F.ls0 = s2.x;
        F.ls1 = s2.y;
        load_coef4<Low>(base + rec.lc + 4u * vb * j, F.lc);
    };
    // the early entries of a round (its first EGR groups) into registers
    auto load_early = [&](const Fld& F) {
        constexpr int EG = EGR;
        if (j >= nr_of(F.shape)) return;
        const RoundRec rec = rec_of(F);
        const unsigned char* base = ring + F.base;
#pragma unroll
        for (int g = 0; g < EG; ++g) {
            const uint32_t e = (uint32_t)g * rec.m + j;
            const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.es + 8u * e);
            es[g][0] = s2.x;
            es[g][1] = s2.y;
            load_coef4<Low>(base + rec.ec + 4u * vb * e, ec[g]);
        }
    };
    // P = (c0 + c1) + (c2 + c3): c holds the register groups' chains; entry groups beyond
    // the register groups (rows longer than 4 * EGR entries) continue from the record
    auto close_early = [&](Acc c0, Acc c1, Acc c2, Acc c3, Fld& F) {
        const uint32_t Eg = eg_of(F.shape);
        if (Eg > (uint32_t)EGR) {
            const RoundRec rec = rec_of(F);
            const unsigned char* base = ring + F.base;
            for (uint32_t g = EGR; g < Eg; ++g) {
                const uint32_t e = g * rec.m + j;
                const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.es + 8u * e);
                Low cf[4];
                load_coef4<Low>(base + rec.ec + 4u * vb * e, cf);
                c0 = acc_fma((Acc)cf[0], xs[s2.x & 0xFFFFu], c0);
                c1 = acc_fma((Acc)cf[1], xs[s2.x >> 16], c1);
                c2 = acc_fma((Acc)cf[2], xs[s2.y & 0xFFFFu], c2);
                c3 = acc_fma((Acc)cf[3], xs[s2.y >> 16], c3);
            }
        }
        F.P = acc_add(acc_add(c0, c1), acc_add(c2, c3));
    };
    // the whole early part of a round at once (prologue, and a round whose halo came late)
    auto early_sum = [&](Fld& F) {
        if (j >= nr_of(F.shape)) return;
        Acc x[EGR][4];
        Acc c[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
        gather_groups<EGR, EGR, Acc>(xs, es, x);
        fma_groups<EGR, EGR, Acc, Low>(ec, x, c);
        close_early(c[0], c[1], c[2], c[3], F);
    };
    auto finish = [&](const Fld& F, const Acc (&xl)[4]) {
        const uint32_t Kg = kg_of(F.shape);  // >= 1: every round has a late group (padding where empty)
        Acc s = F.P;
#pragma unroll
        for (int i = 0; i < 4; ++i) s = acc_fma((Acc)F.lc[i], xl[i], s);
        if (Kg > 1u) {  // more than four late entries: the rest from the record
            const RoundRec rec = rec_of(F);
            const unsigned char* base = ring + F.base;
            for (uint32_t g = 1; g < Kg; ++g) {
                const uint32_t e = g * rec.m + j;
                const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.ls + 8u * e);
                Low cf[4];
                load_coef4<Low>(base + rec.lc + 4u * vb * e, cf);
                s = acc_fma((Acc)cf[0], xs[s2.x & 0xFFFFu], s);
                s = acc_fma((Acc)cf[1], xs[s2.x >> 16], s);
                s = acc_fma((Acc)cf[2], xs[s2.y & 0xFFFFu], s);
                s = acc_fma((Acc)cf[3], xs[s2.y >> 16], s);
            }
        }
        Acc res;
        if (OP == OP_DIV || OP == OP_MUL) res = acc_mul(acc_sub(F.vin, s), F.dg);  // dg = 1/diag for OP_DIV
        else if (OP == OP_NONE) res = acc_sub(F.vin, s);
        else res = acc_sub(acc_mul(F.vin, F.dg), s);                                 // dg = 1/diag
        const double rd = (double)res;
        unsigned long long rbits = (unsigned long long)__double_as_longlong(rd);
        if (rd != rd) rbits = kCanonicalNaN;
        const uint32_t os = F.lo >> 16;
        if (os != kNoSlot) xs[os] = res;
        st_relaxed_u64(a.out + rb + (F.lo & 0xFFFFu), rbits);
    };
    auto wait_landed = [&](uint32_t q) {
        if (ld_acquire_shared_u32(words) > q) return true;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_shared_u32(words) <= q)
            if (give_up(spins, t0)) return false;
        return true;
    };
    auto halo_in = [&](uint32_t q) { return ld_acquire_shared_u32(hflag + q % kStrMaxRounds) == q + 1; };
    auto wait_halo = [&](uint32_t q) {
        if (halo_in(q)) return true;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (!halo_in(q))
            if (give_up(spins, t0)) return false;
        return true;
    };
    auto has_halo = [](const Fld& F) { return (F.shape >> 24) != 0u; };

    bool bad = false;
    Fld F0, F1;
    F0.shape = F1.shape = 0u;
    // prologue: round 0 with its early part summed, round 1's record in registers
    if (!wait_landed(0)) bad = true;
    if (!bad) {
        load_fields(0, F0);
        load_early(F0);
        if (has_halo(F0) && !wait_halo(0)) bad = true;
    }
    if (!bad) early_sum(F0);
    if (!bad && R > 1) {
        if (!wait_landed(1)) bad = true;
        else {
            load_fields(1, F1);
            load_early(F1);
        }
    }
    // One iteration: cur = round i (early part summed), nxt = round i + 1 (record in
    // registers); once round i is finished, cur receives round i + 2.  Returns true when
    // the row threads leave.
    auto step = [&](uint32_t i, Fld& cur, Fld& nxt) -> bool {
        const bool more = i + 1 < R, more2 = i + 2 < R;
        // round i + 1's early part now unless its halo is not in yet (then after the barrier)
        const bool pend = more && !bad && has_halo(nxt) && !halo_in(i + 1);
        const bool live = !bad && j < nr_of(cur.shape);
        const bool early = more && !bad && !pend && j < nr_of(nxt.shape);
        {
            // every value load first: round i's late values, round i + 1's early ones
            Acc xl[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
            if (live) {
                xl[0] = xs[cur.ls0 & 0xFFFFu];
                xl[1] = xs[cur.ls0 >> 16];
                xl[2] = xs[cur.ls1 & 0xFFFFu];
                xl[3] = xs[cur.ls1 >> 16];
            }
            Acc x[EGR][4];
            if (early) gather_groups<EGR, EGR, Acc>(xs, es, x);
            if (live) finish(cur, xl);
            if (early) {
                Acc c[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
                fma_groups<EGR, EGR, Acc, Low>(ec, x, c);
                close_early(c[0], c[1], c[2], c[3], nxt);
            }
        }
        if (more2 && !bad) {
            if (!wait_landed(i + 2)) bad = true;
            else {
                load_fields(i + 2, cur);
                if (!pend) load_early(cur);
            }
        }
        __syncwarp();
        const bool stop = row_barrier_or(bad || vwords[2] != 0u);
        if (threadIdx.x == 0) st_release_shared_u32(words + 1, i + 1);
        if (stop) return true;
        if (pend) {
            if (!wait_halo(i + 1)) {
                bad = true;
            } else {
                early_sum(nxt);
                if (more2) load_early(cur);
            }
        }
        return false;
    };
    for (uint32_t i = 0; i < R; i += 2) {
        if (step(i, F0, F1)) break;
        if (i + 1 >= R || step(i + 1, F1, F0)) break;
    }
}

}  // namespace prism
