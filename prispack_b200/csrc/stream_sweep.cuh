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
// What sits on the chain.  Of a row's ~25 dependencies only a few ("late"
// entries) are rows of the kStreamLate rounds just before; the others ("early"
// entries) were computed earlier or are halo values.  Helper warps sum every
// row's early entries of round q as soon as rounds <= q - kStreamLate - 1 are
// done, and hand the row threads a packet per row (the early sum P, the
// right-hand side, the diagonal, the result slot and the first four late
// entries).  One round on the chain is then: the packet, a few shared-memory
// loads and fused multiply-adds, the result and its stores, and a barrier of
// the four row warps; the early sums of the next rounds overlap it on other
// warps.  The setup orders every row's entries so that the 32 (16 for 8-byte
// slots) rows one wavefront serves read distinct banks.
//
// Roles (416 threads, 13 warps):
//   warps 0..3    row threads: thread j computes row j of each round.  Round i:
//                 wait for its packets, load the late values, add them to P one
//                 fused multiply-add at a time, the result into its slot and into
//                 global memory; barrier (a named barrier with an OR reduction, so
//                 that all four warps take the same decision to leave); thread 0
//                 publishes "rounds done".
//   warps 4..7    helpers: warp 4+h handles rounds h, h+4, ...: waits until rounds
//                 <= q - kStreamLate - 1 are done, round q's record has landed and
//                 its halo is in, then sums the early entries of every row of round
//                 q (slices of 32 rows) and publishes the round's packets.
//   warps 8..11   prefetchers: warp 8+k handles the halo of rounds k, k+4, ...:
//                 polls each halo row in global memory until it is finished,
//                 waits until the slot's previous value has had its last reader,
//                 writes the slot and raises the round's halo flag.
//   warp 12       producer: issues the bulk copies of the records into the ring
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
// CTA to leave; the row warps leave together after their next barrier, the
// helpers and prefetchers at their next wait, and the producer waits (bounded, much longer than any copy takes) for its copies in
// flight before it returns.
#pragma once

#include <type_traits>

#include "host_setup.hpp"
#include "kernels.cuh"

namespace prism {


constexpr int kStrRowWarps = (int)kRoundRows / 32;     // row threads: one per row of a round
constexpr int kStrHelperWarps = 4;                     // early sums: warps kStrRowWarps ..
constexpr int kStrPrefetchWarps = 4;                   // halo copies
constexpr int kStrPrefetch0 = kStrRowWarps + kStrHelperWarps;
constexpr int kStrProducer = kStrPrefetch0 + kStrPrefetchWarps;
constexpr int kStrThreads = 32 * (kStrProducer + 1);
constexpr uint32_t kStrMaxRounds = 64;                 // rounds in flight (ring table and halo flag slots)
constexpr uint32_t kStrPackets = 4;                    // rounds of packets in shared memory
static_assert(kStrPackets > kStreamLate, "a packet slot is refilled only after its round is done");
// copy barriers, halo flags, ring offsets, words, packet flags [kStrPkSlots], packet round
// info [kStrPkSlots]
constexpr uint32_t kStrPkSlots = (kStrPackets + 3u) & ~3u;
constexpr uint32_t kStrFixedSmem = 64 * 8 + 64 * 4 + 64 * 4 + 32 + kStrPkSlots * 4 + kStrPkSlots * 8 + 16;
constexpr unsigned long long kStrDrainNs = 2000000000ull;  // bound of the final wait for copies in flight
static_assert(kStrThreads <= 1024, "warp roles");
static_assert(kStrFixedSmem % 16 == 0, "round table alignment");

// What a helper hands the row thread of one row of a round: the early sum, the
// right-hand side, the diagonal (or its reciprocal), the row (low 16 bits) and result
// slot (high 16 bits), the first two groups of late slots (4 x u16 each; the second
// unused when the round has one) and their coefficients.
template <typename Low, typename Acc>
struct alignas(16) StrPacket {
    Acc P, vin, dg;
    uint32_t lo, ls[4];
    Low lc[8];
};
// 16-byte words of a packet for factor values of vb bytes and value slots of ab bytes
PRISM_HD constexpr uint32_t stream_packet_words(uint32_t vb, uint32_t ab) { return ab == 4 ? 4u : (vb == 4 ? 5u : 7u); }
static_assert(sizeof(StrPacket<float, float>) == 16 * stream_packet_words(4, 4), "packet words");
static_assert(sizeof(StrPacket<float, double>) == 16 * stream_packet_words(4, 8), "packet words");
static_assert(sizeof(StrPacket<double, double>) == 16 * stream_packet_words(8, 8), "packet words");

// Dynamic shared memory of one CTA, in bytes from its start: copy barriers, halo flags,
// ring offsets, words and packet flags (kStrFixedSmem), the round table (16 B per round),
// the value slots (rounded up to 128 B), the packets (kStrPackets rounds, one 16-byte word
// array per packet word), then the ring.  The host sizes the launch with the same function.
struct StrSmem {
    uint32_t meta, xs, pk, ring, total;
};
PRISM_HD inline StrSmem stream_smem(uint32_t meta_slots, uint32_t slots, uint32_t slot_bytes, uint32_t factor_bytes,
                                    uint32_t ring_bytes) {
    StrSmem m;
    m.meta = kStrFixedSmem;
    m.xs = m.meta + 16u * meta_slots;
    m.pk = m.xs + ((slots * slot_bytes + 127u) & ~127u);
    m.ring = m.pk + kStrPackets * kRoundRows * 16u * stream_packet_words(factor_bytes, slot_bytes);
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

// Prep of a paired sweep: each row's right-hand side b'_r = b_r - sum m b_dep (one fused
// multiply-add per entry, in stored order, in double) into its record; the output marked
// pending when mark (not when in == out: rows read other rows of `in`).
template <typename Acc>
static __global__ void __launch_bounds__(kBlock) k_stream_prep_pair(uint32_t n, const uint32_t* __restrict__ in_slot,
                                                                    const uint32_t* __restrict__ mptr,
                                                                    const uint32_t* __restrict__ mdep,
                                                                    const double* __restrict__ mcoef,
                                                                    const double* in, Acc* __restrict__ blob,
                                                                    unsigned long long* out, int mark) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double v = in[r];
        for (uint32_t q = __ldg(mptr + r); q < __ldg(mptr + r + 1); ++q)
            v = __fma_rn(-__ldg(mcoef + q), in[__ldg(mdep + q)], v);
        blob[__ldg(in_slot + r)] = (Acc)v;
        if (mark) out[r] = kPending;
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
    uint32_t* pflag = words + 8;                                               // [kStrPackets] round q's packets: q + 1
    uint2* pinfo = reinterpret_cast<uint2*>(pflag + kStrPkSlots);              // [kStrPackets] {ring offset, shape}
    constexpr uint32_t vb = sizeof(Low), ab = sizeof(Acc);
    constexpr uint32_t PW = stream_packet_words(vb, ab);
    const StrSmem lay = stream_smem(a.meta_slots, a.slots, ab, vb, a.ring_bytes);
    uint4* meta_s = reinterpret_cast<uint4*>(sm + lay.meta);                   // [meta_slots]
    Acc* xs = reinterpret_cast<Acc*>(sm + lay.xs);                             // [slots]; zero slots first
    uint4* pkw = reinterpret_cast<uint4*>(sm + lay.pk);                        // [PW][kStrPackets * kRoundRows]
    unsigned char* ring = sm + lay.ring;
    constexpr uint32_t NZ = ab == 4 ? 32u : 16u;
    const uint32_t b = blockIdx.x;
    const uint32_t rb = a.slab_start[b];
    const uint32_t g0 = a.cta_round[b];
    const uint32_t R = a.cta_round[b + 1] - g0;

    for (uint32_t i = threadIdx.x; i < R; i += blockDim.x) meta_s[i] = __ldg(a.meta + g0 + i);
    for (uint32_t i = threadIdx.x; i < NZ; i += blockDim.x) xs[i] = (Acc)0;
    for (uint32_t i = threadIdx.x; i < kStrMaxRounds; i += blockDim.x) hflag[i] = 0;
    for (uint32_t i = threadIdx.x; i < kStrPackets; i += blockDim.x) pflag[i] = 0;
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

    if (warp >= kStrPrefetch0) {
        // ------------------------------------------------------------------ prefetchers
        // Warp k copies in the halo of rounds k, k + kStrPrefetchWarps, ... and raises each
        // round's flag.
        // Round q's halo is read by its helper once rounds <= q - kStreamLate - 1 are done;
        // each slot's wait (<= q - kStreamLate) lets the copy happen by then.
        for (uint32_t q = (uint32_t)(warp - kStrPrefetch0); q < R; q += kStrPrefetchWarps) {
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

    auto nr_of = [](uint32_t shape) { return shape & 0xFFu; };
    auto eg_of = [](uint32_t shape) { return (shape >> 8) & 0xFFu; };
    auto kg_of = [](uint32_t shape) { return (shape >> 16) & 0xFFu; };
    constexpr uint32_t PKN = kStrPackets * kRoundRows;  // packets of one word array
    using Packet = StrPacket<Low, Acc>;

    if (warp >= kStrRowWarps) {
        // ------------------------------------------------------------------ helpers
        constexpr int EGR = (int)stream_early_groups(ab);  // early entry groups in registers (every round has them)
        const uint32_t l = (uint32_t)lane;
        // tight bounded spin on a shared word (the helpers are on the round chain's critical path)
        auto spin_until = [&](auto ready) {
            if (ready()) return true;
            const unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            while (!ready())
                if (give_up(spins, t0)) return false;
            return true;
        };
        for (uint32_t q = (uint32_t)(warp - kStrRowWarps); q < R; q += kStrHelperWarps) {
            const uint32_t need = q > kStreamLate ? q - kStreamLate : 0u;  // rounds <= q - kStreamLate - 1 done
            bool ok = spin_until([&] { return ld_acquire_shared_u32(words + 1) >= need; }) &&
                      spin_until([&] { return ld_acquire_shared_u32(words) > q; });
            // the halo of every round <= q: round q may read halo rows that an earlier round copied
            // in first; rounds <= q - kStreamLate - 1 are done, so their helpers saw their flags.
            // A flag slot only grows (round h + 1, then h + 65, ... once round h is done), so a
            // value >= h + 1 says round h's halo is in.
            for (uint32_t h = q > kStreamLate ? q - kStreamLate : 0u; ok && h <= q; ++h)
                if ((meta_s[h].z >> 24) != 0u)
                    ok = spin_until([&] { return ld_acquire_shared_u32(hflag + h % kStrMaxRounds) >= h + 1; });
            const uint32_t shape = meta_s[q].z;
            if (!__all_sync(0xFFFFFFFFu, ok)) return;  // the CTA is leaving (status raised by give_up)
            const uint32_t nr = nr_of(shape), Eg = eg_of(shape), Kg = kg_of(shape);
            const uint32_t off = ring_off[q % kStrMaxRounds];
            const RoundRec rec = round_rec(nr, Eg, Kg, vb, ab);
            const unsigned char* base = ring + off;
            uint4* dst = pkw + (q % kStrPackets) * kRoundRows;
            for (uint32_t s0 = 0; s0 < nr; s0 += 32) {  // the same for the whole warp
                const uint32_t r = s0 + l;
                if (r < nr) {
                    union {
                        Packet p;
                        uint4 w[PW];
                    } u;
                    if constexpr (ab == 4) {
                        const uint4 f = *reinterpret_cast<const uint4*>(base + rec.fld + 16u * r);
                        u.p.vin = __uint_as_float(f.x);
                        u.p.dg = __uint_as_float(f.y);
                        u.p.lo = f.z;
                    } else {
                        const double2 f = *reinterpret_cast<const double2*>(base + rec.fld + 16u * r);
                        u.p.vin = f.x;
                        u.p.dg = f.y;
                        u.p.lo = *reinterpret_cast<const uint32_t*>(base + rec.lo + 4u * r);
                    }
                    // late groups 0 and 1
                    const uint2 l2 = *reinterpret_cast<const uint2*>(base + rec.ls + 8u * r);
                    u.p.ls[0] = l2.x;
                    u.p.ls[1] = l2.y;
                    load_coef4<Low>(base + rec.lc + 4u * vb * r, *reinterpret_cast<Low(*)[4]>(u.p.lc));
                    if (Kg > 1u) {
                        const uint32_t e = rec.m + r;
                        const uint2 m2 = *reinterpret_cast<const uint2*>(base + rec.ls + 8u * e);
                        u.p.ls[2] = m2.x;
                        u.p.ls[3] = m2.y;
                        load_coef4<Low>(base + rec.lc + 4u * vb * e, *reinterpret_cast<Low(*)[4]>(u.p.lc + 4));
                    } else {
                        u.p.ls[2] = u.p.ls[3] = 0u;
#pragma unroll
                        for (int t = 4; t < 8; ++t) u.p.lc[t] = (Low)0;
                    }
                    // early part: fma chains c_i over positions 4g + i, P = (c0 + c1) + (c2 + c3)
                    uint32_t es[EGR][2];
                    Low ec[EGR][4];
#pragma unroll
                    for (int g = 0; g < EGR; ++g) {
                        const uint32_t e = (uint32_t)g * rec.m + r;
                        const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.es + 8u * e);
                        es[g][0] = s2.x;
                        es[g][1] = s2.y;
                        load_coef4<Low>(base + rec.ec + 4u * vb * e, ec[g]);
                    }
                    Acc x[EGR][4];
                    gather_groups<EGR, EGR, Acc>(xs, es, x);
                    Acc c[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
                    fma_groups<EGR, EGR, Acc, Low>(ec, x, c);
                    for (uint32_t g = EGR; g < Eg; ++g) {  // more groups than registers: the rest from the record
                        const uint32_t e = g * rec.m + r;
                        const uint2 s2 = *reinterpret_cast<const uint2*>(base + rec.es + 8u * e);
                        Low cf[4];
                        load_coef4<Low>(base + rec.ec + 4u * vb * e, cf);
                        c[0] = acc_fma((Acc)cf[0], xs[s2.x & 0xFFFFu], c[0]);
                        c[1] = acc_fma((Acc)cf[1], xs[s2.x >> 16], c[1]);
                        c[2] = acc_fma((Acc)cf[2], xs[s2.y & 0xFFFFu], c[2]);
                        c[3] = acc_fma((Acc)cf[3], xs[s2.y >> 16], c[3]);
                    }
                    u.p.P = acc_add(acc_add(c[0], c[1]), acc_add(c[2], c[3]));
#pragma unroll
                    for (uint32_t w = 0; w < PW; ++w) dst[w * PKN + r] = u.w[w];
                }
            }
            __syncwarp();
            if (lane == 0) {
                pinfo[q % kStrPackets] = make_uint2(off, shape);
                st_release_shared_u32(pflag + q % kStrPackets, q + 1);
            }
        }
        return;
    }

    // ---------------------------------------------------------------------- row threads
    const uint32_t j = threadIdx.x;
    bool bad = false;
    union Pk {
        Packet p;
        uint4 w[PW];
    };
    auto wait_packet = [&](uint32_t i) {
        const uint32_t ps = i % kStrPackets;
        if (ld_acquire_shared_u32(pflag + ps) == i + 1) return true;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_shared_u32(pflag + ps) != i + 1)
            if (give_up(spins, t0)) return false;
        return true;
    };
    auto load_packet = [&](uint32_t i, Pk& u) {
        const uint4* src = pkw + (i % kStrPackets) * kRoundRows + j;
#pragma unroll
        for (uint32_t w = 0; w < PW; ++w) u.w[w] = src[w * PKN];
    };
    // row j of round i from its packet: the result into its slot; returns the encoded result
    // for global memory, which the caller stores after publishing the round (a release
    // would otherwise wait for that store to reach L2)
    auto compute = [&](uint32_t i, uint32_t shape, const Pk& u) -> unsigned long long {
        const uint32_t Kg = kg_of(shape);  // >= 1: every round has a late group (padding where empty)
        Acc xl[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const uint32_t sl = (u.p.ls[t / 2] >> (16 * (t & 1))) & 0xFFFFu;
            if (t < 4 || Kg > 1u) xl[t] = xs[sl];
        }
        Acc s = u.p.P;
#pragma unroll
        for (int t = 0; t < 4; ++t) s = acc_fma((Acc)u.p.lc[t], xl[t], s);
        if (Kg > 1u) {  // the second late group (warp-uniform)
#pragma unroll
            for (int t = 4; t < 8; ++t) s = acc_fma((Acc)u.p.lc[t], xl[t], s);
        }
        if (Kg > 2u) {  // more than eight late entries: the rest from the record
            const RoundRec rec = round_rec(nr_of(shape), eg_of(shape), Kg, vb, ab);
            const unsigned char* base = ring + pinfo[i % kStrPackets].x;
            for (uint32_t g = 2; g < Kg; ++g) {
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
        if (OP == OP_DIV || OP == OP_MUL) res = acc_mul(acc_sub(u.p.vin, s), u.p.dg);  // dg = 1/diag for OP_DIV
        else if (OP == OP_NONE) res = acc_sub(u.p.vin, s);
        else res = acc_sub(acc_mul(u.p.vin, u.p.dg), s);                                 // dg = 1/diag
        const double rd = (double)res;
        unsigned long long rbits = (unsigned long long)__double_as_longlong(rd);
        if (rd != rd) rbits = kCanonicalNaN;
        const uint32_t os = u.p.lo >> 16;
        if (os != kNoSlot) xs[os] = res;
        return rbits;
    };
    for (uint32_t i = 0; i < R; ++i) {
        const uint32_t shape = meta_s[i].z;
        if (!bad && !wait_packet(i)) bad = true;
        bool mine = false;
        unsigned long long rbits = 0;
        uint32_t orow = 0;
        if (!bad && j < nr_of(shape)) {
            Pk u;
            load_packet(i, u);
            rbits = compute(i, shape, u);
            orow = u.p.lo & 0xFFFFu;
            mine = true;
        }
        __syncwarp();
        const bool stop = row_barrier_or(bad || vwords[2] != 0u);
        if (threadIdx.x == 0) st_release_shared_u32(words + 1, i + 1);
        if (mine) st_relaxed_u64(a.out + rb + orow, rbits);
        if (stop) break;
    }
}

}  // namespace prism
