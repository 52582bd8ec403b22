// Streamed round sweep: one triangular sweep (IncompleteCholesky /
// IncompleteLDLT / IncompleteLU MSolve*UsePtr, IncompleteCholesky.cpp:249-295,
// IncompleteLDLT.cpp:188-233, IncompleteLU.cpp:268-297) as one persistent
// CTA per SM, each owning a slab of contiguous rows (StreamLayout).
//
// Why.  A sweep is a chain of dependency wavefronts (about 2,000 for the
// level-0 ILDLT factor of 3D Poisson 128^3).  When every dependency crosses
// the L2 (k_sweep), each wavefront costs about two L2 round trips.  Here a
// slab computes its rows in rounds of up to 128 mutually independent rows,
// one thread per row, reading every dependency from a shared-memory value
// slot, with an mbarrier between rounds, so the chain inside a slab costs a
// few shared-memory reads and a barrier phase per round.  The L2 is kept off
// the chain in two ways: the slab's round records stream from HBM into a
// shared-memory ring by bulk copies (cp.async.bulk + mbarrier) well ahead of
// their rounds, and values of rows owned by other slabs ("halo" rows, always
// upstream: lower sweeps depend on lower rows only, upper sweeps on higher
// ones) are copied into their slots by prefetcher warps as soon as they are
// finished, while the slab is still working on earlier rounds.
//
// What a round costs (3D Poisson 128^3, level-0 factor, B200): about 0.7 us
// with float arithmetic, in slabs with and without halo rows alike; about
// half is the dot product, half the round's bookkeeping (record fields,
// result, barrier, next record).  Each is a chain of dependent shared-memory
// loads and arithmetic of some tens of cycles a link.
//
// Roles (352 threads; the polling warps sleep between polls so that the row
// threads, which carry the dependency chain, keep the issue slots):
//   warps 0..3    row threads: thread j computes row j of each round, then each
//                 warp arrives on the round's mbarrier and waits for it.  A
//                 wavefront of a slab rarely holds more than 128 rows, so a
//                 slab's chain of rounds is about as long as its chain of levels.
//   warps 4..9    prefetchers: warp 4+k handles rounds k, k+6, ...: it waits
//                 until the round's record has landed, polls each new halo row
//                 in global memory until it is finished, waits until the slot's
//                 previous value has had its last reader (xwait), writes the
//                 slot and arrives on the barrier that ends the round before,
//                 whose phase therefore also means "the next round's halo is in".
//   warp 10       producer: issues the bulk copies of the records into the
//                 ring in order, publishes how many have landed, and recycles
//                 the ring space of finished rounds.
//
// Finished values are published in global memory with the kPending encoding
// of k_sweep (the 8-byte word itself says whether it is finished); a prep
// kernel writes each row's right-hand side into its record and marks the
// output pending before the sweep.
//
// Progress: rounds of a slab depend only on earlier rounds of the slab and on
// upstream slabs, so the most upstream unfinished slab always progresses
// (its halo rows are finished, its records need only ring space that its own
// finished rounds release).  All CTAs are co-resident (cooperative launch,
// one per SM).  There is no hardware barrier: every wait is a bounded poll
// (wait_ns); on expiry the kernel raises status 6 and tells the CTA to leave,
// the producer waits (again bounded) for its copies in flight, and every
// warp returns.
#pragma once

#include <type_traits>

#include "kernels.cuh"

namespace prism {

constexpr int kStrRowWarps = (int)kRoundRows / 32;     // row threads: one per row of a round
constexpr int kStrPrefetchWarps = 6;                   // warps kStrRowWarps .. kStrProducer - 1
constexpr int kStrProducer = kStrRowWarps + kStrPrefetchWarps;
constexpr int kStrThreads = 32 * (kStrProducer + 1);
constexpr uint32_t kStrMaxRounds = 64;                 // rounds in flight (ring table slots)
// copy barriers, round barriers, start barrier (+pad), ring offsets, words
constexpr uint32_t kStrFixedSmem = 64 * 8 + 64 * 8 + 16 + 64 * 4 + 32;
static_assert(kStrThreads <= 1024, "warp roles");

struct StreamArgs {
    const unsigned char* blob;
    const uint4* meta;            // per round: {offset / 16, bytes, nr | L << 16, X}
    const uint32_t* cta_round;    // num_ctas + 1
    const uint32_t* slab_start;   // num_ctas + 1: CTA b owns rows [slab_start[b], slab_start[b+1])
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
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
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
__device__ __forceinline__ bool mbar_try_parity(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
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

// Prep: each row's right-hand side into its record, the output marked pending.
// Safe for in == out (each row is read, then written, by one thread).
static __global__ void __launch_bounds__(kBlock) k_stream_prep(uint32_t n, const uint32_t* __restrict__ in_slot,
                                                               const double* in, double* __restrict__ blob64,
                                                               unsigned long long* out) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double v = in[r];
        blob64[__ldg(in_slot + r)] = v;
        out[r] = kPending;
    }
}

// Acc: the arithmetic type of the sweep (double; float for the single-precision apply,
// whose value slots, products and sums are float and whose results are widened to double).
template <typename Low, int OP, typename Acc>
static __global__ void __launch_bounds__(kStrThreads, 1) k_sweep_stream(const StreamArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* tma_bar = reinterpret_cast<uint64_t*>(sm);                     // [64] record copies
    uint64_t* round_bar = tma_bar + 64;                                      // [64] end of round r (r % 64)
    uint64_t* start_bar = round_bar + 64;                                    // round 0's halo in place
    uint32_t* ring_off = reinterpret_cast<uint32_t*>(sm + 64 * 8 * 2 + 16);  // [64]
    uint32_t* words = ring_off + 64;  // landed, rounds done, abort
    uint4* meta_s = reinterpret_cast<uint4*>(sm + kStrFixedSmem);            // [meta_slots]
    Acc* xs = reinterpret_cast<Acc*>(meta_s + a.meta_slots);                 // [slots]; xs[0] = 0
    unsigned char* ring = reinterpret_cast<unsigned char*>(xs) + ((a.slots * (uint32_t)sizeof(Acc) + 127u) & ~127u);
    const uint32_t b = blockIdx.x;
    const uint32_t rb = a.slab_start[b];
    const uint32_t r0 = a.cta_round[b];
    const uint32_t R = a.cta_round[b + 1] - r0;
    constexpr uint32_t vb = sizeof(Low);

    for (uint32_t i = threadIdx.x; i < R; i += blockDim.x) meta_s[i] = __ldg(a.meta + r0 + i);
    if (threadIdx.x == 0) {
        xs[0] = (Acc)0;
        words[0] = 0;  // records landed
        words[1] = 0;  // rounds done
        words[2] = 0;  // abort

        for (uint32_t i = 0; i < kStrMaxRounds; ++i) {
            mbar_init(tma_bar + i, 1);
            mbar_init(round_bar + i, kStrRowWarps + 1);  // the row warps + the next round's prefetcher
        }
        mbar_init(start_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

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
            while (issued < R && issued - freed < kStrMaxRounds) {
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
            // no copy may still be writing into this CTA's shared memory when it exits
            const unsigned long long t0 = globaltimer_ns();
            while (landed < issued && globaltimer_ns() - t0 < wait_ns) {
                if (mbar_test_parity(tma_bar + landed % kStrMaxRounds, (landed / kStrMaxRounds) & 1u)) ++landed;
            }
        }
        return;
    }

    if (warp >= kStrRowWarps) {
        // ------------------------------------------------------------------ prefetchers
        // Warp k copies in the halo of rounds k, k + 6, ... and then arrives on the barrier
        // that ends the round before (start_bar for round 0).  That barrier's previous phase
        // (64 rounds earlier) is over: the record of round q is in the ring only once round
        // q - 64 is done.  Round R is a stand-in that only arrives.
        for (uint32_t q = (uint32_t)(warp - kStrRowWarps); q <= R; q += kStrPrefetchWarps) {
            bool ok = true;
            unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            if (q == R) {
                while (R >= kStrMaxRounds && ld_acquire_shared_u32(words + 1) + kStrMaxRounds < R + 1) {
                    __nanosleep(spins < 16 ? 64 : 256);  // polling warps leave issue slots to the row threads
                    if (give_up(spins, t0)) {
                        ok = false;
                        break;
                    }
                }
                if (__all_sync(0xFFFFFFFFu, ok) && lane == 0) mbar_arrive(round_bar + (R - 1) % kStrMaxRounds);
                break;
            }
            while (ld_acquire_shared_u32(words) <= q) {
                __nanosleep(spins < 16 ? 64 : 256);  // polling warps leave issue slots to the row threads
                if (give_up(spins, t0)) {
                    ok = false;
                    break;
                }
            }
            if (!__all_sync(0xFFFFFFFFu, ok)) return;
            const uint4 m = meta_s[q];
            const uint32_t X = m.w;
            const RoundRec rec = round_rec(m.z & 0xFFFFu, m.z >> 16, X, vb);
            const unsigned char* base = ring + ring_off[q % kStrMaxRounds];
            const uint32_t* xrow = reinterpret_cast<const uint32_t*>(base + rec.xrow);
            const uint16_t* xslot = reinterpret_cast<const uint16_t*>(base + rec.xslot);
            const uint16_t* xwait = reinterpret_cast<const uint16_t*>(base + rec.xwait);
            for (uint32_t x0 = 0; x0 < X; x0 += 64) {
                // two halo rows per lane in flight at once
                unsigned long long v[2];
                uint32_t idx[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    idx[u] = x0 + (uint32_t)lane + 32u * u;
                    v[u] = idx[u] < X ? ld_relaxed_u64(a.out + xrow[idx[u]]) : 0ull;
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (idx[u] >= X || !ok) continue;
                    if (v[u] == kPending) {
                        const double* p = a.out + xrow[idx[u]];
                        ok = spin_ready([&] { return ld_relaxed_u64(p); }, v[u], status, wait_ns);
                    }
                    const uint32_t need = xwait[idx[u]];
                    if (ok && ld_acquire_shared_u32(words + 1) < need) {
                        t0 = globaltimer_ns();
                        spins = 0;
                        while (ld_acquire_shared_u32(words + 1) < need) {
                            __nanosleep(spins < 16 ? 64 : 256);  // polling warps leave issue slots to the row threads
                            if (give_up(spins, t0)) {
                                ok = false;
                                break;
                            }
                        }
                    }
                    if (ok) xs[xslot[idx[u]]] = (Acc)__longlong_as_double((long long)v[u]);
                }
            }
            if (!__all_sync(0xFFFFFFFFu, ok)) {
                if (lane == 0) {
                    atomicCAS(status, 0, 6);
                    vwords[2] = 1;
                }
                return;
            }
            if (lane == 0) mbar_arrive(q == 0 ? start_bar : round_bar + (q - 1) % kStrMaxRounds);
        }
        return;
    }

    // ---------------------------------------------------------------------- row threads
    // Thread j computes row j of each round: its entries ({slot, coefficient}, one load
    // each) sit at j, j + m, j + 2m, ...
    // of the round's entry table (m = rows rounded up to 8), padded with slot 0 (0.0)
    // to the round's longest row.  Before waiting for the barrier that ends round r,
    // each thread reads round r+1's record -- up to 32 entries, right-hand side,
    // diagonal, slots -- into registers; after it only the value-slot reads (all
    // independent, issued back to back), the sums and the result remain on the chain.
    const uint32_t j = threadIdx.x;
    constexpr int kRegEntries = 32;
    struct Row {
        uint32_t nr, L, m;              // rows, entries per row, stride
        uint32_t os, lr, base;
        Acc vin, dg;
        uint32_t c[kRegEntries];
        Low v[kRegEntries];
    };
    Row cur;
    // record entry e of the round (this thread's entries: e = j, j + m, ...): {slot, coefficient};
    // one 8-byte load for float values, a u16 slot and a double for double values
    auto ent_get = [](const unsigned char* rbase, const RoundRec& rec, uint32_t e, uint32_t& c, Low& v) {
        if constexpr (sizeof(Low) == 4) {
            const unsigned long long w = reinterpret_cast<const unsigned long long*>(rbase + rec.ent)[e];
            c = (uint32_t)w;
            v = __uint_as_float((uint32_t)(w >> 32));
        } else {
            c = reinterpret_cast<const uint16_t*>(rbase + rec.ent)[e];
            v = reinterpret_cast<const double*>(rbase + rec.val)[e];
        }
    };
    auto load_row = [&](uint32_t r, Row& w) {
        const uint4 m = meta_s[r];
        w.nr = m.z & 0xFFFFu;
        w.L = m.z >> 16;
        const RoundRec rec = round_rec(w.nr, w.L, m.w, vb);
        w.base = ring_off[r % kStrMaxRounds];
        w.m = rec.m;
        if (j >= w.nr) return;
        const unsigned char* base = ring + w.base;
        w.vin = (Acc)reinterpret_cast<const double*>(base + rec.in)[j];
        w.dg = (Acc)reinterpret_cast<const double*>(base + rec.diag)[j];
        w.os = reinterpret_cast<const uint16_t*>(base + rec.oslot)[j];
        w.lr = reinterpret_cast<const uint16_t*>(base + rec.lrow)[j];
        // only as many register entries as the round's longest row needs (8, 16, 24, 28 or 32)
        auto fill = [&](auto nconst) {
            constexpr int N = decltype(nconst)::value;
#pragma unroll
            for (int u = 0; u < N; ++u) {
                w.c[u] = 0u;
                w.v[u] = (Low)0;
                if ((uint32_t)u < w.L) ent_get(base, rec, u * rec.m + j, w.c[u], w.v[u]);
            }
        };
        if (w.L <= 8) fill(std::integral_constant<int, 8>{});
        else if (w.L <= 16) fill(std::integral_constant<int, 16>{});
        else if (w.L <= 24) fill(std::integral_constant<int, 24>{});
        else if (w.L <= 28) fill(std::integral_constant<int, 28>{});
        else fill(std::integral_constant<int, 32>{});
    };
    // sum of the first N register entries (N a multiple of 4): value reads first, then four chains
    auto dot_regs = [&](const Row& w, auto nconst) {
        constexpr int N = decltype(nconst)::value;
        Acc x[N];
#pragma unroll
        for (int u = 0; u < N; ++u) x[u] = xs[w.c[u]];
        Acc acc[4] = {(Acc)0, (Acc)0, (Acc)0, (Acc)0};
#pragma unroll
        for (int u = 0; u < N; ++u) acc[u & 3] += (Acc)w.v[u] * x[u];
        return (acc[0] + acc[1]) + (acc[2] + acc[3]);
    };
    auto wait_phase = [&](uint64_t* bar, uint32_t parity) {
        if (mbar_try_parity(bar, parity)) return true;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (!mbar_try_parity(bar, parity))
            if (give_up(spins, t0)) return false;
        return true;
    };
    if (!wait_phase(start_bar, 0)) return;
    load_row(0, cur);
    uint32_t landed_seen = 1;
    for (uint32_t r = 0; r < R; ++r) {
        if (j < cur.nr) {
            Acc s;
            if (cur.L <= 8) s = dot_regs(cur, std::integral_constant<int, 8>{});
            else if (cur.L <= 16) s = dot_regs(cur, std::integral_constant<int, 16>{});
            else if (cur.L <= 24) s = dot_regs(cur, std::integral_constant<int, 24>{});
            else if (cur.L <= 28) s = dot_regs(cur, std::integral_constant<int, 28>{});
            else s = dot_regs(cur, std::integral_constant<int, 32>{});
            if (cur.L > (uint32_t)kRegEntries) {  // rows longer than 32 entries
                const RoundRec rr = round_rec(cur.nr, cur.L, 0u, vb);  // entry sections do not depend on X
                for (uint32_t k = kRegEntries; k < cur.L; ++k) {
                    uint32_t c;
                    Low v;
                    ent_get(ring + cur.base, rr, k * cur.m + j, c, v);
                    s += (Acc)v * xs[c];
                }
            }
            Acc res;
            if (OP == OP_DIV || OP == OP_MUL) res = (cur.vin - s) * cur.dg;  // dg = 1/diag for OP_DIV
            else if (OP == OP_NONE) res = cur.vin - s;
            else res = cur.vin * cur.dg - s;                                  // dg = 1/diag
            const double rd = (double)res;
            unsigned long long rbits = (unsigned long long)__double_as_longlong(rd);
            if (rd != rd) rbits = kCanonicalNaN;
            if (cur.os != kNoSlot) {
                if constexpr (sizeof(Acc) == 8) xs[cur.os] = __longlong_as_double((long long)rbits);
                else xs[cur.os] = res;
            }
            st_relaxed_u64(a.out + rb + cur.lr, rbits);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(round_bar + r % kStrMaxRounds);
        const bool more = r + 1 < R;
        if (more) {
            if (landed_seen <= r + 1) {
                // the next record normally landed long ago; otherwise wait for it here
                const unsigned long long t0 = globaltimer_ns();
                unsigned spins = 0;
                bool ok = true;
                do {
                    uint32_t l = 0;
                    if (lane == 0) l = ld_acquire_shared_u32(words);
                    landed_seen = __shfl_sync(0xFFFFFFFFu, l, 0);
                    if (landed_seen > r + 1) break;
                    ok = !give_up(spins, t0);
                } while (__all_sync(0xFFFFFFFFu, ok));
                if (!__all_sync(0xFFFFFFFFu, ok)) return;
            }
            load_row(r + 1, cur);
        }
        if (!wait_phase(round_bar + r % kStrMaxRounds, (r / kStrMaxRounds) & 1u)) return;
        if (threadIdx.x == 0) st_release_shared_u32(words + 1, r + 1);
    }
}

}  // namespace prism
