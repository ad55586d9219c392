/*
 * The persistent mixed-code decode kernel (mixed.cuh): one grid per code
 * rate takes work items (up to `chunk` frames of one (rate, z)) from its
 * rate's queue and decodes each with a body specialised on z, so every edge
 * address is a compile-time constant as in the specialised decoder
 * (nms_decode.cuh) and no address table is needed.
 *
 * Within an item the CTA runs G = THREADS / z frame slots in lockstep, one
 * thread per expanded row. Every slot owns two posterior buffers in shared
 * memory: while it decodes the frame in one, the next frame of the item is
 * already on its way into the other by a cp.async.bulk copy (TMA, no
 * multicast) completed on that buffer's mbarrier. When a slot's frame
 * converges or reaches the cap, its outputs are written, the prefetched
 * frame becomes current after its initial syndrome check (reference
 * lib/ldpc_decoder.cc:127-139) and the following frame is fetched into the
 * freed buffer (early-exit compaction without a load on the critical path).
 *
 * LAYOUT selects where a thread's compressed messages (M1, M2, NEG per
 * layer) live: in registers, or in shared memory (fewer registers, more
 * resident CTAs). The arithmetic is the plain normalized min-sum of
 * tdmp_layer(), bit-exact with the reference. The six per-rate grids run
 * concurrently or one after another (the handle's launch policy): together
 * they fill each other's stalls, one at a time they keep fewer z bodies in
 * the instruction caches.
 *
 * Every mbarrier wait is bounded: on expiry the kernel records
 * kErrWaitTimeout, waits (bounded) for the copies it has in flight and exits.
 */
#ifndef WLDPC_MIXED_KERNEL_CUH
#define WLDPC_MIXED_KERNEL_CUH

#include "mixed.cuh"

namespace wldpc {

enum MixedLayout : int { kMsgRegisters = 0, kMsgShared = 1 };

using MixedKernel = void (*)(const MixedArgs);

/* resident CTAs per SM the register allocation is sized for. The register
 * file is split over the SM's four schedulers, so w warps per SM leave
 * 16384 / ceil(w / 4) / 32 registers per thread: with the messages in
 * registers the kernel needs more than 96 (15 warps: 128; 12 warps: 168),
 * with them in shared memory 80 suffice (24 warps). */
template <int THREADS, int LAYOUT>
struct MixedOcc {
    static constexpr int MIN_CTAS = LAYOUT == kMsgRegisters ? (THREADS == 96 ? 5 : 2) : (THREADS == 96 ? 8 : 4);
};

/* dynamic shared memory of a CTA: two posterior buffers of 24 floats per
 * thread, plus the messages (3 words per layer per thread) in the shared layout */
constexpr int mixed_smem_bytes(int threads, int layout)
{
    return 2 * 24 * threads * 4 + (layout == kMsgShared ? 3 * kMaxMb * threads * 4 : 0);
}

struct MixedCtl {
    int flist[kMixedMaxChunk];       /* the item's frames, in decode order */
    long long olist[kMixedMaxChunk]; /* and their LLR offsets */
    int frame[kMixedMaxSlots];       /* current frame of each slot, -1 = empty */
    int pre[kMixedMaxSlots];         /* frame prefetched into the other buffer, -1 = none */
    long long off_cur[kMixedMaxSlots], off_pre[kMixedMaxSlots];
    unsigned cur;                    /* bit q: buffer holding slot q's current frame */
    unsigned phase;                  /* bit 8b + q: parity the next wait on bar[b][q] expects */
    unsigned fresh, fail, abort;
    int next;                        /* frames of the item handed out */
    int item;
};

/* The CTA's shared state, at file scope so that the z bodies, which are not
 * inlined, still address it as shared memory: the posterior buffers (and the
 * shared-layout messages) in the dynamic shared memory, the control block and
 * one mbarrier per (buffer, slot). */
extern __shared__ __align__(128) float g_mixed_smem[];
static __shared__ MixedCtl g_mixed_ctl;
static __shared__ __align__(8) uint64_t g_mixed_bar[2][kMixedMaxSlots];

/* Not inlined: each z body gets its own register allocation (with all 19
 * inlined into one kernel the register layout's messages went to local
 * memory); the call happens once per work item. */
template <int R, int Z, int THREADS, int LAYOUT>
__device__ __noinline__ bool mixed_item(const MixedArgs& a, const MixedItem item)
{
    float* const smem = g_mixed_smem;
    MixedCtl& S = g_mixed_ctl;
    auto& bar = g_mixed_bar;
    constexpr int MB = kMb[R];
    constexpr int N = kNB * Z;
    constexpr int G = THREADS / Z;
    constexpr int BUF = 24 * THREADS;          /* floats per buffer set (all slots) */
    static_assert(G >= 1 && G <= kMixedMaxSlots, "slots per CTA");
    static_assert(kMixedMaxChunk <= THREADS, "one thread per frame of an item");
    const int tid = threadIdx.x;
    const int g = tid / Z;
    const int r = tid - g * Z;
    const bool in_slot = g < G;

    /* issue the bulk copy of the item's j-th frame into buffer b of slot q (thread 0) */
    auto fetch = [&](int q, int b, int j) {
        const long long off = S.olist[j];
        S.pre[q] = S.flist[j];
        S.off_pre[q] = off;
        fence_proxy_async_smem();   /* earlier generic reads of that buffer come first */
        mbar_arrive_expect_tx(&bar[b][q], (uint32_t)(N * 4));
        bulk_g2s(smem + b * BUF + q * N, a.llr + off, (uint32_t)(N * 4), &bar[b][q]);
    };

    /* the item's frame list and offsets into shared memory, one per thread */
    if (tid < item.count) {
        const int f = a.perm[item.start + tid];
        S.flist[tid] = f;
        S.olist[tid] = a.offset[f];
    }
    __syncthreads();
    if (tid == 0) {
        S.next = 0;
        S.abort = 0;
        for (int q = 0; q < G; q++) {
            S.frame[q] = -1;
            S.pre[q] = -1;
            const int b = ((S.cur >> q) & 1u) ^ 1u;
            if (S.next < item.count) fetch(q, b, S.next++);
        }
    }
    __syncthreads();

    /* messages: registers (every index a compile-time constant), or shared
     * memory after the two buffer sets, [3][kMaxMb][THREADS] */
    float rM1[MB], rM2[MB];
    uint32_t rNEG[MB];
    float* const sM1 = smem + 2 * BUF + tid;
    float* const sM2 = sM1 + kMaxMb * THREADS;
    uint32_t* const sNEG = reinterpret_cast<uint32_t*>(sM2 + kMaxMb * THREADS);

    int frame = -1, iters = 0;
    long long off = 0;
    bool need_check = false;
    float* P = smem;

    while (true) {
        /* 1. slots that are empty and have a prefetched frame: wait for its copy */
        const int my_pre = in_slot ? S.pre[g] : -1;
        if (in_slot && frame < 0 && my_pre >= 0) {
            const int b = ((S.cur >> g) & 1u) ^ 1u;
            if (!mbar_wait_bounded(&bar[b][g], (S.phase >> (8 * b + g)) & 1u)) atomicOr(&S.abort, 1u);
        }
        __syncthreads();
        if (S.abort) break;
        if (tid == 0) {
            unsigned fresh = 0;
            for (int q = 0; q < G; q++) {
                if (S.frame[q] >= 0 || S.pre[q] < 0) continue;
                const int b = ((S.cur >> q) & 1u) ^ 1u;
                S.phase ^= 1u << (8 * b + q);
                S.cur ^= 1u << q;
                S.frame[q] = S.pre[q];
                S.off_cur[q] = S.off_pre[q];
                S.pre[q] = -1;
                fresh |= 1u << q;
                if (S.next < item.count) fetch(q, b ^ 1, S.next++);
            }
            S.fresh = fresh;
            S.fail = 0;
        }
        __syncthreads();
        if (in_slot && ((S.fresh >> g) & 1u)) {
            frame = S.frame[g];
            off = S.off_cur[g];
            P = smem + ((S.cur >> g) & 1u) * BUF + g * N;
            iters = 0;
            need_check = true;
            static_for<MB>([&](auto I) {
                constexpr int i = decltype(I)::value;
                if constexpr (LAYOUT == kMsgRegisters) {
                    rM1[i] = 0.0f;
                    rM2[i] = 0.0f;
                    rNEG[i] = 0u;
                } else {
                    sM1[i * THREADS] = 0.0f;
                    sM2[i * THREADS] = 0.0f;
                    sNEG[i * THREADS] = 0u;
                }
            });
        }
        float* const Pr = P + r;
        float* const Prz = Pr - Z;

        /* 2. syndrome of the slots loaded or iterated since their last check */
        if (in_slot && frame >= 0 && need_check) {
            const unsigned fail = tdmp_rows_fail<R>([&](auto I, auto E) {
                return edge_ptr<R, Z, decltype(I)::value, decltype(E)::value>(Pr, Prz, r);
            });
            if (fail) atomicOr(&S.fail, 1u << g);
        }
        __syncthreads();

        /* 3. retire converged frames and frames at the cap: outputs from shared memory */
        if (in_slot && frame >= 0 && need_check) {
            need_check = false;
            const bool failed = (S.fail >> g) & 1u;
            if (!failed || iters >= a.max_iter) {
#pragma unroll
                for (int s = 0; s < 6; s++) {
                    const int v = r + s * Z;                  /* float4 group of the frame */
                    const float4 p = reinterpret_cast<const float4*>(P)[v];
                    const uint32_t w = (p.x >= 0.0f ? 1u : 0u) | (p.y >= 0.0f ? 1u << 8 : 0u) |
                                       (p.z >= 0.0f ? 1u << 16 : 0u) | (p.w >= 0.0f ? 1u << 24 : 0u);
                    reinterpret_cast<uint32_t*>(a.hard + off)[v] = w;
                    if (a.post) reinterpret_cast<float4*>(a.post + off)[v] = p;
                }
                if (r == 0) {
                    if (a.status) a.status[frame] = iters | ((failed ? 1 : 0) << 16);
                    S.frame[g] = -1;
                }
                frame = -1;
            }
        }
        __syncthreads();

        /* 4. done when every slot is empty and nothing is in flight; an empty
         * slot with a prefetched frame is refilled before the next iteration */
        bool all_empty = true, refill = false;
        for (int q = 0; q < G; q++) {
            all_empty &= S.frame[q] < 0 && S.pre[q] < 0;
            refill |= S.frame[q] < 0 && S.pre[q] >= 0;
        }
        if (all_empty) break;
        if (refill) continue;

        /* 5. one iteration of every occupied slot (all of them failed their check) */
        const bool active = in_slot && frame >= 0;
        static_for<MB>([&](auto I) {
            constexpr int i = decltype(I)::value;
            if (active) {
                auto at = [&](auto E) { return edge_ptr<R, Z, i, decltype(E)::value>(Pr, Prz, r); };
                if constexpr (LAYOUT == kMsgRegisters) {
                    tdmp_layer<R, i, kNms>(at, rM1[i], rM2[i], rNEG[i]);
                } else {
                    float a1 = sM1[i * THREADS], a2 = sM2[i * THREADS];
                    uint32_t ng = sNEG[i * THREADS];
                    tdmp_layer<R, i, kNms>(at, a1, a2, ng);
                    sM1[i * THREADS] = a1;
                    sM2[i * THREADS] = a2;
                    sNEG[i * THREADS] = ng;
                }
            }
            __syncthreads();
        });
        if (active) {
            iters++;
            need_check = true;
        }
    }
    if (S.abort) {
        /* a staging wait expired: record it, let every copy in flight land, stop */
        if (tid == 0) {
            atomicOr(a.err, kErrWaitTimeout);
            for (int q = 0; q < G; q++)
                if (S.pre[q] >= 0) {
                    const int b = ((S.cur >> q) & 1u) ^ 1u;
                    mbar_wait_bounded(&bar[b][q], (S.phase >> (8 * b + q)) & 1u);
                }
        }
        return false;
    }
    return true;
}

/* One persistent grid per rate: items of any z of rate R, each decoded by the
 * body specialised on its z. */
template <int R, int THREADS, int LAYOUT>
__global__ void __launch_bounds__(THREADS, (MixedOcc<THREADS, LAYOUT>::MIN_CTAS))
mixed_decode_kernel(const __grid_constant__ MixedArgs a)
{
    MixedCtl& S = g_mixed_ctl;
    if (threadIdx.x == 0) {
        for (int b = 0; b < 2; b++)
            for (int q = 0; q < kMixedMaxSlots; q++) mbar_init(&g_mixed_bar[b][q], 1);
        fence_mbar_init();
        S.cur = 0xffffffffu;     /* first frames go into buffer 0 */
        S.phase = 0;
    }
    const MixedItem* items = a.items + (long long)R * a.items_per_rate;
    while (true) {
        if (threadIdx.x == 0) S.item = atomicAdd(&a.queue[R], 1);
        __syncthreads();
        const int k = S.item;
        __syncthreads();
        if (k >= a.num_items[R]) break;
        const MixedItem it = items[k];
        const int zi = it.variant - R * kNumZ;
        bool ok = true;
        static_for<kNumZ>([&](auto ZI) {
            constexpr int zi_c = decltype(ZI)::value;
            if (zi == zi_c) ok = mixed_item<R, kZMin + kZStep * zi_c, THREADS, LAYOUT>(a, it);
        });
        if (!ok) break;
        __syncthreads();
    }
}

}  // namespace wldpc

#endif
