/*
 * The persistent mixed-code decode kernel (mixed.cuh): one grid per code
 * rate takes work items (up to `chunk` frames of one (rate, z)) from its
 * rate's queue. z is a run-time value, so one kernel body serves all 19 z of
 * its rate: every thread's edge addresses for the item's code go into a
 * shared-memory table once per item (one 16-bit load per edge afterwards).
 * A body specialised on z per item kept every address a compile-time
 * constant, but 19 such bodies per kernel overflowed the instruction caches
 * (ncu: 10 no_instruction stalls per issue, issue 16% active) and ran 1.7x
 * slower on the mixed batch.
 *
 * Within an item the CTA runs G = THREADS * RPT / z frame slots in lockstep,
 * z / RPT threads per frame (threads per z: RPT = 1 or 2 expanded rows per
 * thread; a thread's two rows are r and r + z/2, two independent chains of
 * the same layer), and refills a slot as soon as its frame converges or
 * reaches the cap (early-exit compaction). A refilled frame arrives by one
 * cp.async.bulk copy (TMA, no multicast) completed on the slot's mbarrier,
 * and gets its initial syndrome check before its first iteration (reference
 * lib/ldpc_decoder.cc:127-139). The item's frame list and offsets are staged
 * in shared memory at its start, so a refill reads no global memory.
 *
 * LAYOUT selects where a thread's compressed messages (M1, M2, NEG per
 * layer and row) live: in registers, or in shared memory. The arithmetic is the
 * plain normalized min-sum of tdmp_layer(), bit-exact with the reference.
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

/* resident CTAs per SM the register allocation is sized for. One row per
 * thread: 80 registers (the kernel is latency-bound, so resident warps pay
 * more than the few spills of the rate-5/6 kernel cost), and shared memory
 * fits as many CTAs. Two rows per thread: twice the shared memory per
 * thread, so half the CTAs fit, which leaves up to 168 registers. */
template <int THREADS, int RPT>
struct MixedOcc {
    static constexpr int MIN_CTAS = (THREADS == 96 ? 8 : 4) / RPT;
};

/* dynamic shared memory of a CTA of the rate's kernel: the posteriors (24
 * floats per row), the 16-bit address table (one entry per non-zero block
 * per row) and, in the shared layout, the messages (3 words per layer per
 * row); RPT rows per thread. Sized per rate, so 8 CTAs of 96 threads (one
 * row each) fit an SM's 228 KB. */
constexpr int mixed_smem_bytes(int threads, int layout, int rate, int rpt)
{
    return (24 * threads * 4 + num_blocks(rate) * threads * 2 +
            (layout == kMsgShared ? 3 * kMb[rate] * threads * 4 : 0)) * rpt;
}

struct MixedCtl {
    int flist[kMixedMaxChunk];       /* the item's frames, in decode order */
    long long olist[kMixedMaxChunk]; /* and their LLR offsets */
    int frame[kMixedMaxSlots];       /* frame of each slot, -1 = empty */
    long long off[kMixedMaxSlots];
    unsigned phase;                  /* bit q: parity the next wait on bar[q] expects */
    unsigned fresh, fail, abort;
    int next;                        /* frames of the item handed out */
    int item;
};

template <int R, int THREADS, int LAYOUT, int RPT>
__device__ __forceinline__ bool mixed_item(const MixedArgs& a, const MixedItem item, float* smem, MixedCtl& S,
                                           uint64_t* bar)
{
    static_assert(RPT == 1 || RPT == 2, "one or two rows per thread");
    constexpr int MB = kMb[R];
    constexpr int NBLK = num_blocks(R);
    const MixedCode& code = a.codes[item.variant - R * kNumZ];
    const int z = code.z, n = code.n;
    const int zt = z / RPT;             /* threads per frame (z is a multiple of 4) */
    const int G = THREADS / zt;
    const int tid = threadIdx.x;
    const int g = tid / zt;
    const int r = tid - g * zt;         /* rows r + k * zt, k < RPT */
    const bool in_slot = g < G;
    float* const P = smem + (in_slot ? g : 0) * n;
    unsigned short* const A = reinterpret_cast<unsigned short*>(smem + 24 * THREADS * RPT);
    /* this thread's edge addresses for the item's code, [row k][block][thread] */
    for (int k = 0; k < RPT; k++)
        for (int b = 0; b < NBLK; b++) {
            int t = r + k * zt + (int)code.shift[b];
            t = t >= z ? t - z : t;
            A[(k * NBLK + b) * THREADS + tid] = in_slot ? (unsigned short)(code.colz[b] + t) : (unsigned short)0;
        }
    auto addr = [&](int k, int b) -> int { return A[(k * NBLK + b) * THREADS + tid]; };
    /* the item's frame list and offsets, one per thread */
    if (tid < item.count) {
        const int f = a.perm[item.start + tid];
        S.flist[tid] = f;
        S.olist[tid] = a.offset[f];
    }
    if (tid == 0) {
        S.next = 0;
        S.abort = 0;
        S.fail = 0;
        for (int q = 0; q < G; q++) S.frame[q] = -1;
    }

    /* messages: registers (every index a compile-time constant), or shared
     * memory after the address table, [row k][3][MB][THREADS] */
    float rM1[RPT][MB], rM2[RPT][MB];
    uint32_t rNEG[RPT][MB];
    static_assert(THREADS % 2 == 0, "the address table must end on a word boundary");
    float* const sM = smem + 24 * THREADS * RPT + NBLK * THREADS * RPT / 2 + tid;
    auto sM1 = [&](int k, int i) -> float& { return sM[(k * 3 * MB + i) * THREADS]; };
    auto sM2 = [&](int k, int i) -> float& { return sM[(k * 3 * MB + MB + i) * THREADS]; };
    auto sNEG = [&](int k, int i) -> uint32_t& {
        return reinterpret_cast<uint32_t*>(sM)[(k * 3 * MB + 2 * MB + i) * THREADS];
    };

    int frame = -1, iters = 0;
    long long off = 0;
    bool need_check = false;
    bool refill = true;   /* uniform: some slot is empty and the item has frames left */
    __syncthreads();

    while (true) {
        /* 1. refill empty slots (only when one is empty, so an iteration without
         * a converged frame costs no barrier here): thread 0 hands out the
         * item's next frames and starts one bulk copy per refilled slot into
         * its posterior buffer */
        if (refill) {
            if (tid == 0) {
                unsigned fresh = 0;
                for (int q = 0; q < G; q++)
                    if (S.frame[q] < 0 && S.next < item.count) {
                        const int j = S.next++;
                        S.frame[q] = S.flist[j];
                        S.off[q] = S.olist[j];
                        fresh |= 1u << q;
                        fence_proxy_async_smem();   /* the slot's earlier generic reads come first */
                        mbar_arrive_expect_tx(&bar[q], (uint32_t)(n * 4));
                        bulk_g2s(smem + q * n, a.llr + S.olist[j], (uint32_t)(n * 4), &bar[q]);
                    }
                S.fresh = fresh;
            }
            __syncthreads();
            if (in_slot && ((S.fresh >> g) & 1u)) {
                frame = S.frame[g];
                off = S.off[g];
                iters = 0;
                need_check = true;
                if (!mbar_wait_bounded(&bar[g], (S.phase >> g) & 1u)) atomicOr(&S.abort, 1u);
#pragma unroll
                for (int k = 0; k < RPT; k++)
                    static_for<MB>([&](auto I) {
                        constexpr int i = decltype(I)::value;
                        if constexpr (LAYOUT == kMsgRegisters) {
                            rM1[k][i] = 0.0f;
                            rM2[k][i] = 0.0f;
                            rNEG[k][i] = 0u;
                        } else {
                            sM1(k, i) = 0.0f;
                            sM2(k, i) = 0.0f;
                            sNEG(k, i) = 0u;
                        }
                    });
            }
            __syncthreads();
            if (S.abort) break;
            if (tid == 0) S.phase ^= S.fresh;   /* every refilled slot's barrier completed one phase */
        }

        /* 2. syndrome of the slots loaded or iterated since their last check;
         * a slot whose last layer already failed in step 5 (bit g of S.fail,
         * set before that step's last barrier) needs no full check */
        if (in_slot && frame >= 0 && need_check && !((*(volatile unsigned*)&S.fail >> g) & 1u)) {
            unsigned fail = 0;
#pragma unroll
            for (int k = 0; k < RPT; k++)
                fail |= tdmp_rows_fail<R>([&](auto I, auto E) {
                    return P + addr(k, block_index(R, decltype(I)::value, decltype(E)::value));
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
                for (int s = 0; s < 6 * RPT; s++) {
                    const int v = r + s * zt;                 /* float4 group of the frame (6z of them) */
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

        /* 4. done when every slot is empty and no frame is left; an empty
         * slot is refilled before the next iteration while frames remain */
        bool any_empty = false, all_empty = true;
        for (int q = 0; q < G; q++) {
            any_empty |= S.frame[q] < 0;
            all_empty &= S.frame[q] < 0;
        }
        const bool more = S.next < item.count;
        if (tid == 0) S.fail = 0;   /* read in steps 2 and 3, before the barrier above; set again from step 5 on */
        if (all_empty && !more) break;
        refill = any_empty && more;
        if (refill) {
            __syncthreads();        /* these reads come before thread 0's refill writes */
            continue;
        }

        /* 5. one iteration of every occupied slot (all of them failed their
         * check). The last layer's rows also check their parity on the
         * posteriors they write, which no later layer changes in this
         * iteration: a failing one marks its slot in S.fail. */
        const bool active = in_slot && frame >= 0;
        static_for<MB>([&](auto I) {
            constexpr int i = decltype(I)::value;
            constexpr int d = layer_degree(R, i);
            constexpr bool LAST = i == MB - 1;
            if (active) {
                bool last_fail = false;
                /* the layer's rows (independent chains), each with its edge
                 * addresses loaded once for both passes */
#pragma unroll
                for (int k = 0; k < RPT; k++) {
                    int ad[d];
                    static_for<d>([&](auto E) {
                        ad[decltype(E)::value] = addr(k, block_index(R, i, decltype(E)::value));
                    });
                    auto at = [&](auto E) { return P + ad[decltype(E)::value]; };
                    bool odd = false;
                    if constexpr (LAYOUT == kMsgRegisters) {
                        tdmp_layer<R, i, kNms, LAST>(at, rM1[k][i], rM2[k][i], rNEG[k][i], &odd);
                    } else {
                        float a1 = sM1(k, i), a2 = sM2(k, i);
                        uint32_t ng = sNEG(k, i);
                        tdmp_layer<R, i, kNms, LAST>(at, a1, a2, ng, &odd);
                        sM1(k, i) = a1;
                        sM2(k, i) = a2;
                        sNEG(k, i) = ng;
                    }
                    last_fail |= odd;
                }
                if constexpr (LAST) {
                    if (last_fail) atomicOr(&S.fail, 1u << g);
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
        /* a staging wait expired: record it and let every copy in flight land */
        if (tid == 0) {
            atomicOr(a.err, kErrWaitTimeout);
            for (int q = 0; q < G; q++)
                if ((S.fresh >> q) & 1u) mbar_wait_bounded(&bar[q], (S.phase >> q) & 1u);
        }
        return false;
    }
    return true;
}

/* One persistent grid per rate: it takes work items of its rate from its own
 * queue until none are left. */
template <int R, int THREADS, int LAYOUT, int RPT>
__global__ void __launch_bounds__(THREADS, (MixedOcc<THREADS, RPT>::MIN_CTAS))
mixed_decode_kernel(const __grid_constant__ MixedArgs a)
{
    extern __shared__ __align__(128) float smem_mixed[];
    __shared__ __align__(8) uint64_t bar[kMixedMaxSlots];
    __shared__ MixedCtl S;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kMixedMaxSlots; q++) mbar_init(&bar[q], 1);
        fence_mbar_init();
        S.phase = 0;
    }
    const MixedItem* items = a.items + (long long)R * a.items_per_rate;
    while (true) {
        if (threadIdx.x == 0) S.item = atomicAdd(&a.queue[R], 1);
        __syncthreads();
        const int k = S.item;
        __syncthreads();
        if (k >= a.num_items[R]) break;
        if (!mixed_item<R, THREADS, LAYOUT, RPT>(a, items[k], smem_mixed, S, bar)) break;
        __syncthreads();
    }
}

}  // namespace wldpc

#endif
