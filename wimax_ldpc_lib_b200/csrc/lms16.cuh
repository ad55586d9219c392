/*
 * Learned min-sum decoder in packed half precision (f16x2): two frames per
 * thread, one in each 16-bit lane of every register and shared-memory word.
 *
 * The model is the learned decoder's (lms.cuh): per (iteration t, layer i,
 * base column c) a scale a and an offset b, message = s * max(a*mu - b, 0),
 * the layered schedule and stopping rule of the reference decoder
 * (reference lib/ldpc_decoder.cc:122-262, with its compile-time NMS/OMS
 * constants of :17-21,220-231 generalised to trained weights). Here every
 * value is an IEEE binary16 number and every operation rounds to nearest
 * even in binary16; one packed instruction (sub/add/min/max/fma.relu/set)
 * advances both frames, so a frame costs about half the issue slots of the
 * fp32 kernel. The lanes never mix: the outputs of a frame do not depend on
 * its partner.
 *
 * Per frame (a restatement in C is the oracle's wo_learned16_decode_batch):
 *   P[v]  = h(clamp(llr[v], -2048, 2048)), -0 made +0    (input staging)
 *   L_e   = h(P[v_e] - m_e)
 *   m1,m2 = the two smallest |L| of the row, each then min(., 2048)
 *   mu_e  = (|L_e| == m1) ? m2 : m1
 *   m'_e  = s_e * relu(h(a*mu_e - b))                    (one rounding: fma)
 *   P[v_e] = h(L_e + m'_e)
 * with h() rounding to binary16 and s_e the sign the other edges imply
 * (positive LLR = bit 1, so an odd-degree row flips the product of the other
 * signs). Bounds: |llr| <= 2048 and mu <= 2048, and the host accepts only
 * |a| <= 2 and 0 <= b <= 1024, so |m'| <= 4096 and, with at most 6 edges per
 * variable, every posterior stays below 32768: no value overflows. A -0
 * never appears after staging (x - y and x + y give -0 only from a -0
 * operand), so the sign bit of a posterior is its hard decision (x >= 0 is
 * bit 1) and a row's parity is an XOR of sign bits.
 *
 * Early exit per frame: after staging and after every iteration each frame's
 * syndrome is checked; a frame whose syndrome is zero is frozen and its
 * iteration count stops, while its partner decodes on. A frozen lane's
 * messages are set to +0 once and its row minima are masked to 0 in every
 * later layer, so its new messages are s * relu(a*0 - b) = +-0 (b >= 0) and
 * its posteriors are recomputed as (P - 0) + (+-0) = P exactly: they stay as
 * they were when the frame stopped, with no per-edge select. The CTA runs
 * while any of its frames is decoding.
 *
 * Mapping: GP = 32/gcd(z, 32) frame pairs per CTA, so that GP*z threads fill
 * whole warps (z = 96: one pair of 96 threads; z = 48: two pairs; z = 24:
 * four). Thread (g, r) owns row r of every layer of pair g and keeps the
 * messages of its rows, one f16x2 word per non-zero block, in registers;
 * shared memory holds the pairs' posteriors, one f16x2 word per variable.
 * The weights arrive in the kernel parameters as (a, a) and (-b, -b) words.
 */
#ifndef WLDPC_LMS16_CUH
#define WLDPC_LMS16_CUH

#include <cstdint>
#include <cuda_fp16.h>
#include "codes.h"
#include "device_util.cuh"
#include "lms.cuh"
#include "nms_decode.cuh"

namespace wldpc {

constexpr float kLms16Clamp = 2048.0f;          /* input LLR and min-magnitude bound */
constexpr uint32_t kH2Clamp = 0x68006800u;      /* (2048, 2048) in binary16 */
constexpr uint32_t kH2Sign = 0x80008000u;
constexpr float kLms16MaxScale = 2.0f;          /* accepted |a| */
constexpr float kLms16MaxOffset = 1024.0f;      /* accepted b, which must also be >= 0 */

struct Lms16Args {
    const float* llr;       /* frames x n, 16-byte aligned */
    int8_t* hard;           /* frames x n, 4-byte aligned */
    float* post;            /* frames x n or null, 16-byte aligned (may alias llr) */
    int32_t* status;        /* frames or null: iterations | synfail << 16 */
    long long frames;
    int iters;              /* iteration cap */
    int wrows;              /* trained iterations T; iteration t >= T uses row T-1 */
    uint2 wab[kLmsMaxIter][kLmsMaxBlocks];   /* .x = (a, a), .y = (-b, -b) as f16x2 */
};

template <int R, int Z>
struct Lms16Shape {
    static constexpr int MB = kMb[R];
    static constexpr int NBLK = num_blocks(R);
    static constexpr int N = kNB * Z;
    static constexpr int GP = lms_group(Z, N * 4);  /* frame pairs per CTA */
    static constexpr int THREADS = GP * Z;
    static constexpr int FRAMES = 2 * GP;
    static constexpr int SMEM = GP * N * 4;        /* static shared memory (posteriors) */
    /* resident CTAs per SM the register allocation must allow without spills:
     * for 96-thread CTAs, rate 1/2 (degree <= 7) 5 and the higher rates
     * (degree 10-20) 4, scaled down for larger CTAs, and one fewer when a CTA
     * holds four or more pairs (they need more index registers) */
    static constexpr int MIN_CTAS_RAW = (R == 0 ? 480 : 384) / THREADS - (GP >= 4 ? 1 : 0);
    static constexpr int MIN_CTAS = MIN_CTAS_RAW < 1 ? 1 : MIN_CTAS_RAW;
};

/* packed binary16 arithmetic on 32-bit words (lane 0 = low half) */
__device__ __forceinline__ uint32_t h2_sub(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2_add(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2_min(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("min.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t h2_max(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("max.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
/* relu(a*b + c) with one rounding */
__device__ __forceinline__ uint32_t h2_fma_relu(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("fma.rn.relu.f16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
/* 0xffff in each lane where a == b, else 0 */
__device__ __forceinline__ uint32_t h2_eq_mask(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("set.eq.u32.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
/* |a| per lane (an f16x2 abs, which the compiler can fold into the consuming
 * min/max/set as an operand modifier; an integer AND cannot be folded) */
__device__ __forceinline__ uint32_t h2_abs(uint32_t a)
{
    uint32_t d;
    asm("abs.f16x2 %0, %1;" : "=r"(d) : "r"(a));
    return d;
}
/* two floats -> f16x2 (round to nearest even), lane 0 = lo */
__device__ __forceinline__ uint32_t h2_from_floats(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}
__device__ __forceinline__ float h2_lane_to_float(uint32_t w, int lane)
{
    return __half2float(__ushort_as_half((unsigned short)(w >> (16 * lane))));
}
/* per-lane all-ones mask of the lanes in a 2-bit set */
__device__ __forceinline__ uint32_t h2_lanes(unsigned bits)
{
    return ((bits & 1u) ? 0x0000ffffu : 0u) | ((bits & 2u) ? 0xffff0000u : 0u);
}

/* staging of one LLR pair: clamp, round to binary16, -0 -> +0 */
__device__ __forceinline__ uint32_t h2_stage(float x0, float x1)
{
    x0 = fminf(fmaxf(x0, -kLms16Clamp), kLms16Clamp);
    x1 = fminf(fmaxf(x1, -kLms16Clamp), kLms16Clamp);
    return h2_add(h2_from_floats(x0, x1), 0u);
}

/* m1 <= m2: per lane the two smallest of v[LO] .. v[HI-1] (non-negative
 * binary16 values, multiplicity counted), by a balanced tree of min/max;
 * equal to the sequential scan from +inf. */
template <int LO, int HI, int D>
__device__ __forceinline__ void two_min_h2(const uint32_t (&v)[D], uint32_t& m1, uint32_t& m2)
{
    static_assert(HI - LO >= 2, "two_min_h2 needs two values");
    if constexpr (HI - LO == 2) {
        m1 = h2_min(v[LO], v[LO + 1]);
        m2 = h2_max(v[LO], v[LO + 1]);
    } else if constexpr (HI - LO == 3) {
        uint32_t a1, a2;
        two_min_h2<LO, LO + 2>(v, a1, a2);
        const uint32_t c = v[LO + 2];
        m1 = h2_min(a1, c);
        m2 = h2_min(h2_max(a1, c), a2);
    } else {
        constexpr int H = HI - LO;
        constexpr int MID = LO + (H >= 16 ? 8 * (H / 16) : H >= 8 ? 4 * (H / 8) : 2 * (H / 4));
        uint32_t a1, a2, b1, b2;
        two_min_h2<LO, MID>(v, a1, a2);
        if constexpr (HI - MID == 1) {
            const uint32_t c = v[MID];
            m1 = h2_min(a1, c);
            m2 = h2_min(h2_max(a1, c), a2);
        } else {
            two_min_h2<MID, HI>(v, b1, b2);
            m1 = h2_min(a1, b1);
            m2 = h2_min(h2_max(a1, b1), h2_min(a2, b2));
        }
    }
}

template <int R, int Z>
__global__ void __launch_bounds__(Lms16Shape<R, Z>::THREADS, Lms16Shape<R, Z>::MIN_CTAS)
lms16_decode_kernel(const __grid_constant__ Lms16Args a)
{
    using S = Lms16Shape<R, Z>;
    constexpr int MB = S::MB, N = S::N, GP = S::GP, TH = S::THREADS, FR = S::FRAMES;
    constexpr int V4 = N / 4;                 /* groups of 4 variables per frame */
    constexpr int STEPS = GP * V4 / TH;       /* staging / output groups per thread (6) */
    static_assert(GP * V4 % TH == 0, "staging must divide evenly");
    __shared__ __align__(16) uint32_t sP[GP * N];
    __shared__ unsigned s_fail[2], s_last[2], s_half[2];

    const int tid = threadIdx.x;
    const int g = GP == 1 ? 0 : tid / Z;
    const int r = tid - g * Z;
    const long long f0 = (long long)blockIdx.x * FR;
    const long long left = a.frames - f0;
    const int nf = left < FR ? (int)left : FR;
    uint32_t* P = sP + g * N;
    /* edge (I, E) of row r lives at col*Z + (r + s) mod Z: with the two bases
     * P + r and P + r - Z that is one compare and one select per edge, the
     * constant col*Z + s folding into the shared-memory access */
    float* const Pr = reinterpret_cast<float*>(P) + r;
    float* const Prz = Pr - Z;
    auto at = [&](auto I, auto E) -> uint32_t* {
        return reinterpret_cast<uint32_t*>(edge_ptr<R, Z, decltype(I)::value, decltype(E)::value>(Pr, Prz, r));
    };

    if (tid == 0) {
        s_fail[0] = 0;
        s_fail[1] = 0;
        s_last[0] = 0;
        s_last[1] = 0;
        s_half[0] = 0;
        s_half[1] = 0;
    }
    /* staging: word v of pair q holds variable v of frames 2q (low lane) and
     * 2q+1 (high lane); all loads are issued before the conversions */
    {
        float4 x0[STEPS], x1[STEPS];
#pragma unroll
        for (int s = 0; s < STEPS; s++) {
            const int idx = tid + s * TH;
            const int q = idx / V4, v4 = idx - q * V4;
            const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
            x0[s] = 2 * q < nf ? __ldcs(reinterpret_cast<const float4*>(a.llr + (f0 + 2 * q) * N) + v4) : zero;
            x1[s] = 2 * q + 1 < nf ? __ldcs(reinterpret_cast<const float4*>(a.llr + (f0 + 2 * q + 1) * N) + v4)
                                   : zero;
        }
#pragma unroll
        for (int s = 0; s < STEPS; s++) {
            const int idx = tid + s * TH;
            const int q = idx / V4, v4 = idx - q * V4;
            uint4 w;
            w.x = h2_stage(x0[s].x, x1[s].x);
            w.y = h2_stage(x0[s].y, x1[s].y);
            w.z = h2_stage(x0[s].z, x1[s].z);
            w.w = h2_stage(x0[s].w, x1[s].w);
            reinterpret_cast<uint4*>(sP + q * N)[v4] = w;
        }
    }
    __syncthreads();

    /* sign bit of each lane: set where some row of that frame fails, over
     * layers FIRST .. END-1 */
    auto rows_fail = [&](auto FIRST, auto END) -> uint32_t {
        uint32_t acc = 0;
        static_for<decltype(END)::value - decltype(FIRST)::value>([&](auto I_) {
            using I = std::integral_constant<int, decltype(FIRST)::value + decltype(I_)::value>;
            constexpr int d = layer_degree(R, I::value);
            uint32_t x = (d & 1) ? kH2Sign : 0u;   /* parity of the hard bits: d minus the negatives */
            static_for<d>([&](auto E_) { x ^= *at(I{}, E_); });
            acc |= x;
        });
        return acc & kH2Sign;
    };
    /* CTA-wide failing-frame mask: bit 2g + lane. When TH is not a multiple
     * of 32 the last warp is partial and its reduction covers only its lanes. */
    constexpr unsigned kTailLanes = TH % 32;
    const unsigned wmask = (kTailLanes == 0 || tid < TH - (int)kTailLanes) ? 0xffffffffu : (1u << kTailLanes) - 1u;
    auto frame_fail = [&](uint32_t acc, unsigned* slot) -> unsigned {
        unsigned bits = (((acc >> 15) & 1u) | ((acc >> 30) & 2u)) << (2 * g);
        bits = __reduce_or_sync(wmask, bits);
        if ((tid & 31) == 0 && bits) atomicOr(slot, bits);
        __syncthreads();
        return *slot;
    };

    uint32_t Mr[S::NBLK];
#pragma unroll
    for (int q = 0; q < S::NBLK; q++) Mr[q] = 0u;

    const unsigned live = (2 * g < nf ? 1u : 0u) | (2 * g + 1 < nf ? 2u : 0u);
    /* initial syndrome: layer 0's rows first; only lanes that pass there
     * check the other layers */
    using L0 = std::integral_constant<int, 0>;
    using L1 = std::integral_constant<int, 1>;
    using LM = std::integral_constant<int, MB - 1>;
    using LH = std::integral_constant<int, (MB - 1) / 2>;
    using LE = std::integral_constant<int, MB>;
    unsigned fmask = frame_fail(live ? rows_fail(L0{}, L1{}) & h2_lanes(live) : 0u, &s_last[0]);
    if (((1u << nf) - 1u) & ~fmask) {
        const unsigned chk = live & ~(fmask >> (2 * g)) & 3u;
        fmask |= frame_fail(chk ? rows_fail(L1{}, LE{}) & h2_lanes(chk) : 0u, &s_fail[0]);
    }
    unsigned act = (fmask >> (2 * g)) & 3u;   /* lanes of this pair still decoding */
    int it0 = 0, it1 = 0;

    for (int t = 0; t < a.iters && fmask != 0u; ++t) {
        const int slot = (t + 1) & 1;   /* last read two iterations ago, before many barriers */
        if (tid == 0) {
            s_fail[slot] = 0;
            s_last[slot] = 0;
            s_half[slot] = 0;
        }
        const uint32_t am = h2_lanes(act);     /* lanes still decoding; frozen lanes get mu = 0 */
        const uint2* wab = a.wab[t < a.wrows ? t : a.wrows - 1];
        /* parity of the last layer's row from the posteriors it writes (no
         * later layer changes them in this iteration): sign bit per lane */
        uint32_t last_par = 0;
        static_for<MB>([&](auto I) {
            constexpr int d = layer_degree(R, I);
            constexpr int b0 = block_index(R, I, 0);
            constexpr bool LAST = decltype(I)::value == MB - 1;
            if (act) {
                uint32_t L[d], A[d];
                uint32_t sgn = 0;
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    L[e] = h2_sub(*at(I, E_), Mr[b0 + e]);
                    A[e] = h2_abs(L[e]);
                    sgn ^= L[e];
                });
                uint32_t m1, m2;
                two_min_h2<0, d>(A, m1, m2);
                m1 = h2_min(m1, kH2Clamp) & am;
                m2 = h2_min(m2, kH2Clamp) & am;
                /* positive LLR = bit 1: the extrinsic sign flips on odd-degree rows */
                const uint32_t fb = (sgn ^ ((d & 1) ? kH2Sign : 0u)) & kH2Sign;
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    const uint32_t eq = h2_eq_mask(A[e], m1);
                    const uint32_t mu = (eq & m2) | (~eq & m1);
                    const uint2 ab = wab[b0 + e];
                    const uint32_t mag = h2_fma_relu(ab.x, mu, ab.y);
                    const uint32_t msg = mag | ((L[e] ^ fb) & kH2Sign);
                    Mr[b0 + e] = msg;
                    const uint32_t pn = h2_add(L[e], msg);
                    *at(I, E_) = pn;
                    if constexpr (LAST) last_par ^= pn;
                });
                if constexpr (LAST) last_par = (last_par ^ ((d & 1) ? kH2Sign : 0u)) & kH2Sign;
            }
            if constexpr (!LAST) __syncthreads();
        });
        /* stopping rule: a lane with a failing row in the last layer fails;
         * the other active lanes check the remaining layers in two halves,
         * with a vote after each. The first vote is the last layer's barrier. */
        const unsigned lmask = frame_fail(act ? last_par & h2_lanes(act) : 0u, &s_last[slot]);
        unsigned fm = lmask;
        if (fmask & ~fm) {
            const unsigned chk = act & ~(fm >> (2 * g)) & 3u;
            fm |= frame_fail(chk ? rows_fail(L0{}, LH{}) & h2_lanes(chk) : 0u, &s_fail[slot]);
        }
        if (fmask & ~fm) {
            const unsigned chk = act & ~(fm >> (2 * g)) & 3u;
            fm |= frame_fail(chk ? rows_fail(LH{}, LM{}) & h2_lanes(chk) : 0u, &s_half[slot]);
        }
        fmask = fm;
        if (act & 1u) it0 = t + 1;
        if (act & 2u) it1 = t + 1;
        const unsigned nact = (fmask >> (2 * g)) & 3u;
        if (act & ~nact) {   /* lanes that stopped now: their messages become +0 */
            const uint32_t drop = ~h2_lanes(act & ~nact);
#pragma unroll
            for (int q = 0; q < S::NBLK; q++) Mr[q] &= drop;
        }
        act = nact;
    }

    /* outputs: hard bits (sign clear = bit 1) and the posteriors as floats */
#pragma unroll
    for (int s = 0; s < STEPS; s++) {
        const int idx = tid + s * TH;
        const int q = idx / V4, v4 = idx - q * V4;
        const uint4 w = reinterpret_cast<const uint4*>(sP + q * N)[v4];
#pragma unroll
        for (int lane = 0; lane < 2; lane++) {
            const int fr = 2 * q + lane;
            if (fr >= nf) continue;
            const int sh = 15 + 16 * lane;
            const uint32_t hw = ((~w.x >> sh) & 1u) | (((~w.y >> sh) & 1u) << 8) | (((~w.z >> sh) & 1u) << 16) |
                                (((~w.w >> sh) & 1u) << 24);
            reinterpret_cast<uint32_t*>(a.hard + (f0 + fr) * N)[v4] = hw;
            if (a.post)
                reinterpret_cast<float4*>(a.post + (f0 + fr) * N)[v4] =
                    make_float4(h2_lane_to_float(w.x, lane), h2_lane_to_float(w.y, lane),
                                h2_lane_to_float(w.z, lane), h2_lane_to_float(w.w, lane));
        }
    }
    if (a.status && r == 0) {
        if (live & 1u) a.status[f0 + 2 * g] = it0 | ((act & 1u) ? 1 << 16 : 0);
        if (live & 2u) a.status[f0 + 2 * g + 1] = it1 | ((act & 2u) ? 1 << 16 : 0);
    }
}

}  // namespace wldpc

#endif
