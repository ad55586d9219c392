/*
 * Learned (neural) normalized/offset min-sum: decoder, training forward /
 * backward, and Adam, for sm_100a.
 *
 * The model generalises the reference's two min-sum flavours (reference
 * lib/ldpc_decoder.cc:17-21,220-231: message = s * min * 0.815, or
 * s * max(min - 0.10, 0)) to one scale a and one offset b per (iteration t,
 * layer i, base column c):
 *
 *   L_e   = P[v_e] - m_e                       (float)
 *   mu_e  = min over the other edges of |L|    (min1 / min2 from +inf)
 *   m'_e  = s_e * max(a[t,i,c_e] * mu_e - b[t,i,c_e], 0)      (fmaf)
 *   P[v_e] = L_e + m'_e
 *
 * with s_e the sign the other edges imply (sign bit = signbit; positive LLR =
 * bit 1, so an odd-degree row flips the product of the other signs) applied
 * as a product with +-1.0 (the reference's MS form s * min; it flips the
 * sign bit of the magnitude exactly, signed zeros included), the
 * same layered schedule as the plain decoder, T <= 8 trained iterations
 * (a decoder may run past T with the weights of iteration T-1), and
 * the reference's stopping rule (slice x >= 0, stop at a zero syndrome).
 * Weights a = 0.815, b = 0 give a float normalized min-sum.
 *
 * Messages: the decoder keeps every edge's message in a register of the
 * thread that owns the edge's row (one per non-zero block: 76 to 88), so
 * pass 1 reads the old message without a load and without recomputing it
 * from compressed state and the previous iteration's weights; shared memory
 * holds only the posteriors. The weights are read from the kernel
 * parameters as (a, b) pairs (staging them in shared memory measured 21%
 * slower). The sign
 * parity is an XOR of the L words and the two minima come from a balanced
 * tree. All arithmetic is fp32.
 *
 * Training (one frame per CTA of z threads): the forward pass runs all T
 * iterations, stores the posterior and the messages at every iteration
 * boundary (checkpoints) and the BCE loss mean over iterations, bits and
 * frames (positive LLR = bit 1: loss = softplus(sg * P), sg = +1 for bit 0,
 * -1 for bit 1). The backward pass walks the iterations in reverse: it
 * restores iteration t's inputs from the checkpoints, recomputes its forward
 * keeping every edge's L, and back-propagates through its layers in reverse.
 * Subgradients: sign() and the argmin choice are constant, d|x|/dx = sign(x),
 * relu'(0) = 0; edge e != i1 takes its magnitude from i1 (the first edge with
 * |L| == min1), edge i1 from i2 (the first other edge with |L| == min2).
 * Per-CTA weight gradients go to a per-frame partial array; a second kernel
 * reduces them in a fixed order (deterministic) and applies Adam.
 */
#ifndef WLDPC_LMS_CUH
#define WLDPC_LMS_CUH

#include <cstdint>
#include "codes.h"
#include "device_util.cuh"
#include "nms_decode.cuh"

namespace wldpc {

constexpr int kLmsMaxIter = 8;
constexpr int kLmsMaxBlocks = 96;

/* Weights per (iteration, non-zero block): blocks in row-major base-matrix
 * order, so block b of layer i has column layer_col(rate, i, e). */
struct LmsWeights {
    float a[kLmsMaxIter][kLmsMaxBlocks];
    float b[kLmsMaxIter][kLmsMaxBlocks];
};

struct LmsArgs {
    const float* llr;       /* frames x n, 16-byte aligned */
    int8_t* hard;           /* frames x n, 4-byte aligned */
    float* post;            /* frames x n or null */
    int32_t* status;        /* frames or null: iterations | synfail << 16 */
    unsigned* err;
    long long frames;
    int iters;              /* iteration cap */
    int wrows;              /* trained iterations T <= kLmsMaxIter; iteration t >= T uses row T-1 */
    unsigned wait_limit_us = kWaitLimitUs;   /* bound of the staging wait (the drain wait after a timeout is full) */
    float2 wab[kLmsMaxIter][kLmsMaxBlocks];   /* (a, b) per (iteration, block): one 8-byte load per edge */
};

/* Frames (or frame pairs) per CTA for the learned decoders: 32/gcd(z, 32)
 * of them make the CTA a whole number of warps; while that would exceed 384
 * threads (the register file must hold a few such CTAs at ~128 registers per
 * thread) or 100 KB of posteriors, halve it (the last warp is then partial). */
constexpr int lms_group(int z, int frame_bytes)
{
    int g = 32 / gcd_c(z, 32);
    while (g > 1 && (g * z > 384 || g * frame_bytes > 100 * 1024)) g /= 2;
    return g;
}

template <int R, int Z>
struct LmsShape {
    static constexpr int MB = kMb[R];
    static constexpr int NBLK = num_blocks(R);
    static constexpr int N = kNB * Z;
    static constexpr int E = NBLK * Z;
    static constexpr int G = lms_group(Z, N * 4);   /* frames per CTA */
    static constexpr int THREADS = G * Z;
    static constexpr int SMEM = G * N * 4;
};

/* ------------------------------------------------------------ inference */

/* Edge addressing of the fp32 decoder: the index col*z + (r + s) mod z
 * (edge_var_c) where that measured faster on a B200 (by 1-18%; all 114 codes
 * timed, outputs identical), else a pointer chosen by one compare and select
 * (edge_ptr), which was up to 8% faster on the others. */
constexpr bool lms_index_addressing(int R, int Z)
{
    switch (R) {
    case 0: return Z == 68;
    case 1: return Z == 40 || Z == 96;
    case 2: return Z == 80;
    case 3: return Z == 64 || Z == 96;
    case 4: return Z == 64 || Z == 96;
    default: return Z == 80 || Z == 96;
    }
}

template <int R, int Z, int I, int E>
__device__ __forceinline__ float* lms_edge(float* P, float* Pr, float* Prz, int r)
{
    if constexpr (lms_index_addressing(R, Z))
        return P + edge_var_c<R, Z, I, E>(r);
    else
        return edge_ptr<R, Z, I, E>(Pr, Prz, r);
}

template <int R, int Z>
__global__ void __launch_bounds__(LmsShape<R, Z>::THREADS)
lms_decode_kernel(const __grid_constant__ LmsArgs a)
{
    using S = LmsShape<R, Z>;
    constexpr int MB = S::MB, N = S::N, G = S::G;
    extern __shared__ __align__(128) float smem_lms[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned s_fail[2], s_last[2], s_half[2];

    const int tid = threadIdx.x;
    const int g = G == 1 ? 0 : tid / Z;
    const int r = tid - g * Z;
    const long long f0 = (long long)blockIdx.x * G;
    const long long left = a.frames - f0;
    const int nf = left < G ? (int)left : G;
    float* P = smem_lms + g * N;                 /* posteriors of frame g */
    float* const Pr = P + r;                     /* lms_edge bases */
    float* const Prz = Pr - Z;

    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        s_fail[0] = 0;
        s_fail[1] = 0;
        s_last[0] = 0;
        s_last[1] = 0;
        s_half[0] = 0;
        s_half[1] = 0;
        const uint32_t bytes = (uint32_t)(nf * N * 4);
        mbar_arrive_expect_tx(&bar, bytes);
        bulk_g2s(smem_lms, a.llr + f0 * N, bytes, &bar);
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, a.wait_limit_us);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            atomicOr(a.err, kErrWaitTimeout);
            mbar_wait_bounded(&bar, 0, kWaitLimitUs);   /* let an in-flight copy land before exit */
        }
        return;
    }

    /* syndrome of the thread's rows in layers FIRST .. END-1: 1 if any fails */
    auto rows_fail = [&](auto FIRST, auto END) -> unsigned {
        unsigned fail = 0;
        static_for<decltype(END)::value - decltype(FIRST)::value>([&](auto I_) {
            using I = std::integral_constant<int, decltype(FIRST)::value + decltype(I_)::value>;
            constexpr int d = layer_degree(R, I::value);
            bool odd = (d & 1) != 0;   /* parity of the hard bits: d minus the negatives */
            static_for<d>([&](auto E_) {
                odd = odd != (*lms_edge<R, Z, I::value, E_>(P, Pr, Prz, r) < 0.0f);
            });
            fail |= odd ? 1u : 0u;
        });
        return fail;
    };
    /* per-frame OR over the CTA (bit g: frame g); one barrier */
    auto frame_fail = [&](unsigned fail, unsigned* slot) -> unsigned {
        if constexpr (G == 1) {
            return __syncthreads_or((int)fail) ? 1u : 0u;
        } else {
            if (fail) atomicOr(slot, 1u << g);
            __syncthreads();
            return *slot;
        }
    };

    /* this thread's check-to-variable messages, one per block (its row of every
     * layer), in registers: every index is a compile-time constant */
    float Mr[S::NBLK];
#pragma unroll
    for (int q = 0; q < S::NBLK; q++) Mr[q] = 0.0f;

    /* initial syndrome (reference lib/ldpc_decoder.cc:127-139): layer 0's
     * rows first; only frames that pass there check the other layers */
    using L0 = std::integral_constant<int, 0>;
    using L1 = std::integral_constant<int, 1>;
    using LM = std::integral_constant<int, MB - 1>;
    using LH = std::integral_constant<int, (MB - 1) / 2>;
    using LE = std::integral_constant<int, MB>;
    const bool live = g < nf;
    const unsigned lives = (1u << nf) - 1u;
    unsigned fmask = frame_fail(live ? rows_fail(L0{}, L1{}) : 0u, &s_last[0]);
    if (lives & ~fmask)
        fmask |= frame_fail(live && !((fmask >> g) & 1u) ? rows_fail(L1{}, LE{}) : 0u, &s_fail[0]);
    bool active = live && ((fmask >> g) & 1u);
    int iters = 0;

    for (int t = 0; t < a.iters && fmask != 0u; ++t) {
        const int slot = (t + 1) & 1;   /* read last two iterations ago, before many barriers */
        if constexpr (G > 1) {
            if (tid == 0) {
                s_fail[slot] = 0;
                s_last[slot] = 0;
                s_half[slot] = 0;
            }
        }
        /* parity of the last layer's row from the posteriors it writes: no
         * later layer changes them in this iteration, so they are final */
        bool last_odd = false;
        /* this iteration's (a, b) pairs: the same address in every thread */
        const float2* const wab = a.wab[t < a.wrows ? t : a.wrows - 1];
        static_for<MB>([&](auto I) {
            constexpr int d = layer_degree(R, I);
            constexpr int b0 = block_index(R, I, 0);
            constexpr bool LAST = decltype(I)::value == MB - 1;
            if (active) {
                float L[d];
                uint32_t sgn = 0;
                float m1, m2;
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    const float x = *lms_edge<R, Z, I, e>(P, Pr, Prz, r);
                    const float l = __fsub_rn(x, Mr[b0 + e]);
                    L[e] = l;
                    sgn ^= __float_as_uint(l);   /* bit 31: parity of the negative L */
                });
                two_min_abs<0, d>(L, m1, m2);
                /* positive LLR = bit 1: the extrinsic sign flips on odd-degree rows */
                const uint32_t fb = (sgn ^ ((uint32_t)(d & 1) << 31)) & 0x80000000u;
                const uint32_t fbo = fb | 0x3f800000u;   /* with sign(L_e): +-1.0 */
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    const float l = L[e];
                    const float mu = (fabsf(l) == m1) ? m2 : m1;
                    const float2 ab = wab[b0 + e];
                    const float mag = fmaxf(__fmaf_rn(ab.x, mu, -ab.y), 0.0f);
                    const float msg = __fmul_rn(mag, __uint_as_float((__float_as_uint(l) & 0x80000000u) ^ fbo));
                    Mr[b0 + e] = msg;
                    const float pn = __fadd_rn(l, msg);
                    *lms_edge<R, Z, I, e>(P, Pr, Prz, r) = pn;
                    if constexpr (LAST) last_odd = last_odd != (pn < 0.0f);
                });
                if constexpr (LAST) last_odd = last_odd != ((d & 1) != 0);
            }
            if constexpr (!LAST) __syncthreads();
        });
        /* stopping rule (zero syndrome over every row): a frame with a failing
         * row in the last layer fails; the other active frames check the
         * remaining layers in two halves, with a vote after each (a frame that
         * fails in the first half skips the second). The first vote is the last
         * layer's barrier. */
        const unsigned lmask = frame_fail(active && last_odd ? 1u : 0u, &s_last[slot]);
        unsigned fm = lmask;
        if (fmask & ~fm)
            fm |= frame_fail(active && !((fm >> g) & 1u) ? rows_fail(L0{}, LH{}) : 0u, &s_fail[slot]);
        if (fmask & ~fm)
            fm |= frame_fail(active && !((fm >> g) & 1u) ? rows_fail(LH{}, LM{}) : 0u, &s_half[slot]);
        fmask = fm;
        if (active) {
            iters = t + 1;
            active = (fmask >> g) & 1u;
        }
    }

    const int total = nf * N;
    int8_t* hard = a.hard + f0 * N;
    for (int v = tid * 4; v < total; v += S::THREADS * 4) {
        const float4 p = *reinterpret_cast<const float4*>(smem_lms + v);
        const uint32_t wv = (p.x >= 0.0f ? 1u : 0u) | (p.y >= 0.0f ? 1u << 8 : 0u) |
                            (p.z >= 0.0f ? 1u << 16 : 0u) | (p.w >= 0.0f ? 1u << 24 : 0u);
        *reinterpret_cast<uint32_t*>(hard + v) = wv;
        if (a.post) *reinterpret_cast<float4*>(a.post + f0 * N + v) = p;
    }
    if (a.status && live && r == 0) a.status[f0 + g] = iters | ((active ? 1 : 0) << 16);
}

/* ------------------------------------------------------------- training */

struct LmsTrainArgs {
    const float* llr;       /* frames x n */
    const uint8_t* cw;      /* frames x n transmitted bits (0/1) */
    float* ck_post;         /* frames x T x n: posterior after iteration t */
    float* ck_msg;          /* frames x (T-1) x E: messages after iteration t */
    float* gpart;           /* frames x 2 x T x NBLK: per-frame weight gradient */
    float* loss_part;       /* frames: per-frame loss */
    const float* wa;        /* T x NBLK scales (device) */
    const float* wb;        /* T x NBLK offsets (device) */
    long long frames;
    int iters;              /* T */
    float inv_norm;         /* 1 / (T * n * frames) */
};

__device__ __forceinline__ float softplus_f(float x) { return x > 0.0f ? x + log1pf(__expf(-x)) : log1pf(__expf(x)); }
__device__ __forceinline__ float sigmoid_f(float x) { return 1.0f / (1.0f + __expf(-x)); }

template <int R, int Z>
struct LmsTrainShape {
    static constexpr int MB = kMb[R];
    static constexpr int NBLK = num_blocks(R);
    static constexpr int N = kNB * Z;
    static constexpr int E = NBLK * Z;
    /* P, M, L, gP, gM and the CTA's weight gradient */
    static constexpr int SMEM = (2 * N + 3 * E + 2 * kLmsMaxIter * NBLK) * 4;
};

/* one layer of one iteration; optionally records L per edge */
template <int R, int Z, int I, bool RECORD>
__device__ __forceinline__ void lms_layer(float* P, float* M, float* Ls, const float* wa, const float* wb, int r)
{
    constexpr int d = layer_degree(R, I);
    constexpr int b0 = block_index(R, I, 0);
    float L[d];
    uint32_t sgn = 0;
    float m1 = __int_as_float(0x7f800000), m2 = __int_as_float(0x7f800000);
    static_for<d>([&](auto E_) {
        constexpr int e = decltype(E_)::value;
        const float l = __fsub_rn(P[edge_var_c<R, Z, I, e>(r)], M[(b0 + e) * Z + r]);
        L[e] = l;
        if constexpr (RECORD) Ls[(b0 + e) * Z + r] = l;
        sgn = __funnelshift_l(__float_as_uint(l), sgn, 1);
        const float al = fabsf(l);
        m2 = fminf(m2, fmaxf(m1, al));
        m1 = fminf(m1, al);
    });
    const uint32_t fbo = ((uint32_t)((__popc(sgn) & 1) ^ (d & 1)) << 31) | 0x3f800000u;
    static_for<d>([&](auto E_) {
        constexpr int e = decltype(E_)::value;
        const float l = L[e];
        const float mu = (fabsf(l) == m1) ? m2 : m1;
        const float mag = fmaxf(__fmaf_rn(wa[b0 + e], mu, -wb[b0 + e]), 0.0f);
        const float msg = __fmul_rn(mag, __uint_as_float((__float_as_uint(l) & 0x80000000u) ^ fbo));
        M[(b0 + e) * Z + r] = msg;
        P[edge_var_c<R, Z, I, e>(r)] = __fadd_rn(l, msg);
    });
}

template <int R, int Z>
__global__ void __launch_bounds__(Z)
lms_train_kernel(const __grid_constant__ LmsTrainArgs a)
{
    using S = LmsTrainShape<R, Z>;
    constexpr int MB = S::MB, N = S::N, E = S::E, NBLK = S::NBLK;
    extern __shared__ __align__(128) float smem_tr[];
    float* P = smem_tr;
    float* gP = P + N;
    float* M = gP + N;
    float* Ls = M + E;
    float* gM = Ls + E;
    float* gW = gM + E;                          /* [2][T][NBLK] */
    __shared__ float s_red[32];

    const int r = threadIdx.x;
    const long long f = blockIdx.x;
    if (f >= a.frames) return;
    const int T = a.iters;
    const float* llr = a.llr + f * N;
    const uint8_t* cw = a.cw + f * N;
    float* ckp = a.ck_post + f * (long long)T * N;
    float* ckm = a.ck_msg + f * (long long)(T > 1 ? T - 1 : 0) * E;

    for (int q = r; q < N; q += Z) { P[q] = llr[q]; gP[q] = 0.0f; }
    for (int q = r; q < E; q += Z) { M[q] = 0.0f; gM[q] = 0.0f; }
    for (int q = r; q < 2 * T * NBLK; q += Z) gW[q] = 0.0f;
    __syncthreads();

    /* forward: T iterations with checkpoints and the loss */
    float loss = 0.0f;
    for (int t = 0; t < T; t++) {
        static_for<MB>([&](auto I) {
            lms_layer<R, Z, decltype(I)::value, false>(P, M, nullptr, a.wa + t * NBLK, a.wb + t * NBLK, r);
            __syncthreads();
        });
        for (int q = r; q < N; q += Z) {
            const float p = P[q];
            ckp[(long long)t * N + q] = p;
            loss += softplus_f(cw[q] ? -p : p);
        }
        if (t < T - 1)
            for (int q = r; q < E; q += Z) ckm[(long long)t * E + q] = M[q];
    }
    /* block reduction of the loss (per thread into shared memory, then thread 0) */
    for (int q = r; q < 32; q += Z) s_red[q] = 0.0f;
    __syncthreads();
    atomicAdd(&s_red[r & 31], loss);
    __syncthreads();
    if (r == 0) {
        float s = 0.0f;
        for (int q = 0; q < 32; q++) s += s_red[q];
        a.loss_part[f] = s * a.inv_norm;
    }
    __syncthreads();

    /* backward */
    for (int t = T - 1; t >= 0; t--) {
        /* restore the inputs of iteration t and recompute it, keeping L */
        const float* pin = t == 0 ? llr : ckp + (long long)(t - 1) * N;
        for (int q = r; q < N; q += Z) P[q] = pin[q];
        for (int q = r; q < E; q += Z) M[q] = t == 0 ? 0.0f : ckm[(long long)(t - 1) * E + q];
        __syncthreads();
        static_for<MB>([&](auto I) {
            lms_layer<R, Z, decltype(I)::value, true>(P, M, Ls, a.wa + t * NBLK, a.wb + t * NBLK, r);
            __syncthreads();
        });
        /* loss gradient at the end of iteration t */
        for (int q = r; q < N; q += Z) {
            const float p = P[q];
            const float sg = cw[q] ? -1.0f : 1.0f;
            gP[q] += sg * sigmoid_f(sg * p) * a.inv_norm;
        }
        __syncthreads();
        static_for<MB>([&](auto IR) {
            constexpr int I = MB - 1 - decltype(IR)::value;
            constexpr int d = layer_degree(R, I);
            constexpr int b0 = block_index(R, I, 0);
            float L[d], gL[d];
            float m1 = __int_as_float(0x7f800000), m2 = __int_as_float(0x7f800000);
            uint32_t negpar = (uint32_t)(d & 1);   /* odd-degree rows flip the extrinsic sign */
            static_for<d>([&](auto E_) {
                constexpr int e = decltype(E_)::value;
                L[e] = Ls[(b0 + e) * Z + r];
                gL[e] = gP[edge_var_c<R, Z, I, e>(r)];
                negpar ^= __float_as_uint(L[e]) >> 31;
                const float al = fabsf(L[e]);
                m2 = fminf(m2, fmaxf(m1, al));
                m1 = fminf(m1, al);
            });
            int i1 = -1, i2 = -1;
            static_for<d>([&](auto E_) {
                constexpr int e = decltype(E_)::value;
                if (i1 < 0 && fabsf(L[e]) == m1) i1 = e;
            });
            static_for<d>([&](auto E_) {
                constexpr int e = decltype(E_)::value;
                if (i2 < 0 && e != i1 && fabsf(L[e]) == m2) i2 = e;
            });
            float g_to_i1 = 0.0f, g_to_i2 = 0.0f;
            static_for<d>([&](auto E_) {
                constexpr int e = decltype(E_)::value;
                const float l = L[e];
                const bool is_i1 = (e == i1);
                const float mu = (fabsf(l) == m1) ? m2 : m1;
                const float wa = a.wa[t * NBLK + b0 + e], wb = a.wb[t * NBLK + b0 + e];
                const float pre = __fmaf_rn(wa, mu, -wb);
                const float s = ((negpar ^ (__float_as_uint(l) >> 31)) & 1u) ? -1.0f : 1.0f;
                const float G = gL[e] + gM[(b0 + e) * Z + r];
                float ga = 0.0f, gb = 0.0f;
                if (pre > 0.0f) {
                    ga = G * s * mu;
                    gb = -G * s;
                    const float gmu = G * s * wa;
                    if (is_i1) g_to_i2 += gmu;
                    else g_to_i1 += gmu;
                }
                /* reduce over the rows of this block (the CTA's z threads):
                 * whole warps shuffle, a partial last warp adds per thread */
                if constexpr (Z % 32 == 0) {
                    for (int o = 16; o > 0; o >>= 1) {
                        ga += __shfl_xor_sync(0xffffffffu, ga, o);
                        gb += __shfl_xor_sync(0xffffffffu, gb, o);
                    }
                    if ((r & 31) == 0) {
                        atomicAdd(&gW[t * NBLK + b0 + e], ga);
                        atomicAdd(&gW[(T + t) * NBLK + b0 + e], gb);
                    }
                } else if (ga != 0.0f || gb != 0.0f) {
                    atomicAdd(&gW[t * NBLK + b0 + e], ga);
                    atomicAdd(&gW[(T + t) * NBLK + b0 + e], gb);
                }
            });
            static_for<d>([&](auto E_) {
                constexpr int e = decltype(E_)::value;
                const float sgn_l = (__float_as_uint(L[e]) >> 31) ? -1.0f : 1.0f;
                float g = gL[e];
                if (e == i1) g += g_to_i1 * sgn_l;
                if (e == i2) g += g_to_i2 * sgn_l;
                gP[edge_var_c<R, Z, I, e>(r)] = g;
                gM[(b0 + e) * Z + r] = -g;
            });
            __syncthreads();
        });
    }
    for (int q = r; q < 2 * T * NBLK; q += Z) a.gpart[f * 2 * T * NBLK + q] = gW[q];
}

/* Column sums of the per-frame gradients in frame order, then Adam. One
 * thread per weight; w holds a then b, [T][NBLK] each. */
struct AdamArgs {
    const float* gpart;      /* frames x nw */
    const float* loss_part;  /* frames */
    float* grad;             /* nw, written (the reduced gradient) */
    float* w;                /* nw parameters */
    float* m;                /* nw first moments */
    float* v;                /* nw second moments */
    float* loss_out;         /* one float: the batch loss, or null */
    long long frames;
    int nw;
    int step;                /* 1-based Adam step */
    float lr, beta1, beta2, eps;
    int apply;               /* 0: only reduce the gradient */
};

}  // namespace wldpc

#endif
