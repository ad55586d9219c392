/*
 * Plain layered (TDMP) min-sum decoder for sm_100a, bit-exact with the
 * reference ldpc_decoder::decode(float*, int8_t*) (reference
 * lib/ldpc_decoder.cc:122-262), in its three compile-time flavours
 * (reference lib/ldpc_decoder.cc:17-21,215-238):
 *   kNms: message = s * float((double)min * 0.815), posterior added in fp64
 *   kOms: message = s * float(max((double)min - 0.10, 0)), posterior in fp64
 *   kMs : message = s * min, posterior added in fp32
 *
 * Mapping. One CTA decodes G frames, G = 32/gcd(z, 32), so that G*z threads
 * fill whole warps (z = 96: one frame of 96 threads). Thread (g, r) owns
 * expanded row r of every layer of frame g. A layer is one base row; its z rows
 * touch disjoint variables (every block is a z x z circulant), so processing
 * them concurrently is identical to the reference's sequential row order.
 * Layers run in table order with a CTA barrier between them, as the reference.
 *
 * Data. The frame's LLRs are staged global -> shared with one TMA bulk copy
 * and updated in place as the posterior (24z floats). Check-to-variable
 * messages live in registers, either in compressed form per row (the two
 * rounded message magnitudes float(D1), float(D2), the argmin edge and one
 * sign bit per edge) or, for the codes where it measured faster, as one
 * float per edge (tdmp_edge_messages). Circulant shifts are compile-time
 * constants: the address of edge e of row r is col*z + (r + shift) mod z.
 *
 * Arithmetic that must round exactly as the reference (x86, no FMA):
 *   L = post - msg                      float subtract
 *   D = (double)min * 0.815             __dmul_rn (no contraction)
 *   msg' = (float)(+-D)                 __double2float_rn
 *   post' = (float)((double)L +- D)     __dadd_rn then __double2float_rn
 * The sign test is x < 0 (-0.0 is non-negative), which is how the reference's
 * -ffast-math build evaluates std::signbit (reference lib/CMakeLists.txt:6);
 * a canonicalising +0.0f add turns -0.0 into +0.0 before its sign bit is read.
 * min1/min2 track the two smallest |L| starting from 10000.0f (reference
 * lib/ldpc_decoder.cc:150,198); an edge whose |L| equals min1 receives min2,
 * which equals the reference's per-edge recomputation, ties included.
 *
 * Stopping rule (reference lib/ldpc_decoder.cc:127-139,241-251): slice
 * (x >= 0) and check every row after staging and after every iteration; a
 * frame stops at the first zero syndrome. Outputs: hard bits (int8 0/1),
 * optionally the posterior, and status = iterations | synfail << 16.
 */
#ifndef WLDPC_NMS_DECODE_CUH
#define WLDPC_NMS_DECODE_CUH

#include <cstdint>
#include "codes.h"
#include "device_util.cuh"

namespace wldpc {

enum DecodeMode : int { kNms = 0, kOms = 1, kMs = 2 };

struct DecodeArgs {
    const float* llr;       /* frames x n, 16-byte aligned */
    int8_t* hard;           /* frames x n, 4-byte aligned */
    float* post;            /* frames x n or null, 16-byte aligned (may alias llr) */
    int32_t* status;        /* frames or null */
    unsigned* err;          /* error word (kErr*) */
    long long frames;
    int max_iter;
    unsigned wait_limit_us = kWaitLimitUs;   /* bound of the staging wait (the drain wait after a timeout is full) */
    /* used only by the kernels whose z is a run-time value (ZT == 0): */
    int z;
    unsigned short shift[96];   /* per non-zero block, row-major over base rows */
    unsigned short colz[96];    /* block column * z */
};

/* Shape of a TDMP launch. ZT > 0: z is a compile-time constant and a CTA
 * holds G = 32/gcd(z, 32) frames; ZT == 0: z comes from DecodeArgs and a CTA
 * holds one frame of z threads. */
template <int R, int ZT>
struct TdmpShape {
    static constexpr int MB = kMb[R];
    static constexpr int G = ZT > 0 ? 32 / gcd_c(ZT, 32) : 1;
    static constexpr int THREADS = ZT > 0 ? G * ZT : kZMax;
    static constexpr int SMEM = G * kNB * (ZT > 0 ? ZT : kZMax) * 4;
};

/* index of the e-th block of base row i in row-major block order */
constexpr int block_index(int rate, int i, int e)
{
    int b = 0;
    for (int q = 0; q < i; q++) b += layer_degree(rate, q);
    return b + e;
}

/* variable index of edge E of layer I for row r, z a compile-time constant */
template <int R, int Z, int I, int E>
__device__ __forceinline__ int edge_var_c(int r)
{
    constexpr int col = layer_col(R, I, E);
    constexpr int s = layer_shift(R, Z, I, E);
    int t = r + s;
    t = (t >= Z) ? t - Z : t;
    return col * Z + t;
}

/* posterior of edge E of layer I for row r, z a compile-time constant, given
 * Pr = P + r and Prz = P + r - Z: the row's variable is col*Z + (r + s) mod Z,
 * i.e. Pr or Prz (whichever keeps r + s - {0, Z} inside the block) plus the
 * constant col*Z + s, so an edge costs one compare and one select and the
 * constant folds into the shared-memory access */
template <int R, int Z, int I, int E>
__device__ __forceinline__ float* edge_ptr(float* Pr, float* Prz, int r)
{
    constexpr int col = layer_col(R, I, E);
    constexpr int s = layer_shift(R, Z, I, E);
    if constexpr (s == 0) {
        return Pr + col * Z;
    } else {
        return ((r < Z - s) ? Pr : Prz) + (col * Z + s);
    }
}

/* variable index of edge E of layer I for row r */
template <int R, int ZT, int I, int E>
__device__ __forceinline__ int edge_var(int r, const DecodeArgs& a)
{
    if constexpr (ZT > 0) {
        return edge_var_c<R, ZT, I, E>(r);
    } else {
        constexpr int b = block_index(R, I, E);
        int t = r + (int)a.shift[b];
        t = (t >= a.z) ? t - a.z : t;
        return (int)a.colz[b] + t;
    }
}

/* posterior of edge E of layer I for row r: edge_ptr when z is a
 * compile-time constant, else the run-time-z index */
template <int R, int ZT, int I, int E>
__device__ __forceinline__ float* post_ptr(float* P, float* Pr, float* Prz, int r, const DecodeArgs& a)
{
    if constexpr (ZT > 0) {
        return edge_ptr<R, ZT, I, E>(Pr, Prz, r);
    } else {
        return P + edge_var<R, ZT, I, E>(r, a);
    }
}

__device__ __forceinline__ float canon(float x) { return __fadd_rn(x, 0.0f); }

/* One layer (base row I) of one iteration for the thread's row: pass 1
 * (L = posterior - old message, sign bits, the two minima), pass 2 (new
 * messages and posteriors in the mode's arithmetic) and the new compressed
 * messages M1, M2 (rounded magnitudes) and NEG (sign bit d-1-e of edge e |
 * argmin edge << 27). at(e) gives the posterior of edge e of this layer for
 * this row. Used by the specialised decoder and by the mixed-code decoder.
 * With PAR, *odd is set to whether the row fails the parity check on the
 * posteriors this layer writes (hard bit x >= 0). */
template <int R, int I, int MODE, bool PAR = false, typename At>
__device__ __forceinline__ void tdmp_layer(At&& at, float& M1, float& M2, uint32_t& NEG, bool* odd = nullptr)
{
    constexpr int d = layer_degree(R, I);
    float L[d];
    uint32_t LC[d];
    uint32_t sgn = 0;
    float m1, m2;
    const float oM1 = M1, oM2 = M2;
    const uint32_t oNeg = NEG;
    const int oIdx = (int)(oNeg >> 27);
    /* pass 1: L = post - old message, sign bits, two minima */
    static_for<d>([&](auto E) {
        constexpr int e = decltype(E)::value;
        const float x = *at(E);
        const float mag = (oIdx == e) ? oM2 : oM1;
        const uint32_t sb = (oNeg << (32 - d + e)) & 0x80000000u;
        const float msg = __uint_as_float(__float_as_uint(mag) | sb);
        const float l = __fsub_rn(x, msg);
        L[e] = l;
        LC[e] = __float_as_uint(canon(l));
        sgn = __funnelshift_l(LC[e], sgn, 1);
    });
    two_min_abs<0, d>(L, m1, m2);
    m1 = fminf(m1, 10000.0f);
    m2 = fminf(m2, 10000.0f);
    /* bit (d-1-e) of sgn is neg(L_e); message e is negative iff
     * (d & 1) ^ parity(neg) ^ neg(L_e)  (reference :148,172,191) */
    const uint32_t flip = (uint32_t)((d & 1) ^ (__popc(sgn) & 1));
    const uint32_t dmask = (d >= 32) ? 0xffffffffu : ((1u << d) - 1u);
    int nIdx = 0;
    bool par = false;   /* parity of the negative posteriors written (PAR) */
    if constexpr (MODE == kMs) {
        const uint32_t fb = flip << 31;
        static_for<d>([&](auto E) {
            constexpr int e = decltype(E)::value;
            const float l = L[e];
            const bool is_min = fabsf(l) == m1;
            const float mu = is_min ? m2 : m1;
            nIdx = is_min ? e : nIdx;
            const uint32_t sb = (LC[e] & 0x80000000u) ^ fb;
            const float t = __uint_as_float(__float_as_uint(mu) | sb);
            const float pn = __fadd_rn(l, t);
            *at(E) = pn;
            if constexpr (PAR) par = par != (pn < 0.0f);
        });
        M1 = m1;
        M2 = m2;
    } else {
        double D1, D2;
        if constexpr (MODE == kNms) {
            D1 = __dmul_rn((double)m1, 0.815);
            D2 = __dmul_rn((double)m2, 0.815);
        } else {
            const double t1 = __dsub_rn((double)m1, 0.10);
            const double t2 = __dsub_rn((double)m2, 0.10);
            D1 = t1 < 0.0 ? 0.0 : t1;
            D2 = t2 < 0.0 ? 0.0 : t2;
        }
        const uint32_t fb = flip << 31;
        const int h1 = __double2hiint(D1) ^ (int)fb, l1 = __double2loint(D1);
        const int h2 = __double2hiint(D2) ^ (int)fb, l2 = __double2loint(D2);
        static_for<d>([&](auto E) {
            constexpr int e = decltype(E)::value;
            const float l = L[e];
            const bool is_min = fabsf(l) == m1;
            nIdx = is_min ? e : nIdx;
            int hi = is_min ? h2 : h1;
            const int lo = is_min ? l2 : l1;
            hi ^= (int)(LC[e] & 0x80000000u);
            const double t = __hiloint2double(hi, lo);
            const float pn = __double2float_rn(__dadd_rn((double)l, t));
            *at(E) = pn;
            if constexpr (PAR) par = par != (pn < 0.0f);
        });
        M1 = __double2float_rn(D1);
        M2 = __double2float_rn(D2);
    }
    NEG = ((sgn ^ (flip ? dmask : 0u)) & dmask) | ((uint32_t)nIdx << 27);
    if constexpr (PAR) *odd = par != ((d & 1) != 0);
}

/* The same layer with one message per edge kept as a float in a register
 * (Mr, indexed by block), normalized min-sum only: pass 1 reads the old
 * message directly instead of rebuilding it from M1 / M2 / NEG. The stored
 * values are identical to the compressed form's (+-float(D1) or
 * +-float(D2)): where several edges tie at the minimum, D1 == D2. PAR and
 * odd as in tdmp_layer. */
template <int R, int I, bool PAR = false, typename At, int NB>
__device__ __forceinline__ void tdmp_layer_edges(At&& at, float (&Mr)[NB], bool* odd = nullptr)
{
    constexpr int d = layer_degree(R, I);
    constexpr int b0 = block_index(R, I, 0);
    float L[d];
    uint32_t LC[d];
    uint32_t sgn = 0;
    float m1, m2;
    static_for<d>([&](auto E) {
        constexpr int e = decltype(E)::value;
        const float l = __fsub_rn(*at(E), Mr[b0 + e]);
        L[e] = l;
        LC[e] = __float_as_uint(canon(l));
        sgn ^= LC[e];   /* bit 31: parity of the negative L */
    });
    two_min_abs<0, d>(L, m1, m2);
    m1 = fminf(m1, 10000.0f);
    m2 = fminf(m2, 10000.0f);
    const uint32_t fb = (sgn ^ ((uint32_t)(d & 1) << 31)) & 0x80000000u;
    const double D1 = __dmul_rn((double)m1, 0.815), D2 = __dmul_rn((double)m2, 0.815);
    /* the magnitudes carry the row's sign flip already (they are >= +0), so
     * edge e's sign is one XOR with the sign bit of its L */
    const uint32_t f1 = __float_as_uint(__double2float_rn(D1)) | fb, f2 = __float_as_uint(__double2float_rn(D2)) | fb;
    const int h1 = __double2hiint(D1) ^ (int)fb, l1 = __double2loint(D1);
    const int h2 = __double2hiint(D2) ^ (int)fb, l2 = __double2loint(D2);
    bool par = false;
    static_for<d>([&](auto E) {
        constexpr int e = decltype(E)::value;
        const float l = L[e];
        const bool is_min = fabsf(l) == m1;
        const uint32_t sb = LC[e] & 0x80000000u;
        int hi = is_min ? h2 : h1;
        const int lo = is_min ? l2 : l1;
        hi ^= (int)sb;
        const float pn = __double2float_rn(__dadd_rn((double)l, __hiloint2double(hi, lo)));
        *at(E) = pn;
        if constexpr (PAR) par = par != (pn < 0.0f);
        Mr[b0 + e] = __uint_as_float((is_min ? f2 : f1) ^ sb);
    });
    if constexpr (PAR) *odd = par != ((d & 1) != 0);
}

/* Which message layout the specialised normalized min-sum decoder uses: one
 * float per edge in registers where that measured more than 1% faster on a
 * B200 (all 114 codes timed both ways, outputs identical: 36 codes, by up to
 * 24%), else the compressed per-row form (3 registers per layer), which was
 * up to 1.6x faster on the others: the per-edge form needs 128-168 registers
 * and so fewer resident CTAs. Bit (z - 24) / 4 of kEdgeMsgZ[rate]. */
constexpr uint32_t kEdgeMsgZ[kRates] = {0x44f55u, 0x44644u, 0x44654u, 0x40c44u, 0x40cc4u, 0x40004u};

constexpr bool tdmp_edge_messages(int rate, int z, int mode)
{
    return mode == kNms && z >= kZMin && z <= kZMax && z % kZStep == 0 &&
           ((kEdgeMsgZ[rate] >> ((z - kZMin) / kZStep)) & 1u) != 0;
}

/* Syndrome of the thread's rows in layers FIRST .. END-1 (default: all): 1
 * if any row fails. The
 * hard decision is x >= 0 (-0.0 is bit 1); a row of degree d fails when d
 * minus its number of negative posteriors is odd. at(I, E) as in tdmp_layer. */
template <int R, int FIRST = 0, int END = kMb[R], typename At>
__device__ __forceinline__ unsigned tdmp_rows_fail(At&& at)
{
    unsigned fail = 0;
    static_for<END - FIRST>([&](auto I_) {
        using I = std::integral_constant<int, FIRST + decltype(I_)::value>;
        constexpr int d = layer_degree(R, I::value);
        bool odd = (d & 1) != 0;
        static_for<d>([&](auto E) { odd = odd != (*at(I{}, E) < 0.0f); });
        fail |= odd ? 1u : 0u;
    });
    return fail;
}

template <int R, int ZT, int MODE>
__global__ void __launch_bounds__(TdmpShape<R, ZT>::THREADS)
tdmp_decode_kernel(const __grid_constant__ DecodeArgs a)
{
    using S = TdmpShape<R, ZT>;
    constexpr int MB = S::MB, G = S::G;
    const int Z = ZT > 0 ? ZT : a.z;
    const int N = kNB * Z;
    const int nthreads = G * Z;
    extern __shared__ __align__(128) float smem_post[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned s_fail[2], s_last[2], s_half[2];

    const int tid = threadIdx.x;
    const int g = G == 1 ? 0 : tid / Z;
    const int r = tid - g * Z;
    const long long f0 = (long long)blockIdx.x * G;
    const long long left = a.frames - f0;
    const int nf = left < G ? (int)left : G;
    float* P = smem_post + g * N;
    float* const Pr = P + r;
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
        bulk_g2s(smem_post, a.llr + f0 * N, bytes, &bar);
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

    /* syndrome of the current posterior for this thread's rows in layers
     * FIRST .. END-1: 1 if any fails */
    auto rows_fail = [&](auto FIRST, auto END) -> unsigned {
        return tdmp_rows_fail<R, decltype(FIRST)::value, decltype(END)::value>([&](auto I, auto E) {
            return post_ptr<R, ZT, decltype(I)::value, decltype(E)::value>(P, Pr, Prz, r, a);
        });
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

    /* compressed messages per layer: magnitudes and NEG = sign bits (bit
     * d-1-e for edge e) | argmin edge << 27; or one float per edge */
    constexpr bool EDGE_MSGS = tdmp_edge_messages(R, ZT, MODE);
    float M1[MB], M2[MB];
    uint32_t NEG[MB];
    float Mr[EDGE_MSGS ? num_blocks(R) : 1];
#pragma unroll
    for (int i = 0; i < MB; i++) { M1[i] = 0.0f; M2[i] = 0.0f; NEG[i] = 0u; }
#pragma unroll
    for (int q = 0; q < (EDGE_MSGS ? num_blocks(R) : 1); q++) Mr[q] = 0.0f;

    for (int it = 1; it <= a.max_iter && fmask != 0u; ++it) {
        const int slot = it & 1;   /* last read two iterations ago, before many barriers */
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
        static_for<MB>([&](auto I) {
            constexpr bool LAST = decltype(I)::value == MB - 1;
            if (active) {
                auto at = [&](auto E) { return post_ptr<R, ZT, decltype(I)::value, decltype(E)::value>(P, Pr, Prz, r, a); };
                if constexpr (EDGE_MSGS)
                    tdmp_layer_edges<R, decltype(I)::value, LAST>(at, Mr, &last_odd);
                else
                    tdmp_layer<R, decltype(I)::value, MODE, LAST>(at, M1[I], M2[I], NEG[I], &last_odd);
            }
            if constexpr (!LAST) __syncthreads();
        });
        /* stopping rule (zero syndrome over every row, reference
         * lib/ldpc_decoder.cc:242-251): a frame with a failing row in the last
         * layer fails; the other active frames check the remaining layers in
         * two halves, with a vote after each (a frame that fails in the first
         * half skips the second). The first vote is the last layer's barrier. */
        const unsigned lmask = frame_fail(active && last_odd ? 1u : 0u, &s_last[slot]);
        unsigned fm = lmask;
        if (fmask & ~fm)
            fm |= frame_fail(active && !((fm >> g) & 1u) ? rows_fail(L0{}, LH{}) : 0u, &s_fail[slot]);
        if (fmask & ~fm)
            fm |= frame_fail(active && !((fm >> g) & 1u) ? rows_fail(LH{}, LM{}) : 0u, &s_half[slot]);
        fmask = fm;
        if (active) {
            iters = it;
            active = (fmask >> g) & 1u;
        }
    }

    /* outputs: hard bits and posterior, vectorised over the CTA's frames */
    const int total = nf * N;
    int8_t* hard = a.hard + f0 * N;
    for (int v = tid * 4; v < total; v += nthreads * 4) {
        const float4 p = *reinterpret_cast<const float4*>(smem_post + v);
        const uint32_t w = (p.x >= 0.0f ? 1u : 0u) | (p.y >= 0.0f ? 1u << 8 : 0u) |
                           (p.z >= 0.0f ? 1u << 16 : 0u) | (p.w >= 0.0f ? 1u << 24 : 0u);
        *reinterpret_cast<uint32_t*>(hard + v) = w;
        if (a.post) *reinterpret_cast<float4*>(a.post + f0 * N + v) = p;
    }
    if (a.status && live && r == 0)
        a.status[f0 + g] = iters | ((active ? 1 : 0) << 16);
}

}  // namespace wldpc

#endif
