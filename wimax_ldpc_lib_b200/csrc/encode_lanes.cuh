/*
 * Dual-diagonal encoder specialised on (rate, z): one frame per lane for the
 * GF(2) work, one warp per frame for the memory traffic. Bit-exact with the
 * reference ldpc_encoder::encode_data (reference lib/ldpc_encoder.cc:29-105);
 * the block recursion is the one written out in encode.cuh.
 *
 * A warp encodes 32 frames in three phases:
 *  A. per frame, the whole warp reads the k info bytes in 16-byte (or 8-byte)
 *     chunks, coalesced, copies them to the systematic part of the codeword
 *     (reference :90, so non-0/1 bytes pass through) and packs them into bits
 *     (any non-zero byte is a 1, reference :43) in the frame's row of shared
 *     memory;
 *  B. each lane takes one frame's row and computes V = H_info u, the
 *     recursion and the F correction with every column, shift and word index
 *     a compile-time constant (no address arithmetic, no divergence: all lanes
 *     run the same code on different rows), and writes the m parity bits as
 *     one contiguous bit array to the frame's output row;
 *  C. per frame, the whole warp expands the parity bits to bytes and stores
 *     them in 16-byte (or 8-byte) chunks, coalesced.
 * Rows are an odd number of words apart, so lane-per-frame accesses hit 32
 * different banks.
 */
#ifndef WLDPC_ENCODE_LANES_CUH
#define WLDPC_ENCODE_LANES_CUH

#include <cstdint>
#include <type_traits>
#include "codes.h"
#include "encode.cuh"

namespace wldpc {

template <int R, int Z>
struct EncLanes {
    static constexpr int MB = kMb[R], KB = kNB - MB;
    static constexpr int K = KB * Z, M = MB * Z, N = kNB * Z;
    static constexpr int NW = (Z + 31) / 32;            /* words per z-bit block */
    static constexpr int LASTBITS = Z - 32 * (NW - 1);  /* valid bits of a block's last word */
    static constexpr uint32_t LASTMASK = LASTBITS < 32 ? (1u << (LASTBITS % 32)) - 1u : 0xffffffffu;
    static constexpr int KWORDS = (K + 31) / 32;
    static constexpr int MWORDS = (M + 31) / 32;
    static constexpr int UROW = KWORDS | 1;             /* odd stride */
    static constexpr int OROW = MWORDS | 1;
    static constexpr int CB = (K % 16 == 0) ? 16 : 8;   /* bytes per lane per memory chunk */
    static constexpr int WARPS = 4;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int SMEM_WORDS = WARPS * 32 * (UROW + OROW);
    static constexpr int D = D_of(R, Z), X = kX[R];
};

/* 4 bits, bit j = byte j of w is non-zero */
__device__ __forceinline__ uint32_t nonzero_nibble(uint32_t w)
{
    const uint32_t nz = (((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w) & 0x80808080u;   /* bit 8j+7 */
    return (nz * 0x00204081u) >> 28;                                              /* to bits 28+j */
}

/* 4 bytes 0/1 from the low 4 bits of b */
__device__ __forceinline__ uint32_t nibble_bytes(uint32_t b)
{
    return ((b & 0xFu) * 0x00204081u) & 0x01010101u;
}

/* bits [P, P+32) of a word array held in registers or shared memory, P a
 * compile-time constant; words past the end read as 0 */
template <int P, int NWORDS, typename Get>
__device__ __forceinline__ uint32_t bits32_at(Get&& get)
{
    constexpr int w = P >> 5, b = P & 31;
    const uint32_t lo = w < NWORDS ? get(std::integral_constant<int, (w < NWORDS ? w : 0)>{}) : 0u;
    if constexpr (b == 0) {
        return lo;
    } else {
        const uint32_t hi = (w + 1) < NWORDS ? get(std::integral_constant<int, ((w + 1) < NWORDS ? w + 1 : 0)>{}) : 0u;
        return __funnelshift_r(lo, hi, b);
    }
}

/* 32 bits of the z-bit column that starts at bit CB0 of a packed array,
 * rotated to start at row T: bit j = column[(T + j) mod Z] for j < Z (bits
 * j >= Z of a block's last word are not meaningful) */
template <int Z, int CB0, int T, int NWORDS, typename Get>
__device__ __forceinline__ uint32_t rot32_at(Get&& get)
{
    uint32_t v = bits32_at<CB0 + T, NWORDS>(get);
    constexpr int k1 = Z - T;
    if constexpr (k1 < 32) v = (v & ((1u << k1) - 1u)) | (bits32_at<CB0, NWORDS>(get) << k1);
    return v;
}

template <int R, int Z>
__global__ void __launch_bounds__(EncLanes<R, Z>::THREADS)
encode_lanes_kernel(const uint8_t* __restrict__ info, uint8_t* __restrict__ cw, long long frames)
{
    using S = EncLanes<R, Z>;
    constexpr int MB = S::MB, NW = S::NW, K = S::K, M = S::M, N = S::N, CB = S::CB;
    constexpr int UROW = S::UROW, OROW = S::OROW;
    __shared__ uint32_t smem[S::SMEM_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long f0 = ((long long)blockIdx.x * S::WARPS + warp) * 32;
    if (f0 >= frames) return;
    const int nf = frames - f0 < 32 ? (int)(frames - f0) : 32;
    uint32_t* const U = smem + warp * 32 * (UROW + OROW);
    uint32_t* const O = U + 32 * UROW;

    /* A. pack the info bits of each frame (and copy the systematic bytes);
     * the loads of FA frames are issued before any is used, so that a warp
     * keeps FA * RND chunks per lane in flight */
    using Vec = typename std::conditional<CB == 16, uint4, uint2>::type;
    constexpr int KCH = K / CB;                 /* chunks per frame */
    constexpr int RND = (KCH + 31) / 32;        /* chunks per lane per frame */
    constexpr int FA = RND <= 3 ? 4 : 3;
    for (int ff0 = 0; ff0 < nf; ff0 += FA) {
        Vec v[FA][RND];
#pragma unroll
        for (int a = 0; a < FA; a++)
#pragma unroll
            for (int r = 0; r < RND; r++) {
                const int q = 32 * r + lane;
                if (ff0 + a < nf && q < KCH)
                    v[a][r] = __ldcs(reinterpret_cast<const Vec*>(info + (f0 + ff0 + a) * K) + q);
                else
                    v[a][r] = Vec{};
            }
#pragma unroll
        for (int a = 0; a < FA; a++) {
            const int ff = ff0 + a;
            if (ff >= nf) break;   /* uniform over the warp */
            uint8_t* x = cw + (f0 + ff) * N;
            uint32_t* urow = U + ff * UROW;
#pragma unroll
            for (int r = 0; r < RND; r++) {
                const int q = 32 * r + lane;
                uint32_t bits;
                if constexpr (CB == 16) {
                    const uint4 w = v[a][r];
                    if (q < KCH) reinterpret_cast<uint4*>(x)[q] = w;
                    bits = nonzero_nibble(w.x) | (nonzero_nibble(w.y) << 4) | (nonzero_nibble(w.z) << 8) |
                           (nonzero_nibble(w.w) << 12);
                    bits |= __shfl_down_sync(0xffffffffu, bits, 1) << 16;
                    if (q < KCH && (q & 1) == 0) urow[q >> 1] = bits;
                } else {
                    const uint2 w = v[a][r];
                    if (q < KCH) reinterpret_cast<uint2*>(x)[q] = w;
                    bits = nonzero_nibble(w.x) | (nonzero_nibble(w.y) << 4);
                    bits |= __shfl_down_sync(0xffffffffu, bits, 1) << 8;
                    bits |= __shfl_down_sync(0xffffffffu, bits, 2) << 16;
                    if (q < KCH && (q & 3) == 0) urow[q >> 2] = bits;
                }
            }
        }
    }
    __syncwarp();

    /* B. one frame per lane: V = H_info u, the recursion, the F correction */
    if (lane < nf) {
        const uint32_t* urow = U + lane * UROW;
        auto getu = [&](auto W) { return urow[decltype(W)::value]; };
        uint32_t P[MB][NW];
        static_for<MB>([&](auto I) {
            constexpr int i = decltype(I)::value;
            static_for<NW>([&](auto Wd) {
                constexpr int w = decltype(Wd)::value;
                uint32_t v = 0;
                static_for<layer_info_degree(R, i)>([&](auto E) {
                    constexpr int e = decltype(E)::value;   /* info blocks come first in a row */
                    constexpr int c = layer_col(R, i, e), s = layer_shift(R, Z, i, e);
                    constexpr int t = (32 * w + s) % Z;
                    v ^= rot32_at<Z, c * Z, t, S::KWORDS>(getu);
                });
                if constexpr (w == NW - 1) v &= S::LASTMASK;
                P[i][w] = v;   /* V for now */
            });
        });
        /* recursion, word-wise (encode.cuh): P_{mb-1} = V_{mb-1};
         * P_b = P_{b-1} ^ V_{b-1} (b = 1..X, P_0 = 0); P_b = V_b ^ P_{b+1}
         * (b = mb-2 .. X+1); P_0 = V_X ^ P_{X+1} ^ P_X */
        constexpr int X = S::X;
        static_for<NW>([&](auto Wd) {
            constexpr int w = decltype(Wd)::value;
            uint32_t Vv[MB];
            static_for<MB>([&](auto I) { Vv[decltype(I)::value] = P[decltype(I)::value][w]; });
            uint32_t acc = 0;
            static_for<X>([&](auto B) {
                constexpr int b = decltype(B)::value + 1;
                acc ^= Vv[b - 1];
                P[b][w] = acc;
            });
            static_for<MB - 2 - X>([&](auto B) {
                constexpr int b = MB - 2 - decltype(B)::value;
                P[b][w] = Vv[b] ^ P[b + 1][w];
            });
            P[0][w] = Vv[X] ^ P[X + 1][w] ^ P[X][w];
        });
        /* F correction (block b >= 1, row r gets P_0[(r + D) mod z]) and the
         * parity bits as one contiguous array: bit b*z + r */
        auto getp0 = [&](auto W) { return P[0][decltype(W)::value]; };
        uint32_t out[S::MWORDS];
#pragma unroll
        for (int j = 0; j < S::MWORDS; j++) out[j] = 0u;
        static_for<MB>([&](auto B) {
            constexpr int b = decltype(B)::value;
            static_for<NW>([&](auto Wd) {
                constexpr int w = decltype(Wd)::value;
                uint32_t v = P[b][w];
                if constexpr (b > 0) v ^= rot32_at<Z, 0, (32 * w + S::D) % Z, NW>(getp0);
                if constexpr (w == NW - 1) v &= S::LASTMASK;
                constexpr int gp = b * Z + 32 * w, j = gp >> 5, sh = gp & 31;
                out[j] |= v << sh;
                if constexpr (sh != 0 && j + 1 < S::MWORDS) out[j + 1] |= v >> (32 - sh);
            });
        });
        uint32_t* orow = O + lane * OROW;
#pragma unroll
        for (int j = 0; j < S::MWORDS; j++) orow[j] = out[j];
    }
    __syncwarp();

    /* C. parity bytes of each frame, coalesced */
    constexpr int MCH = M / CB;
    for (int ff = 0; ff < nf; ff++) {
        uint8_t* x = cw + (f0 + ff) * N + K;
        const uint32_t* orow = O + ff * OROW;
#pragma unroll
        for (int base = 0; base < MCH; base += 32) {
            const int q = base + lane;
            if (q < MCH) {
                if constexpr (CB == 16) {
                    const uint32_t b = orow[q >> 1] >> ((q & 1) * 16);
                    uint4 v;
                    v.x = nibble_bytes(b);
                    v.y = nibble_bytes(b >> 4);
                    v.z = nibble_bytes(b >> 8);
                    v.w = nibble_bytes(b >> 12);
                    __stcs(reinterpret_cast<uint4*>(x) + q, v);
                } else {
                    const uint32_t b = orow[q >> 2] >> ((q & 3) * 8);
                    uint2 v;
                    v.x = nibble_bytes(b);
                    v.y = nibble_bytes(b >> 4);
                    __stcs(reinterpret_cast<uint2*>(x) + q, v);
                }
            }
        }
    }
}

}  // namespace wldpc

#endif
