/*
 * compute_syndrome over a batch of byte-per-bit words, specialised on
 * (rate, z): one frame per lane for the parity work, one warp per frame for
 * the memory traffic (as the encoder in encode_lanes.cuh).
 *
 * The reference (lib/ldpc_decoder.cc:67-104) XORs the bytes of each check row
 * and counts the rows whose XOR is non-zero (or returns 1 at the first one
 * with early exit; the count and the early-exit answer differ only in that
 * the latter is min(count, 1)). A byte XOR is the XOR of its 8 bit planes, so
 * a row fails when any plane has odd parity. A warp checks 32 frames:
 *  A. per frame, the whole warp reads the n bytes in 16-byte chunks,
 *     coalesced, packs bit 0 of every byte into the frame's row of shared
 *     memory and notes whether any byte has another bit set;
 *  B. each lane takes one frame's row and XORs, per check-row word, the
 *     rotated 32-bit extractions of the row's blocks (every column, shift
 *     and word index a compile-time constant), keeping the failing-row words;
 *  then, only when some frame of the warp has bytes other than 0 and 1, the
 *  warp repeats A and B for bit planes 1..7 of those frames and ORs the
 *  failing-row words; finally each lane counts its frame's failing rows.
 */
#ifndef WLDPC_SYNDROME_LANES_CUH
#define WLDPC_SYNDROME_LANES_CUH

#include <cstdint>
#include "codes.h"
#include "encode_lanes.cuh"

namespace wldpc {

template <int R, int Z>
struct SynLanes {
    static constexpr int MB = kMb[R], N = kNB * Z;
    static constexpr int NW = (Z + 31) / 32;            /* words per z-row block */
    static constexpr int LASTBITS = Z - 32 * (NW - 1);
    static constexpr uint32_t LASTMASK = LASTBITS < 32 ? (1u << (LASTBITS % 32)) - 1u : 0xffffffffu;
    static constexpr int NWORDS = (N + 31) / 32;
    static constexpr int ROW = NWORDS | 1;              /* odd stride: lanes hit 32 banks */
    static constexpr int NCH = N / 16;                  /* 16-byte chunks per frame */
    static constexpr int RND = (NCH + 31) / 32;
    static constexpr int FA = RND <= 3 ? 4 : 2;         /* frames whose loads are in flight together */
    static constexpr int WARPS = 4;
    static constexpr int THREADS = 32 * WARPS;
};

/* bit p of each byte of w, gathered: bit j = bit p of byte j */
__device__ __forceinline__ uint32_t plane_nibble(uint32_t w, int p)
{
    return (((w >> p) & 0x01010101u) * 0x01020408u) >> 24;
}

template <int R, int Z>
__global__ void __launch_bounds__(SynLanes<R, Z>::THREADS)
syndrome_lanes_kernel(const int8_t* __restrict__ bits, uint32_t* __restrict__ out, long long frames,
                      int early_exit)
{
    using S = SynLanes<R, Z>;
    constexpr int MB = S::MB, NW = S::NW, N = S::N, NCH = S::NCH, RND = S::RND, FA = S::FA, ROW = S::ROW;
    __shared__ uint32_t smem[S::WARPS * 32 * ROW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long f0 = ((long long)blockIdx.x * S::WARPS + warp) * 32;
    if (f0 >= frames) return;
    const int nf = frames - f0 < 32 ? (int)(frames - f0) : 32;
    uint32_t* const U = smem + warp * 32 * ROW;

    /* A: bit plane p of the frames in `which` (bit ff: frame ff) into their
     * rows; returns the frames whose bytes have bits other than bit 0 */
    auto pack_plane = [&](int p, uint32_t which) -> uint32_t {
        uint32_t upper_frames = 0;
        for (int ff0 = 0; ff0 < nf; ff0 += FA) {
            uint4 v[FA][RND];
#pragma unroll
            for (int a = 0; a < FA; a++)
#pragma unroll
                for (int r = 0; r < RND; r++) {
                    const int q = 32 * r + lane;
                    const int ff = ff0 + a;
                    if (ff < nf && ((which >> ff) & 1u) && q < NCH)
                        v[a][r] = __ldcs(reinterpret_cast<const uint4*>(bits + (f0 + ff) * N) + q);
                    else
                        v[a][r] = make_uint4(0u, 0u, 0u, 0u);
                }
#pragma unroll
            for (int a = 0; a < FA; a++) {
                const int ff = ff0 + a;
                if (ff >= nf) break;                        /* uniform over the warp */
                if (!((which >> ff) & 1u)) continue;        /* uniform over the warp */
                uint32_t* row = U + ff * ROW;
                uint32_t upper = 0;
#pragma unroll
                for (int r = 0; r < RND; r++) {
                    const int q = 32 * r + lane;
                    const uint4 w = v[a][r];
                    upper |= (w.x | w.y | w.z | w.w) & 0xFEFEFEFEu;
                    uint32_t b = plane_nibble(w.x, p) | (plane_nibble(w.y, p) << 4) | (plane_nibble(w.z, p) << 8) |
                                 (plane_nibble(w.w, p) << 12);
                    b |= __shfl_down_sync(0xffffffffu, b, 1) << 16;
                    if (q < NCH && (q & 1) == 0) row[q >> 1] = b;
                }
                if (__any_sync(0xffffffffu, upper != 0u)) upper_frames |= 1u << ff;
            }
        }
        return upper_frames;
    };

    /* B: failing-row words of this lane's frame for the plane in its row */
    uint32_t fail[MB][NW];
#pragma unroll
    for (int i = 0; i < MB; i++)
#pragma unroll
        for (int w = 0; w < NW; w++) fail[i][w] = 0u;
    auto row_parities = [&]() {
        const uint32_t* row = U + lane * ROW;
        auto get = [&](auto W) { return row[decltype(W)::value]; };
        static_for<MB>([&](auto I) {
            constexpr int i = decltype(I)::value;
            static_for<NW>([&](auto Wd) {
                constexpr int w = decltype(Wd)::value;
                uint32_t v = 0;
                static_for<layer_degree(R, i)>([&](auto E) {
                    constexpr int e = decltype(E)::value;
                    constexpr int c = layer_col(R, i, e), s = layer_shift(R, Z, i, e);
                    v ^= rot32_at<Z, c * Z, (32 * w + s) % Z, S::NWORDS>(get);
                });
                if constexpr (w == NW - 1) v &= S::LASTMASK;
                fail[i][w] |= v;
            });
        });
    };

    const uint32_t all = nf >= 32 ? 0xffffffffu : (1u << nf) - 1u;
    const uint32_t upper = pack_plane(0, all);
    __syncwarp();
    if (lane < nf) row_parities();
    if (upper) {
        for (int p = 1; p < 8; p++) {
            __syncwarp();
            pack_plane(p, upper);
            __syncwarp();
            if (lane < nf && ((upper >> lane) & 1u)) row_parities();
        }
    }
    if (lane < nf) {
        uint32_t count = 0;
#pragma unroll
        for (int i = 0; i < MB; i++)
#pragma unroll
            for (int w = 0; w < NW; w++) count += __popc(fail[i][w]);
        out[f0 + lane] = early_exit ? (count != 0u ? 1u : 0u) : count;
    }
}

}  // namespace wldpc

#endif
