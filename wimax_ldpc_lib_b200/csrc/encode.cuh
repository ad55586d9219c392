/*
 * Dual-diagonal WiMAX encoder over packed GF(2) words, bit-exact with the
 * reference ldpc_encoder::encode_data (reference lib/ldpc_encoder.cc:29-105),
 * and on-device synthetic frame generation (info bits, encoder, BPSK, AWGN,
 * LLR) that feeds the decoders.
 *
 * One warp encodes one frame. The k info bits are packed into a flat bit
 * array; column c occupies bits c*z .. c*z+z-1. A circulant block with shift s
 * maps row r to column bit (r + s) mod z, so 32 rows of a block are one
 * rotated 32-bit extraction (rot32) from the packed column. With V_i the z-bit
 * vector of base row i of H_info * u (reference compute_v, :29-48, info
 * columns only, any non-zero byte counts as 1), the reference recursion
 * (reference :50-105) is, block-wise:
 *   P_{mb-1} = V_{mb-1}
 *   P_b = P_{b-1} ^ V_{b-1}        b = 1..X       (P_0 starts at zero)
 *   P_b = V_b ^ P_{b+1}            b = mb-2 .. X+1
 *   P_0 = V_X ^ P_{X+1} ^ P_X
 *   parity block 0 = P_0; parity block b >= 1, row r = P_b[r] ^ P_0[(r + D) mod z]
 * The systematic part is a byte copy of the input (reference :90), so
 * non-0/1 input bytes pass through unchanged exactly as in the reference.
 */
#ifndef WLDPC_ENCODE_CUH
#define WLDPC_ENCODE_CUH

#include <cstdint>
#include "codes.h"
#include "device_util.cuh"

namespace wldpc {

/* Runtime description of one (rate, z) code, passed by value to kernels. */
struct CodeDesc {
    int rate, z, mb, kb, n, k, m, D, X, nblk, nw;   /* nw = words per z-bit block */
    unsigned zinv;                       /* ceil(2^20 / z): p / z = (p * zinv) >> 20 for p <= 12 z */
    unsigned char row_start[kMaxMb + 1];
    unsigned char col[96];
    unsigned char shift[96];
    unsigned char info_start[kMaxMb + 1];   /* the info-column blocks of each row: */
    uint32_t info_blk[96];                  /* col * z | shift << 16 */
};

inline CodeDesc make_code_desc(int rate, int z)
{
    CodeDesc c{};
    c.rate = rate;
    c.z = z;
    c.mb = kMb[rate];
    c.kb = kNB - c.mb;
    c.n = kNB * z;
    c.k = c.kb * z;
    c.m = c.mb * z;
    c.D = D_of(rate, z);
    c.X = kX[rate];
    c.nw = (z + 31) / 32;
    c.zinv = ((1u << 20) + (unsigned)z - 1u) / (unsigned)z;
    int b = 0, q = 0;
    for (int i = 0; i < c.mb; i++) {
        c.row_start[i] = (unsigned char)b;
        c.info_start[i] = (unsigned char)q;
        for (int j = 0; j < kNB; j++) {
            const int p = kBase[rate][i][j];
            if (p < 0) continue;
            c.col[b] = (unsigned char)j;
            c.shift[b] = (unsigned char)shift_rule(rate, p, z);
            if (j < c.kb) c.info_blk[q++] = (uint32_t)(j * z) | ((uint32_t)c.shift[b] << 16);
            b++;
        }
    }
    c.row_start[c.mb] = (unsigned char)b;
    c.info_start[c.mb] = (unsigned char)q;
    c.nblk = b;
    return c;
}

/* bits [pos, pos+32) of a packed little-endian bit array */
__device__ __forceinline__ uint32_t get_bits32(const uint32_t* a, int pos)
{
    const int w = pos >> 5, b = pos & 31;
    return __funnelshift_r(a[w], a[w + 1], b);
}

/* 32 bits of the z-bit column starting at bit cb, rotated to start at row t
 * (0 <= t < z): bit j = column[(t + j) mod z]. Bits j >= z (last word of a
 * block) are not meaningful. Needs one readable word past the column end. */
__device__ __forceinline__ uint32_t rot32(const uint32_t* a, int cb, int z, int t)
{
    uint32_t v = get_bits32(a, cb + t);
    const int k1 = z - t;
    if (k1 < 32) v = (v & ((1u << k1) - 1u)) | (get_bits32(a, cb) << k1);
    return v;
}

/* Per-warp scratch of the encoder in shared memory (words). */
struct EncScratch {
    uint32_t U[kNB * kZMax / 32 + 4];   /* packed info bits, +padding */
    uint32_t V[kMaxMb * 3];             /* [layer][word] */
    uint32_t P[kMaxMb * 3 + 4];         /* [block][word], block 0 first, +padding */
    uint32_t out[kMaxMb * 3];           /* parity bits to emit, [block][word] */
};

/* p / nw for the words per block nw in {1, 2, 3} and 0 <= p < 2^15, without
 * an integer division (p / 3 as a multiply and shift) */
__device__ __forceinline__ int div_nw(int p, int nw)
{
    return nw == 1 ? p : (nw == 2 ? (p >> 1) : (int)(((unsigned)p * 0xAAABu) >> 17));
}

/* Encodes the packed info bits in s.U into parity words s.out (all lanes of
 * the warp participate; U must be written and visible before the call). */
__device__ __forceinline__ void warp_encode_parity(const CodeDesc& c, EncScratch& s, int lane)
{
    const int nw = c.nw, z = c.z;
    /* V = H_info * u, one (layer, word) pair per lane */
    for (int p = lane; p < c.mb * nw; p += 32) {
        const int i = div_nw(p, nw), w = p - i * nw;
        uint32_t v = 0;
        for (int q = c.info_start[i]; q < c.info_start[i + 1]; q++) {
            const uint32_t cs = c.info_blk[q];   /* one constant load per block */
            int t = 32 * w + (int)(cs >> 16);
            t = t >= z ? t - z : t;
            t = t >= z ? t - z : t;
            v ^= rot32(s.U, (int)(cs & 0xffffu), z, t);
        }
        const int rem = z - 32 * w;
        if (rem < 32) v &= (1u << rem) - 1u;
        s.V[i * nw + w] = v;
    }
    __syncwarp();
    /* dual-diagonal recursion, one word column per lane */
    if (lane < nw) {
        const int w = lane, mb = c.mb, X = c.X;
        uint32_t* P = s.P;
        const uint32_t* V = s.V;
        P[(mb - 1) * nw + w] = V[(mb - 1) * nw + w];
        uint32_t acc = 0;
        for (int b = 1; b <= X; b++) {
            acc ^= V[(b - 1) * nw + w];
            P[b * nw + w] = acc;
        }
        for (int b = mb - 2; b >= X + 1; b--) P[b * nw + w] = V[b * nw + w] ^ P[(b + 1) * nw + w];
        P[w] = V[X * nw + w] ^ P[(X + 1) * nw + w] ^ P[X * nw + w];
    }
    if (lane == 0) { s.P[c.mb * nw] = 0; s.P[c.mb * nw + 1] = 0; }
    __syncwarp();
    /* F correction: block b >= 1 row r gets P_0[(r + D) mod z]; P_0's words
     * are contiguous at the start of s.P, so it is its own packed column. */
    for (int p = lane; p < c.mb * nw; p += 32) {
        const int b = div_nw(p, nw), w = p - b * nw;
        uint32_t v = s.P[p];
        if (b > 0) {
            int t = 32 * w + c.D;
            t = t >= z ? t - z : t;
            t = t >= z ? t - z : t;
            v ^= rot32(s.P, 0, z, t);
        }
        s.out[p] = v;
    }
    __syncwarp();
}

/* bytes 0/1 of parity bits r..r+3 of block b */
__device__ __forceinline__ uint32_t parity_bytes4(const EncScratch& s, int nw, int b, int r)
{
    const uint32_t w = s.out[b * nw + (r >> 5)] >> (r & 31);
    return (w & 1u) | ((w & 2u) << 7) | ((w & 4u) << 14) | ((w & 8u) << 21);
}

}  // namespace wldpc

#endif
