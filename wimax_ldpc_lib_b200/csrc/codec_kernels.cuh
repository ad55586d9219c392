/*
 * Launchers for the encoder / frame generation / syndrome / input-adapter
 * kernels (codec_kernels.cu) and the TDMP decoders (tdmp_dispatch.cu).
 */
#ifndef WLDPC_CODEC_KERNELS_CUH
#define WLDPC_CODEC_KERNELS_CUH

#include <cstdint>
#include <cuda_runtime.h>
#include "encode.cuh"
#include "nms_decode.cuh"

namespace wldpc {

struct FramegenArgs {
    uint64_t seed;
    uint64_t first_frame;   /* global index of frame 0 of this batch */
    long long frames;
    float ebno_lo, ebno_hi; /* Eb/N0 (dB) drawn uniformly per frame */
    uint8_t* info;          /* frames x k bytes 0/1, or null */
    uint8_t* cw;            /* frames x n bytes 0/1, or null */
    float* llr;             /* frames x n, or null (16-byte aligned) */
    float* ebno_out;        /* frames, or null */
};

/* null-space description of H for random codewords: A is rank x words
 * (row i restricted to the free columns, packed), pivot_col[rank],
 * free_col[nfree] (device pointers) */
struct NullspaceArgs {
    const uint32_t* A;
    const unsigned short* pivot_col;
    const unsigned short* free_col;
    int rank, nfree, words;
};

cudaError_t launch_framegen_nullspace(const CodeDesc& c, const FramegenArgs& a, const NullspaceArgs& ns,
                                      cudaStream_t st);
/* encoder specialised on (rate, z), one frame per lane (encode_lanes.cuh);
 * info and codeword must be aligned to `align` bytes */
struct EncLanesLaunch {
    void (*kernel)(const uint8_t*, uint8_t*, long long);
    int align;
    int threads;        /* per CTA: 32 frames per warp */
};
/* entry for (rate, z) or null (rate 3/4B has no encoder) */
const EncLanesLaunch* enc_lanes_entry(int rate, int z);
/* compute_syndrome specialised on (rate, z), one frame per lane
 * (syndrome_lanes.cuh); the bytes must be 16-byte aligned */
struct SynLanesLaunch {
    void (*kernel)(const int8_t*, uint32_t*, long long, int);
    int threads;        /* per CTA: 32 frames per warp */
};
const SynLanesLaunch* syn_lanes_entry(int rate, int z);
/* the encoder over a batch: the (rate, z)-specialised kernel when the
 * buffers are aligned for it, else the generic one-warp-per-frame kernel */
cudaError_t launch_encode_bytes(const CodeDesc& c, const uint8_t* info, uint8_t* cw, long long frames,
                                cudaStream_t st);
cudaError_t launch_framegen(const CodeDesc& c, const FramegenArgs& a, cudaStream_t st);
/* compute_syndrome over a batch (syndrome_lanes.cuh); the bytes must be
 * 16-byte aligned (the C ABI stages them in its own device buffers) */
cudaError_t launch_syndrome(const CodeDesc& c, const int8_t* bits, uint32_t* out, long long frames,
                            int early_exit, cudaStream_t st);
cudaError_t launch_bits_to_llr(const int8_t* bits, float* llr, long long count, cudaStream_t st);
/* the reference BER_runner's periodic LFSR info-bit stream */
cudaError_t upload_lfsr_period(const uint32_t* words);
cudaError_t launch_wait_bound(uint32_t limit_us, unsigned long long* out, cudaStream_t st);
cudaError_t launch_lfsr_bits(unsigned long long first_bit, long long nbits, uint8_t* out, cudaStream_t st);

/* TDMP decoder specialised on (rate, z, mode) */
struct TdmpLaunch {
    void (*kernel)(const DecodeArgs);
    int threads;        /* per CTA (run-time z: z) */
    int frames_per_cta;
    int smem;           /* dynamic shared memory bytes (run-time z: 96 z) */
    bool runtime_z;     /* z, shifts and columns are passed in DecodeArgs */
};
/* entry for (rate, z, mode) or null if not built */
const TdmpLaunch* tdmp_entry(int rate, int z, int mode);
cudaError_t launch_tdmp(int rate, int z, int mode, const DecodeArgs& a, cudaStream_t st);

}  // namespace wldpc

#endif
