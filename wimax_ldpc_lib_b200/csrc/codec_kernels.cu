/*
 * Encoder, frame generation and input-adapter kernels, and the launchers of
 * the (rate, z)-specialised encoder and compute_syndrome kernels
 * (encode_lanes.cuh, syndrome_lanes.cuh).
 *
 *  encode_bytes_kernel  - ldpc_encoder::encode_data over a batch
 *                         (reference lib/ldpc_encoder.cc:50-105), one warp per
 *                         frame, for buffers not aligned for encode_lanes_kernel
 *                         and for rate 3/4B
 *  framegen_kernel      - seeded synthetic frames: Philox info bits, the same
 *                         encoder on packed words, BPSK bit*2-1 (reference
 *                         lib/BER_runner.cc:183), AWGN, LLR = 2y/sigma^2
 *  bits_to_llr_kernel   - the int8 input adapter bit*2.0-1.0 (reference
 *                         lib/ldpc_decoder.cc:108-118)
 */
#include <cstdint>
#include "codec_kernels.cuh"

namespace wldpc {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int round = 0; round < 10; round++) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* Philox block: counter (word, frame lo, frame hi, stream), key = seed */
__device__ __forceinline__ void philox_at(uint64_t seed, uint64_t frame, uint32_t word, uint32_t stream,
                                          uint32_t o[4])
{
    o[0] = word; o[1] = (uint32_t)frame; o[2] = (uint32_t)(frame >> 32); o[3] = stream;
    philox4x32_10(o, (uint32_t)seed, (uint32_t)(seed >> 32));
}

__device__ __forceinline__ float unif24(uint32_t x) { return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f); }


/* BPSK bit*2-1 (positive = bit 1), AWGN from Philox stream 1 by Box-Muller,
 * LLR = 2y/sigma^2, four code bits per Philox block; bits4(j) returns code
 * bits j..j+3 in its low 4 bits. */
template <typename Bits4>
__device__ __forceinline__ void emit_llr(const CodeDesc& c, const FramegenArgs& a, long long f, uint64_t g, float scale,
                                         float sigma, int lane, Bits4 bits4)
{
    float4* l4 = reinterpret_cast<float4*>(a.llr + f * c.n);
    for (int j = lane * 4; j < c.n; j += 128) {
        const uint32_t bits = bits4(j);
        uint32_t o[4];
        philox_at(a.seed, g, (uint32_t)(j >> 2), 1u, o);
        float nrm[4];
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const float u1 = unif24(o[2 * p]), u2 = unif24(o[2 * p + 1]);
            const float rad = sqrtf(-2.0f * logf(u1));
            float sn, cs;
            sincospif(2.0f * u2, &sn, &cs);
            nrm[2 * p] = rad * cs;
            nrm[2 * p + 1] = rad * sn;
        }
        float4 v;
        v.x = scale * ((bits & 1u ? 1.0f : -1.0f) + sigma * nrm[0]);
        v.y = scale * ((bits & 2u ? 1.0f : -1.0f) + sigma * nrm[1]);
        v.z = scale * ((bits & 4u ? 1.0f : -1.0f) + sigma * nrm[2]);
        v.w = scale * ((bits & 8u ? 1.0f : -1.0f) + sigma * nrm[3]);
        l4[j >> 2] = v;
    }
}

/* per-frame Eb/N0 (Philox stream 2) and the noise scale, in float */
__device__ __forceinline__ void frame_noise(const CodeDesc& c, const FramegenArgs& a, uint64_t g, float& ebno,
                                            float& sigma, float& scale)
{
    uint32_t eo[4];
    philox_at(a.seed, g, 0u, 2u, eo);
    ebno = __fadd_rn(a.ebno_lo, __fmul_rn(__fsub_rn(a.ebno_hi, a.ebno_lo), unif24(eo[0])));
    const float rate = (float)c.k / (float)c.n;
    const float ebno_lin = exp10f(ebno * 0.1f);
    const float sigma2 = 1.0f / (2.0f * rate * ebno_lin);
    sigma = sqrtf(sigma2);
    scale = 2.0f / sigma2;
}

constexpr int kEncWarps = 8;

__global__ void __launch_bounds__(32 * kEncWarps)
encode_bytes_kernel(CodeDesc c, const uint8_t* __restrict__ info, uint8_t* __restrict__ cw, long long frames)
{
    __shared__ EncScratch scratch[kEncWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long f = (long long)blockIdx.x * kEncWarps + warp;
    if (f >= frames) return;
    EncScratch& s = scratch[warp];
    const uint8_t* u = info + f * c.k;
    uint8_t* x = cw + f * c.n;
    /* one pass over the info bytes, 4 per lane (k is a multiple of 4): the
     * systematic copy of the raw bytes (reference :90) and the packed bits,
     * any non-zero byte a 1 (reference :43). A lane's 4 bytes give 4 bits;
     * 8 lanes OR their nibbles into one 32-bit word. */
    const int kw = (c.k + 31) / 32, k4 = c.k >> 2;
    const uint32_t* u4 = reinterpret_cast<const uint32_t*>(u);
    uint32_t* x4 = reinterpret_cast<uint32_t*>(x);
    for (int base = 0; base < k4; base += 32) {
        const int j = base + lane;
        uint32_t v = 0;
        if (j < k4) {
            v = u4[j];
            x4[j] = v;
        }
        /* bit t of the nibble: byte t of v is non-zero */
        const uint32_t nib = (((__vcmpne4(v, 0u) & 0x01010101u) * 0x01020408u) >> 24) & 0xFu;
        uint32_t wv = nib << (4 * (lane & 7));
        wv |= __shfl_xor_sync(0xffffffffu, wv, 1);
        wv |= __shfl_xor_sync(0xffffffffu, wv, 2);
        wv |= __shfl_xor_sync(0xffffffffu, wv, 4);
        if ((lane & 7) == 0) s.U[(base >> 3) + (lane >> 3)] = wv;
    }
    __syncwarp();
    if (lane < 4) s.U[kw + lane] = 0;
    __syncwarp();
    warp_encode_parity(c, s, lane);
    /* parity bytes, 4 per lane and store (z is a multiple of 4, so the 4 bits
     * never straddle a block or a word) */
    for (int q = lane; q < c.m >> 2; q += 32) {
        const int pos = q * 4;
        const int b = (int)(((unsigned)pos * c.zinv) >> 20);
        x4[k4 + q] = parity_bytes4(s, c.nw, b, pos - b * c.z);
    }
}

__global__ void __launch_bounds__(32 * kEncWarps)
framegen_kernel(CodeDesc c, FramegenArgs a)
{
    __shared__ EncScratch scratch[kEncWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long f = (long long)blockIdx.x * kEncWarps + warp;
    if (f >= a.frames) return;
    EncScratch& s = scratch[warp];
    const uint64_t g = a.first_frame + (uint64_t)f;
    /* info bits: Philox stream 0, 128 bits per block */
    const int kblk = (c.k + 127) / 128;
    for (int q = lane; q < kblk; q += 32) {
        uint32_t o[4];
        philox_at(a.seed, g, (uint32_t)q, 0u, o);
#pragma unroll
        for (int t = 0; t < 4; t++) s.U[4 * q + t] = o[t];
    }
    __syncwarp();
    /* clear the bits past k so that packed views stay canonical */
    if (lane == 0) {
        const int kw = (c.k + 31) / 32;
        if (c.k & 31) s.U[kw - 1] &= (1u << (c.k & 31)) - 1u;
        for (int t = kw; t < kw + 4; t++) s.U[t] = 0;
    }
    __syncwarp();
    warp_encode_parity(c, s, lane);

    float ebno, sigma, scale;
    frame_noise(c, a, g, ebno, sigma, scale);
    if (a.ebno_out && lane == 0) a.ebno_out[f] = ebno;

    if (a.info) {
        uint32_t* i4 = reinterpret_cast<uint32_t*>(a.info + f * c.k);
        for (int j = lane * 4; j < c.k; j += 128) {
            const uint32_t w = s.U[j >> 5] >> (j & 31);
            i4[j >> 2] = (w & 1u) | ((w & 2u) << 7) | ((w & 4u) << 14) | ((w & 8u) << 21);
        }
    }
    if (a.cw) {
        uint32_t* x4 = reinterpret_cast<uint32_t*>(a.cw + f * c.n);
        for (int j = lane * 4; j < c.k; j += 128) {
            const uint32_t w = s.U[j >> 5] >> (j & 31);
            x4[j >> 2] = (w & 1u) | ((w & 2u) << 7) | ((w & 4u) << 14) | ((w & 8u) << 21);
        }
        for (int q = lane; q < c.m >> 2; q += 32) {
            const int pos = q * 4;
            const int b = (int)(((unsigned)pos * c.zinv) >> 20);
            x4[(c.k >> 2) + q] = parity_bytes4(s, c.nw, b, pos - b * c.z);
        }
    }
    if (a.llr) {
        const uint32_t* U = s.U;
        const uint32_t* out = s.out;
        emit_llr(c, a, f, g, scale, sigma, lane, [&](int j) -> uint32_t {
            if (j < c.k) return U[j >> 5] >> (j & 31);
            const int p = j - c.k, b = (int)(((unsigned)p * c.zinv) >> 20), r = p - b * c.z;
            return out[b * c.nw + (r >> 5)] >> (r & 31);
        });
    }
}


/* Random codewords from the null space of H (any rate, 3/4B included): with
 * H in reduced row-echelon form, pivot column p_i of row i and free columns
 * F, a codeword takes random free bits u (Philox stream 0) and
 * c[p_i] = parity(A_i & u), A_i = row i restricted to F. Then the same AWGN /
 * LLR model as framegen_kernel. One warp per frame. */
__global__ void __launch_bounds__(32 * kEncWarps)
framegen_nullspace_kernel(CodeDesc c, FramegenArgs a, NullspaceArgs ns)
{
    __shared__ uint32_t s_u[kEncWarps][kMaxN / 32 + 4];
    __shared__ uint32_t s_cw[kEncWarps][kMaxN / 32 + 4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long f = (long long)blockIdx.x * kEncWarps + warp;
    if (f >= a.frames) return;
    const uint64_t g = a.first_frame + (uint64_t)f;
    uint32_t* U = s_u[warp];
    uint32_t* C = s_cw[warp];
    const int fw = (ns.nfree + 31) / 32;
    for (int q = lane; q * 4 < fw; q += 32) {
        uint32_t o[4];
        philox_at(a.seed, g, (uint32_t)q, 0u, o);
#pragma unroll
        for (int t = 0; t < 4; t++)
            if (4 * q + t < fw) U[4 * q + t] = o[t];
    }
    for (int q = lane; q < c.n / 32 + 1; q += 32) C[q] = 0u;
    __syncwarp();
    if (lane == 0 && (ns.nfree & 31)) U[fw - 1] &= (1u << (ns.nfree & 31)) - 1u;
    __syncwarp();
    /* free bits */
    for (int j = lane; j < ns.nfree; j += 32)
        if ((U[j >> 5] >> (j & 31)) & 1u) atomicOr(&C[ns.free_col[j] >> 5], 1u << (ns.free_col[j] & 31));
    /* pivot bits */
    for (int i = lane; i < ns.rank; i += 32) {
        const uint32_t* Ai = ns.A + (size_t)i * ns.words;
        uint32_t par = 0;
        for (int q = 0; q < fw; q++) par ^= __popc(Ai[q] & U[q]);
        if (par & 1u) atomicOr(&C[ns.pivot_col[i] >> 5], 1u << (ns.pivot_col[i] & 31));
    }
    __syncwarp();
    float ebno, sigma, scale;
    frame_noise(c, a, g, ebno, sigma, scale);
    if (a.ebno_out && lane == 0) a.ebno_out[f] = ebno;
    if (a.cw) {
        uint32_t* x4 = reinterpret_cast<uint32_t*>(a.cw + f * c.n);
        for (int j = lane * 4; j < c.n; j += 128) {
            const uint32_t w = C[j >> 5] >> (j & 31);
            x4[j >> 2] = (w & 1u) | ((w & 2u) << 7) | ((w & 4u) << 14) | ((w & 8u) << 21);
        }
    }
    if (a.llr) emit_llr(c, a, f, g, scale, sigma, lane, [&](int j) -> uint32_t { return C[j >> 5] >> (j & 31); });
}

/* bit*2.0-1.0 with the reference's double literals (reference
 * lib/ldpc_decoder.cc:108-118): for an int8 bit the result 2b - 1 is an odd
 * integer in [-257, 253], which a float holds exactly, so integer arithmetic
 * and an exact conversion give the float the double computation rounds to.
 * The conversion adds 2b - 1 to the mantissa of 1.5 * 2^23 (whose unit in
 * the last place is 1) and subtracts 1.5 * 2^23 again; both steps are exact
 * for |2b - 1| < 2^22. */
__device__ __forceinline__ float bit_to_llr(int b)
{
    return __int_as_float(0x4B3FFFFF + 2 * b) - 12582912.0f;
}

/* 4 bytes in and one float4 out per thread and step where the bytes are
 * 4-byte and the LLRs 16-byte aligned (both coalesced over a warp: 128 bytes
 * in, 512 out), the loads of four steps issued before any is used; a scalar
 * loop takes the rest */
__global__ void bits_to_llr_kernel(const int8_t* __restrict__ bits, float* __restrict__ llr, long long count)
{
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long nvec = ((uintptr_t)bits % 4 == 0 && (uintptr_t)llr % 16 == 0) ? count / 4 : 0;
    const unsigned int* in = reinterpret_cast<const unsigned int*>(bits);
    float4* out = reinterpret_cast<float4*>(llr);
    for (long long v = t0; v < nvec; v += 4 * stride) {
        uint32_t x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) x[u] = v + u * stride < nvec ? __ldcs(in + v + u * stride) : 0u;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (v + u * stride < nvec)   /* byte j sign-extended: (int)(x << (24 - 8j)) >> 24 */
                __stcs(out + v + u * stride,
                       make_float4(bit_to_llr((int)(x[u] << 24) >> 24), bit_to_llr((int)(x[u] << 16) >> 24),
                                   bit_to_llr((int)(x[u] << 8) >> 24), bit_to_llr((int)x[u] >> 24)));
    }
    for (long long i = nvec * 4 + t0; i < count; i += stride) llr[i] = bit_to_llr(bits[i]);
}

/* The reference BER_runner's info-bit stream (reference lib/BER_runner.cc:35-41,
 * 124-146): an LFSR x^31 + x^28 + 1 from 0xdeadbeef, restarted every 115200
 * bits, so the stream is periodic. g_lfsr_period holds one period packed 32
 * bits per word (written once per device from the host); bit p of the stream
 * is bit (p mod 115200) of the period. */
constexpr int kLfsrPeriod = 115200;
__device__ uint32_t g_lfsr_period[kLfsrPeriod / 32];

/* 16 bits of the period from bit p on (p < kLfsrPeriod), wrapping at the
 * period's end, which falls on a word boundary */
__device__ __forceinline__ uint32_t lfsr_bits16(unsigned p)
{
    constexpr unsigned kWords = kLfsrPeriod / 32;
    const unsigned w = p >> 5;
    const uint32_t lo = g_lfsr_period[w], hi = g_lfsr_period[w + 1 == kWords ? 0 : w + 1];
    return __funnelshift_r(lo, hi, p & 31) & 0xFFFFu;
}

/* Output bytes 0/1. Where out is 16-byte aligned, a thread writes 16 bytes
 * per step (one modulo per 16 bits, the bits expanded to bytes by
 * multiplication, one 16-byte store); a scalar loop takes the rest. */
__global__ void lfsr_bits_kernel(unsigned long long first_bit, long long nbits, uint8_t* __restrict__ out)
{
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long nvec = ((uintptr_t)out % 16 == 0) ? nbits / 16 : 0;
    for (long long g = t0; g < nvec; g += stride) {
        const unsigned p = (unsigned)((first_bit + 16ull * (unsigned long long)g) % kLfsrPeriod);
        const uint32_t b = lfsr_bits16(p);
        __stcs(reinterpret_cast<uint4*>(out) + g,
               make_uint4(((b & 0xFu) * 0x00204081u) & 0x01010101u, (((b >> 4) & 0xFu) * 0x00204081u) & 0x01010101u,
                          (((b >> 8) & 0xFu) * 0x00204081u) & 0x01010101u,
                          (((b >> 12) & 0xFu) * 0x00204081u) & 0x01010101u));
    }
    for (long long j = nvec * 16 + t0; j < nbits; j += stride) {
        const unsigned p = (unsigned)((first_bit + (unsigned long long)j) % kLfsrPeriod);
        out[j] = (uint8_t)((g_lfsr_period[p >> 5] >> (p & 31)) & 1u);
    }
}

/* How long the decoders' bounded wait with limit limit_us takes on an
 * mbarrier phase that never completes: one thread initialises a barrier
 * expecting two arrivals, arrives once, runs the wait on it and records the
 * elapsed global-timer nanoseconds and whether the wait (wrongly)
 * succeeded. Nothing is copied, so nothing is in flight when it exits. */
__global__ void wait_bound_kernel(uint32_t limit_us, unsigned long long* out)
{
    __shared__ __align__(8) uint64_t bar;
    mbar_init(&bar, 2);
    fence_mbar_init();
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bar)) : "memory");
    const unsigned long long t0 = global_ns();
    const bool ok = mbar_wait_bounded(&bar, 0, limit_us);
    out[0] = global_ns() - t0;
    out[1] = ok ? 1ull : 0ull;
}

cudaError_t launch_wait_bound(uint32_t limit_us, unsigned long long* out, cudaStream_t st)
{
    wait_bound_kernel<<<1, 1, 0, st>>>(limit_us, out);
    return cudaGetLastError();
}

cudaError_t upload_lfsr_period(const uint32_t* words)
{
    return cudaMemcpyToSymbol(g_lfsr_period, words, sizeof(uint32_t) * (kLfsrPeriod / 32));
}

cudaError_t launch_lfsr_bits(unsigned long long first_bit, long long nbits, uint8_t* out, cudaStream_t st)
{
    if (nbits <= 0) return cudaSuccess;
    long long blocks = (nbits / 16 + 255) / 256 + 1;
    if (blocks > 148 * 16) blocks = 148 * 16;
    lfsr_bits_kernel<<<(unsigned)blocks, 256, 0, st>>>(first_bit, nbits, out);
    return cudaGetLastError();
}

/* ---------------------------------------------------------------- launchers */

extern const EncLanesLaunch kEncLanes_r0[kNumZ];
extern const EncLanesLaunch kEncLanes_r1[kNumZ];
extern const EncLanesLaunch kEncLanes_r2[kNumZ];
extern const EncLanesLaunch kEncLanes_r3[kNumZ];
extern const EncLanesLaunch kEncLanes_r5[kNumZ];

const EncLanesLaunch* enc_lanes_entry(int rate, int z)
{
    static const EncLanesLaunch* const tables[kRates] = {kEncLanes_r0, kEncLanes_r1, kEncLanes_r2,
                                                         kEncLanes_r3, nullptr, kEncLanes_r5};
    if (!valid_rate(rate) || !valid_z(z) || !tables[rate]) return nullptr;
    return &tables[rate][z_index(z)];
}

cudaError_t launch_encode_bytes(const CodeDesc& c, const uint8_t* info, uint8_t* cw, long long frames,
                                cudaStream_t st)
{
    if (frames <= 0) return cudaSuccess;
    const EncLanesLaunch* e = enc_lanes_entry(c.rate, c.z);
    if (e && ((uintptr_t)info % e->align) == 0 && ((uintptr_t)cw % e->align) == 0) {
        const long long frames_per_cta = e->threads;   /* one frame per thread */
        e->kernel<<<(unsigned)((frames + frames_per_cta - 1) / frames_per_cta), e->threads, 0, st>>>(info, cw,
                                                                                                   frames);
        return cudaGetLastError();
    }
    const long long blocks = (frames + kEncWarps - 1) / kEncWarps;
    encode_bytes_kernel<<<(unsigned)blocks, 32 * kEncWarps, 0, st>>>(c, info, cw, frames);
    return cudaGetLastError();
}

cudaError_t launch_framegen(const CodeDesc& c, const FramegenArgs& a, cudaStream_t st)
{
    if (a.frames <= 0) return cudaSuccess;
    const long long blocks = (a.frames + kEncWarps - 1) / kEncWarps;
    framegen_kernel<<<(unsigned)blocks, 32 * kEncWarps, 0, st>>>(c, a);
    return cudaGetLastError();
}

cudaError_t launch_framegen_nullspace(const CodeDesc& c, const FramegenArgs& a, const NullspaceArgs& ns,
                                      cudaStream_t st)
{
    if (a.frames <= 0) return cudaSuccess;
    const long long blocks = (a.frames + kEncWarps - 1) / kEncWarps;
    framegen_nullspace_kernel<<<(unsigned)blocks, 32 * kEncWarps, 0, st>>>(c, a, ns);
    return cudaGetLastError();
}

extern const SynLanesLaunch kSynLanes_r0[kNumZ];
extern const SynLanesLaunch kSynLanes_r1[kNumZ];
extern const SynLanesLaunch kSynLanes_r2[kNumZ];
extern const SynLanesLaunch kSynLanes_r3[kNumZ];
extern const SynLanesLaunch kSynLanes_r4[kNumZ];
extern const SynLanesLaunch kSynLanes_r5[kNumZ];

const SynLanesLaunch* syn_lanes_entry(int rate, int z)
{
    static const SynLanesLaunch* const tables[kRates] = {kSynLanes_r0, kSynLanes_r1, kSynLanes_r2,
                                                         kSynLanes_r3, kSynLanes_r4, kSynLanes_r5};
    if (!valid_rate(rate) || !valid_z(z)) return nullptr;
    return &tables[rate][z_index(z)];
}

cudaError_t launch_syndrome(const CodeDesc& c, const int8_t* bits, uint32_t* out, long long frames,
                            int early_exit, cudaStream_t st)
{
    if (frames <= 0) return cudaSuccess;
    const SynLanesLaunch* e = syn_lanes_entry(c.rate, c.z);
    if (!e || ((uintptr_t)bits % 16) != 0 || ((uintptr_t)out % 4) != 0) return cudaErrorInvalidValue;
    const long long frames_per_cta = e->threads;   /* one frame per thread */
    e->kernel<<<(unsigned)((frames + frames_per_cta - 1) / frames_per_cta), e->threads, 0, st>>>(bits, out, frames,
                                                                                               early_exit);
    return cudaGetLastError();
}

cudaError_t launch_bits_to_llr(const int8_t* bits, float* llr, long long count, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    long long blocks = (count / 4 + 255) / 256 + 1;
    if (blocks > 148 * 32) blocks = 148 * 32;
    bits_to_llr_kernel<<<(unsigned)blocks, 256, 0, st>>>(bits, llr, count);
    return cudaGetLastError();
}

}  // namespace wldpc
