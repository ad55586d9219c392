/* Dispatch of the TDMP decoders: NMS specialised on (rate, z), OMS / MS on
 * the rate with z at run time. */
#include "codec_kernels.cuh"

namespace wldpc {

extern const TdmpLaunch kTdmpNms_r0[kNumZ];
extern const TdmpLaunch kTdmpNms_r1[kNumZ];
extern const TdmpLaunch kTdmpNms_r2[kNumZ];
extern const TdmpLaunch kTdmpNms_r3[kNumZ];
extern const TdmpLaunch kTdmpNms_r4[kNumZ];
extern const TdmpLaunch kTdmpNms_r5[kNumZ];
extern const TdmpLaunch kTdmpGeneric[kRates][2];

static const TdmpLaunch* const kNmsTables[kRates] = {kTdmpNms_r0, kTdmpNms_r1, kTdmpNms_r2,
                                               kTdmpNms_r3, kTdmpNms_r4, kTdmpNms_r5};

const TdmpLaunch* tdmp_entry(int rate, int z, int mode)
{
    if (!valid_rate(rate) || !valid_z(z) || mode < 0 || mode > 2) return nullptr;
    if (mode == kNms) return &kNmsTables[rate][z_index(z)];
    return &kTdmpGeneric[rate][mode - 1];
}

cudaError_t launch_tdmp(int rate, int z, int mode, const DecodeArgs& args, cudaStream_t st)
{
    const TdmpLaunch* e = tdmp_entry(rate, z, mode);
    if (!e) return cudaErrorInvalidValue;
    if (args.frames <= 0) return cudaSuccess;
    DecodeArgs a = args;
    int threads = e->threads, smem = e->smem;
    if (e->runtime_z) {
        const CodeDesc c = make_code_desc(rate, z);
        a.z = z;
        for (int b = 0; b < c.nblk; b++) {
            a.shift[b] = c.shift[b];
            a.colz[b] = (unsigned short)(c.col[b] * z);
        }
        threads = z;
        smem = c.n * 4;
    }
    const long long ctas = (a.frames + e->frames_per_cta - 1) / e->frames_per_cta;
    if (ctas > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) {
        cudaError_t err = cudaFuncSetAttribute(e->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (err != cudaSuccess) return err;
    }
    e->kernel<<<(unsigned)ctas, threads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace wldpc
