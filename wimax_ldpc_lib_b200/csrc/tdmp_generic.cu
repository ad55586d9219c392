/* Offset and plain min-sum TDMP decoders (the reference's alternative
 * compile-time flavours, reference lib/ldpc_decoder.cc:20-21,227-237),
 * specialised on the rate with z a run-time value: one frame per CTA. */
#include "codec_kernels.cuh"

namespace wldpc {

#define WLDPC_TDMP_GEN(R, M) {&tdmp_decode_kernel<R, 0, M>, 0, 1, 0, true}

extern const TdmpLaunch kTdmpGeneric[kRates][2] = {
    {WLDPC_TDMP_GEN(0, kOms), WLDPC_TDMP_GEN(0, kMs)}, {WLDPC_TDMP_GEN(1, kOms), WLDPC_TDMP_GEN(1, kMs)},
    {WLDPC_TDMP_GEN(2, kOms), WLDPC_TDMP_GEN(2, kMs)}, {WLDPC_TDMP_GEN(3, kOms), WLDPC_TDMP_GEN(3, kMs)},
    {WLDPC_TDMP_GEN(4, kOms), WLDPC_TDMP_GEN(4, kMs)}, {WLDPC_TDMP_GEN(5, kOms), WLDPC_TDMP_GEN(5, kMs)},
};

}  // namespace wldpc
