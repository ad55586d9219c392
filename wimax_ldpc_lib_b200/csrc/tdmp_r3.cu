/* Normalized min-sum TDMP decoders for rate enum 3, specialised on each of
 * the 19 expansion factors (the shipped reference flavour, the hot path). */
#include "codec_kernels.cuh"

namespace wldpc {

#define WLDPC_TDMP_NMS(Z) \
    {&tdmp_decode_kernel<3, Z, kNms>, TdmpShape<3, Z>::THREADS, TdmpShape<3, Z>::G, TdmpShape<3, Z>::SMEM, false}

extern const TdmpLaunch kTdmpNms_r3[kNumZ] = {
    WLDPC_TDMP_NMS(24), WLDPC_TDMP_NMS(28), WLDPC_TDMP_NMS(32), WLDPC_TDMP_NMS(36), WLDPC_TDMP_NMS(40),
    WLDPC_TDMP_NMS(44), WLDPC_TDMP_NMS(48), WLDPC_TDMP_NMS(52), WLDPC_TDMP_NMS(56), WLDPC_TDMP_NMS(60),
    WLDPC_TDMP_NMS(64), WLDPC_TDMP_NMS(68), WLDPC_TDMP_NMS(72), WLDPC_TDMP_NMS(76), WLDPC_TDMP_NMS(80),
    WLDPC_TDMP_NMS(84), WLDPC_TDMP_NMS(88), WLDPC_TDMP_NMS(92), WLDPC_TDMP_NMS(96),
};

}  // namespace wldpc
