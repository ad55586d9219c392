/* Lane-per-frame encoders for rate enum 5, specialised on each of the 19
 * expansion factors (encode_lanes.cuh). */
#include "codec_kernels.cuh"
#include "encode_lanes.cuh"

namespace wldpc {

#define WLDPC_ENC_LANES(Z) {&encode_lanes_kernel<5, Z>, EncLanes<5, Z>::CB, EncLanes<5, Z>::THREADS}

extern const EncLanesLaunch kEncLanes_r5[kNumZ] = {
    WLDPC_ENC_LANES(24), WLDPC_ENC_LANES(28), WLDPC_ENC_LANES(32), WLDPC_ENC_LANES(36), WLDPC_ENC_LANES(40),
    WLDPC_ENC_LANES(44), WLDPC_ENC_LANES(48), WLDPC_ENC_LANES(52), WLDPC_ENC_LANES(56), WLDPC_ENC_LANES(60),
    WLDPC_ENC_LANES(64), WLDPC_ENC_LANES(68), WLDPC_ENC_LANES(72), WLDPC_ENC_LANES(76), WLDPC_ENC_LANES(80),
    WLDPC_ENC_LANES(84), WLDPC_ENC_LANES(88), WLDPC_ENC_LANES(92), WLDPC_ENC_LANES(96),
};

}  // namespace wldpc
