/* Lane-per-frame compute_syndrome for rate enum 1, specialised on each of
 * the 19 expansion factors (syndrome_lanes.cuh). */
#include "codec_kernels.cuh"
#include "syndrome_lanes.cuh"

namespace wldpc {

#define WLDPC_SYN_LANES(Z) {&syndrome_lanes_kernel<1, Z>, SynLanes<1, Z>::THREADS}

extern const SynLanesLaunch kSynLanes_r1[kNumZ] = {
    WLDPC_SYN_LANES(24), WLDPC_SYN_LANES(28), WLDPC_SYN_LANES(32), WLDPC_SYN_LANES(36), WLDPC_SYN_LANES(40),
    WLDPC_SYN_LANES(44), WLDPC_SYN_LANES(48), WLDPC_SYN_LANES(52), WLDPC_SYN_LANES(56), WLDPC_SYN_LANES(60),
    WLDPC_SYN_LANES(64), WLDPC_SYN_LANES(68), WLDPC_SYN_LANES(72), WLDPC_SYN_LANES(76), WLDPC_SYN_LANES(80),
    WLDPC_SYN_LANES(84), WLDPC_SYN_LANES(88), WLDPC_SYN_LANES(92), WLDPC_SYN_LANES(96),
};

}  // namespace wldpc
