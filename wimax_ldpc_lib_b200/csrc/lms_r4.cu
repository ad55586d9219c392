/* Learned min-sum decoder and training kernels for rate enum 4 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<4, Z>, LmsShape<4, Z>::THREADS, LmsShape<4, Z>::G, LmsShape<4, Z>::SMEM, \
     &lms_train_kernel<4, Z>, LmsTrainShape<4, Z>::SMEM, \
     &lms16_decode_kernel<4, Z>, Lms16Shape<4, Z>::THREADS, Lms16Shape<4, Z>::FRAMES}

extern const LmsLaunch kLms_r4[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
