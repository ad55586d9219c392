/* Learned min-sum decoder and training kernels for rate enum 3 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<3, Z>, LmsShape<3, Z>::THREADS, LmsShape<3, Z>::G, LmsShape<3, Z>::SMEM, \
     &lms_train_kernel<3, Z>, LmsTrainShape<3, Z>::SMEM, \
     &lms16_decode_kernel<3, Z>, Lms16Shape<3, Z>::THREADS, Lms16Shape<3, Z>::FRAMES}

extern const LmsLaunch kLms_r3[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
