/* Learned min-sum decoder and training kernels for rate enum 0 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<0, Z>, LmsShape<0, Z>::THREADS, LmsShape<0, Z>::G, LmsShape<0, Z>::SMEM, \
     &lms_train_kernel<0, Z>, LmsTrainShape<0, Z>::SMEM, \
     &lms16_decode_kernel<0, Z>, Lms16Shape<0, Z>::THREADS, Lms16Shape<0, Z>::FRAMES}

extern const LmsLaunch kLms_r0[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
