/* Learned min-sum decoder and training kernels for rate enum 1 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<1, Z>, LmsShape<1, Z>::THREADS, LmsShape<1, Z>::G, LmsShape<1, Z>::SMEM, \
     &lms_train_kernel<1, Z>, LmsTrainShape<1, Z>::SMEM, \
     &lms16_decode_kernel<1, Z>, Lms16Shape<1, Z>::THREADS, Lms16Shape<1, Z>::FRAMES}

extern const LmsLaunch kLms_r1[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
