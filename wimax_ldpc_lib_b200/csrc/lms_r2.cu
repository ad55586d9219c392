/* Learned min-sum decoder and training kernels for rate enum 2 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<2, Z>, LmsShape<2, Z>::THREADS, LmsShape<2, Z>::G, LmsShape<2, Z>::SMEM, \
     &lms_train_kernel<2, Z>, LmsTrainShape<2, Z>::SMEM, \
     &lms16_decode_kernel<2, Z>, Lms16Shape<2, Z>::THREADS, Lms16Shape<2, Z>::FRAMES}

extern const LmsLaunch kLms_r2[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
