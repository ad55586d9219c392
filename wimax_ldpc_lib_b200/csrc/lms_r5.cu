/* Learned min-sum decoder and training kernels for rate enum 5 at the
 * expansion factors the learned path supports (z = 24, 48, 96). */
#include "lms_dispatch.cuh"

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z) \
    {Z, &lms_decode_kernel<5, Z>, LmsShape<5, Z>::THREADS, LmsShape<5, Z>::G, LmsShape<5, Z>::SMEM, \
     &lms_train_kernel<5, Z>, LmsTrainShape<5, Z>::SMEM, \
     &lms16_decode_kernel<5, Z>, Lms16Shape<5, Z>::THREADS, Lms16Shape<5, Z>::FRAMES}

extern const LmsLaunch kLms_r5[kLmsNumZ] = {WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(96)};

}  // namespace wldpc
