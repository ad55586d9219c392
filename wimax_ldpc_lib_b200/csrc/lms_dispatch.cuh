/* Dispatch table of the learned min-sum kernels (lms.cuh). */
#ifndef WLDPC_LMS_DISPATCH_CUH
#define WLDPC_LMS_DISPATCH_CUH

#include "lms.cuh"

namespace wldpc {

constexpr int kLmsNumZ = 3;   /* z = 24, 48, 96 */

struct LmsLaunch {
    int z;
    void (*decode)(const LmsArgs);
    int threads, frames_per_cta, smem;
    void (*train)(const LmsTrainArgs);
    int train_smem;          /* train CTA = z threads, one frame */
};

const LmsLaunch* lms_entry(int rate, int z);

}  // namespace wldpc

#endif
