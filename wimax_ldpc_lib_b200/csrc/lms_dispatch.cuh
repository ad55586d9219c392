/* Dispatch table of the learned min-sum kernels (lms.cuh, lms16.cuh). */
#ifndef WLDPC_LMS_DISPATCH_CUH
#define WLDPC_LMS_DISPATCH_CUH

#include "lms.cuh"
#include "lms16.cuh"

namespace wldpc {

/* every code has learned kernels: 19 expansion factors, instantiated in two
 * halves per rate (lms_instances.cuh), z = 24..56 and z = 60..96 */
constexpr int kLmsHalf0 = 9;

struct LmsLaunch {
    int z;
    void (*decode)(const LmsArgs);
    int threads, frames_per_cta, smem;
    void (*train)(const LmsTrainArgs);
    int train_smem;          /* train CTA = z threads, one frame */
    void (*decode16)(const Lms16Args);   /* packed-half decoder (lms16.cuh) */
    int threads16, frames16;             /* its CTA size and frames per CTA (static shared memory) */
};

const LmsLaunch* lms_entry(int rate, int z);

}  // namespace wldpc

#endif
