/* Instantiation unit of the learned min-sum kernels (lms.cuh, lms16.cuh) for
 * one code rate and one half of the 19 expansion factors. The Makefile
 * compiles it once per (rate, half) as CUDA with -DWLDPC_LMS_RATE=r and
 * -DWLDPC_LMS_HALF=h (h = 0: z = 24..56, h = 1: z = 60..96), so the 342
 * kernels (decoder, training and packed-binary16 decoder for 114 codes) build
 * in 12 parallel translation units. Each unit defines the dispatch rows
 * kLms_r<r>_h<h>[] that lms_entry() (lms_capi.cu) looks up. */
#include "lms_dispatch.cuh"

#if !defined(WLDPC_LMS_RATE) || !defined(WLDPC_LMS_HALF)
#error "compile with -DWLDPC_LMS_RATE=<0..5> -DWLDPC_LMS_HALF=<0|1>"
#endif

namespace wldpc {

#define WLDPC_LMS_ENTRY(Z)                                                                                     \
    {Z, &lms_decode_kernel<WLDPC_LMS_RATE, Z>, LmsShape<WLDPC_LMS_RATE, Z>::THREADS,                           \
     LmsShape<WLDPC_LMS_RATE, Z>::G, LmsShape<WLDPC_LMS_RATE, Z>::SMEM, &lms_train_kernel<WLDPC_LMS_RATE, Z>, \
     LmsTrainShape<WLDPC_LMS_RATE, Z>::SMEM, &lms16_decode_kernel<WLDPC_LMS_RATE, Z>,                         \
     Lms16Shape<WLDPC_LMS_RATE, Z>::THREADS, Lms16Shape<WLDPC_LMS_RATE, Z>::FRAMES}

#define WLDPC_LMS_PASTE2(a, b, c, d) a##b##c##d
#define WLDPC_LMS_PASTE(a, b, c, d) WLDPC_LMS_PASTE2(a, b, c, d)
#define WLDPC_LMS_TABLE WLDPC_LMS_PASTE(kLms_r, WLDPC_LMS_RATE, _h, WLDPC_LMS_HALF)

#if WLDPC_LMS_HALF == 0
extern const LmsLaunch WLDPC_LMS_TABLE[kLmsHalf0] = {
    WLDPC_LMS_ENTRY(24), WLDPC_LMS_ENTRY(28), WLDPC_LMS_ENTRY(32), WLDPC_LMS_ENTRY(36), WLDPC_LMS_ENTRY(40),
    WLDPC_LMS_ENTRY(44), WLDPC_LMS_ENTRY(48), WLDPC_LMS_ENTRY(52), WLDPC_LMS_ENTRY(56)};
#else
extern const LmsLaunch WLDPC_LMS_TABLE[kNumZ - kLmsHalf0] = {
    WLDPC_LMS_ENTRY(60), WLDPC_LMS_ENTRY(64), WLDPC_LMS_ENTRY(68), WLDPC_LMS_ENTRY(72), WLDPC_LMS_ENTRY(76),
    WLDPC_LMS_ENTRY(80), WLDPC_LMS_ENTRY(84), WLDPC_LMS_ENTRY(88), WLDPC_LMS_ENTRY(92), WLDPC_LMS_ENTRY(96)};
#endif

}  // namespace wldpc
