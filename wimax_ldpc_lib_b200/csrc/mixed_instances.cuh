/* Instantiation unit of the mixed-code decode kernels (mixed_kernel.cuh) for
 * one code rate: the Makefile compiles it once per rate as CUDA with
 * -DWLDPC_MIXED_RATE=r, so the 48 kernels (6 rates x CTA size 96 or 192 x
 * messages in registers or shared memory x one or two rows per thread, each
 * with a body for all 19 z) build in parallel translation units. It defines
 * the dispatch row kMixed_r<r>[threads][layout][rows - 1] that mixed.cu
 * looks up. */
#include "mixed_kernel.cuh"

#if !defined(WLDPC_MIXED_RATE)
#error "compile with -DWLDPC_MIXED_RATE=<0..5>"
#endif

namespace wldpc {

#define WLDPC_MIXED_PASTE2(a, b) a##b
#define WLDPC_MIXED_PASTE(a, b) WLDPC_MIXED_PASTE2(a, b)

#define WLDPC_MIXED_K(T, L, RPT) &mixed_decode_kernel<WLDPC_MIXED_RATE, T, L, RPT>

extern const MixedKernel WLDPC_MIXED_PASTE(kMixed_r, WLDPC_MIXED_RATE)[2][2][2] = {
    {{WLDPC_MIXED_K(96, kMsgRegisters, 1), WLDPC_MIXED_K(96, kMsgRegisters, 2)},
     {WLDPC_MIXED_K(96, kMsgShared, 1), WLDPC_MIXED_K(96, kMsgShared, 2)}},
    {{WLDPC_MIXED_K(192, kMsgRegisters, 1), WLDPC_MIXED_K(192, kMsgRegisters, 2)},
     {WLDPC_MIXED_K(192, kMsgShared, 1), WLDPC_MIXED_K(192, kMsgShared, 2)}}};

}  // namespace wldpc
