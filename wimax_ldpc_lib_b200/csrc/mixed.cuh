/*
 * Persistent decoder for batches that mix codes (all six rates, all 19 z),
 * with the plain normalized min-sum arithmetic of nms_decode.cuh (bit-exact
 * with the reference, reference lib/ldpc_decoder.cc:122-262).
 *
 * One launch decodes the whole batch:
 *   1. binning (mixed_count / mixed_plan / mixed_scatter): frames are
 *      grouped by code (variant = rate * 19 + z index) and cut into work
 *      items of at most `chunk` frames of one code;
 *   2. mixed_decode_kernel<rate, threads, layout, rows> (mixed_kernel.cuh):
 *      one persistent grid per rate, the six launched concurrently or one
 *      after another; each CTA takes work items of its rate from that rate's
 *      counter. The CTA runs G = threads * rows / z frame slots in lockstep
 *      (rows = 1 or 2 expanded rows per thread; z a run-time value, edge
 *      addresses from a per-item shared-memory table)
 *      and refills a slot with the item's next frame (one bulk copy) as soon
 *      as its frame converges or reaches the cap (early-exit compaction). A
 *      refilled frame gets its initial syndrome check before its first
 *      iteration, as in the reference (reference lib/ldpc_decoder.cc:127-139).
 * The binning kernels and the six decode grids (forked onto six streams) are
 * captured in one CUDA graph, so a batch is one graph launch. CTA size, rows
 * per thread (threads per z), message layout (registers or shared memory),
 * chunk and launch policy are picked by the handle's autotuner.
 */
#ifndef WLDPC_MIXED_CUH
#define WLDPC_MIXED_CUH

#include <cstdint>
#include "codes.h"
#include "device_util.cuh"
#include "nms_decode.cuh"

namespace wldpc {

constexpr int kVariants = kRates * kNumZ;   /* 114 */
constexpr int kMixedMaxSlots = 16;         /* frames per CTA: 192 threads x 2 rows / z = 24 */
constexpr int kMixedMaxChunk = 64;         /* frames per work item */

/* one code of a rate, as the mixed kernel needs it (z at run time) */
struct MixedCode {
    unsigned short z, n;
    unsigned short colz[96];    /* block column * z, row-major block order */
    unsigned char shift[96];
};

struct MixedItem {
    int variant;
    int start;                  /* into the sorted frame list */
    int count;
};

struct MixedArgs {
    const uint8_t* variant;     /* per frame: rate * 19 + (z - 24) / 4 */
    const long long* offset;    /* per frame: element offset of its n values (a multiple of 4) */
    const float* llr;
    int8_t* hard;
    float* post;                /* or null */
    int32_t* status;            /* per frame, or null */
    const int* perm;            /* frames sorted by variant */
    const MixedItem* items;     /* per rate: items_per_rate entries */
    const int* num_items;       /* per rate */
    int* queue;                 /* per rate: work-item counter, zero at launch */
    long long items_per_rate;
    unsigned* err;
    long long frames;
    int max_iter;
    MixedCode codes[kNumZ];     /* the launched rate's 19 codes, by z index */
};

}  // namespace wldpc

#endif
