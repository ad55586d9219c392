/*
 * Persistent decoder for batches that mix codes (all six rates, all 19 z),
 * with the plain normalized min-sum arithmetic of nms_decode.cuh (bit-exact
 * with the reference, reference lib/ldpc_decoder.cc:122-262).
 *
 * One launch decodes the whole batch:
 *   1. binning (mixed_count / mixed_plan / mixed_scatter): frames are
 *      grouped by code (variant = rate * 19 + z index) and cut into work
 *      items of at most `chunk` frames of one code;
 *   2. mixed_decode_kernel<rate>: one persistent grid per rate, all six
 *      launched concurrently; each CTA takes work items of its rate from that
 *      rate's counter. Within an item the CTA runs G = THREADS / z frame
 *      slots in lockstep (one thread per expanded row, as the specialised
 *      kernel) and refills a slot with the item's next frame as soon as its
 *      frame converges or reaches the cap (early-exit compaction), so no slot
 *      idles while the item has frames left. A refilled frame gets its initial
 *      syndrome check before its first iteration, as in the reference
 *      (reference lib/ldpc_decoder.cc:127-139).
 * Codes are read from a __constant__ table (z, block columns x z, shifts);
 * each rate has its own kernel (one kernel for all six would need the union
 * of their registers), z is a run-time value, and each thread's edge
 * addresses for the current code sit in a shared-memory table. The binning
 * kernels and the six decode kernels (forked onto six streams) are captured
 * in one CUDA graph, so a batch is one graph launch.
 */
#ifndef WLDPC_MIXED_CUH
#define WLDPC_MIXED_CUH

#include <cstdint>
#include "codes.h"
#include "device_util.cuh"
#include "nms_decode.cuh"

namespace wldpc {

constexpr int kVariants = kRates * kNumZ;   /* 114 */

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
    const long long* offset;    /* per frame: element offset of its n values */
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
};

}  // namespace wldpc

#endif
