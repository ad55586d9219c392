/*
 * wimax_ldpc_b200 -- C ABI of the B200-native WiMAX (IEEE 802.16e) QC-LDPC codec.
 *
 * The reference library (myersw12/wimax_ldpc_lib) exposes C++ classes only
 * (reference include/ldpc_decoder.h, include/ldpc_encoder.h,
 * include/BER_runner.h) and has no FFI of its own. This header is the flat
 * boundary those classes map onto: one opaque handle per reference object,
 * one entry point per public method, plain pointers and sizes, int status
 * codes. The C++ facade in include/wimax_ldpc_lib/ re-creates the reference
 * classes on top of it; a ctypes / cgo / JNI binding binds these symbols.
 *
 * Conventions (same as the reference):
 *   rate   coderate enum: 0 = 1/2, 1 = 2/3A, 2 = 2/3B, 3 = 3/4A, 4 = 3/4B, 5 = 5/6
 *          (reference include/enums.h:4-12)
 *   z      expansion factor 24..96 step 4; n = 24*z (reference lib/ldpc.cc:15-16)
 *   LLR    positive means bit 1; hard decision is x >= 0 (reference
 *          lib/ldpc_decoder.cc:130,242; BPSK bit*2-1 in lib/BER_runner.cc:183)
 *
 * Every function returns WLDPC_OK (0) or a negative WLDPC_ERR_* code.
 * Handles are not thread-safe (one per host thread), like the reference
 * objects, which share per-object scratch (reference lib/ldpc_decoder.cc:36).
 * The product path runs on the GPU only; without a CUDA device, calls that
 * compute return WLDPC_ERR_NO_DEVICE.
 */
#ifndef WIMAX_LDPC_B200_H
#define WIMAX_LDPC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define WLDPC_API __attribute__((visibility("default")))
#else
#define WLDPC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define WLDPC_OK 0
#define WLDPC_ERR_ARG (-1)          /* null / misaligned pointer, bad size or mode */
#define WLDPC_ERR_CODE (-2)         /* invalid rate or z; the reference throws std::exception */
#define WLDPC_ERR_CUDA (-3)         /* a CUDA runtime call or kernel launch failed */
#define WLDPC_ERR_NO_DEVICE (-4)    /* no usable CUDA device */
#define WLDPC_ERR_TIMEOUT (-5)      /* a bounded device-side wait expired */
#define WLDPC_ERR_UNSUPPORTED (-6)  /* operation not available for this code */
#define WLDPC_ERR_SCRATCH (-7)      /* request larger than the allocation-free entry point's scratch */

/* Decoder flavours: the reference's compile-time switch (reference
 * lib/ldpc_decoder.cc:17-21), selectable at run time here. */
#define WLDPC_MODE_NMS 0            /* normalized min-sum x0.815, as shipped */
#define WLDPC_MODE_OMS 1            /* offset min-sum, offset 0.10 */
#define WLDPC_MODE_MS 2             /* plain min-sum */

WLDPC_API const char* wldpc_strerror(int code);
/* ABI version: major * 10000 + minor * 100 + patch */
WLDPC_API int wldpc_version(void);

/* ------------------------------------------------------------ code tables */

typedef struct wldpc_code_info {
    int rate, z;
    int n;        /* codeword bits, reference m_N (lib/ldpc.cc:16) */
    int m;        /* parity bits, reference m_M (lib/ldpc.cc:18-44) */
    int k;        /* info bits, n - m */
    int rows;     /* expanded check rows, reference m_row_size */
    int cols;     /* max row degree, reference m_col_size */
    int D, X;     /* encoder constants, reference m_D / m_X */
    int layers;   /* base rows */
    int edges;    /* non-zero entries of H */
} wldpc_code_info;

/* Replaces ldpc::ldpc(rate, z, threads) + set_checknode_array (reference
 * lib/ldpc.cc:11-62,69-1206): WLDPC_ERR_CODE where the reference throws. */
WLDPC_API int wldpc_code_info_get(int rate, unsigned z, wldpc_code_info* out);

/* The expanded check-node table in the reference's layout: int16
 * [rows][cols], -1 padded (reference lib/matrices/wimax_N_RATE.cc).
 * capacity is in elements. */
WLDPC_API int wldpc_checknode_table(int rate, unsigned z, int16_t* out, size_t capacity);

/* ---------------------------------------------------------------- decoder */

typedef struct wldpc_decoder wldpc_decoder;

/* Replaces ldpc_decoder::ldpc_decoder(rate, z, max_iter, num_threads)
 * (reference include/ldpc_decoder.h:25-28, lib/ldpc_decoder.cc:27-59).
 * num_threads is kept for signature parity and unused, as in the reference.
 * mode is WLDPC_MODE_*; the reference build is WLDPC_MODE_NMS. */
WLDPC_API int wldpc_decoder_create(int rate, unsigned z, unsigned max_iter, unsigned num_threads, int mode,
                         wldpc_decoder** out);
/* Replaces ldpc_decoder::~ldpc_decoder (reference lib/ldpc_decoder.cc:61-65). */
WLDPC_API int wldpc_decoder_destroy(wldpc_decoder* dec);

/* Replaces unsigned ldpc_decoder::decode(float* rx_codeword, int8_t* decoded)
 * (reference include/ldpc_decoder.h:33, lib/ldpc_decoder.cc:122-262). Host
 * pointers. rx_codeword (n floats) is overwritten with the posterior LLRs and
 * decoded receives n bytes 0/1, exactly as the reference. *num_errors gets the
 * reference's return value: 0 when the syndrome is satisfied (and always 0
 * when max_iter == 0), 1 otherwise. *iterations (nullable) receives the
 * iterations executed, which the reference does not report. Synchronous. */
WLDPC_API int wldpc_decoder_decode(wldpc_decoder* dec, float* rx_codeword, int8_t* decoded, unsigned* num_errors,
                         int* iterations);

/* Replaces unsigned ldpc_decoder::decode(int8_t* rx_codeword, int8_t* decoded)
 * (reference include/ldpc_decoder.h:32, lib/ldpc_decoder.cc:108-118): the
 * bytes are mapped to bit*2.0-1.0 and decoded; the input is not modified. */
WLDPC_API int wldpc_decoder_decode_bits(wldpc_decoder* dec, const int8_t* rx_codeword, int8_t* decoded,
                              unsigned* num_errors);

/* Replaces unsigned ldpc_decoder::compute_syndrome(int8_t*, bool)
 * (reference include/ldpc_decoder.h:31, lib/ldpc_decoder.cc:67-104): number
 * of failing check rows (row parity is the XOR of the bytes), or 0/1 when
 * exit_early is non-zero. */
WLDPC_API int wldpc_decoder_compute_syndrome(wldpc_decoder* dec, const int8_t* rx_codeword, int exit_early,
                                   unsigned* num_errors);

/* Batched decode on device memory, asynchronous on `stream` (a cudaStream_t;
 * NULL is the CUDA default stream). The batch form of decode(float*, int8_t*):
 *   llr       frames x n float32, 16-byte aligned
 *   decoded   frames x n int8 (0/1), 4-byte aligned
 *   posterior frames x n float32 or NULL, 16-byte aligned; may equal llr
 *             (in-place posterior, the reference's semantics)
 *   status    frames int32 or NULL: iterations | (syndrome_failed << 16)
 * The reference return value of frame f is (max_iter == 0) ? 0 : status>>16. */
WLDPC_API int wldpc_decode_batch_device(wldpc_decoder* dec, const float* llr, int8_t* decoded, float* posterior,
                              int32_t* status, size_t frames, void* stream);

/* Batched decode of host buffers (pinned or pageable), synchronous, with the
 * host<->device copies pipelined against the kernels. rx_codewords is
 * overwritten with the posterior (reference semantics); num_errors and
 * status are nullable (frames entries each). */
WLDPC_API int wldpc_decode_batch_host(wldpc_decoder* dec, float* rx_codewords, int8_t* decoded, uint32_t* num_errors,
                            int32_t* status, size_t frames);
/* As wldpc_decode_batch_host without the posterior: llr is read only and
 * only the hard decisions (and num_errors / status, nullable) come back, the
 * outputs that BER_runner (reference lib/BER_runner.cc:194-199) and
 * test_decoder (reference lib/decode_example.cc:128-148) use. It moves n
 * bytes per frame back to the host instead of 5n. Synchronous. */
WLDPC_API int wldpc_decode_batch_host_hard(wldpc_decoder* dec, const float* llr, int8_t* decoded,
                                           uint32_t* num_errors, int32_t* status, size_t frames);

/* Batch form of decode(int8_t*, int8_t*) over host buffers (frames x n bytes
 * in and out; num_errors nullable), as the reference's test_decoder drives it
 * (reference lib/decode_example.cc:128-135). Synchronous. */
WLDPC_API int wldpc_decode_bits_batch_host(wldpc_decoder* dec, const int8_t* bits, int8_t* decoded,
                                           uint32_t* num_errors, size_t frames);
/* Batch form of compute_syndrome(int8_t*, bool) over host buffers. */
WLDPC_API int wldpc_syndrome_batch_host(wldpc_decoder* dec, const int8_t* bits, int exit_early, uint32_t* counts,
                                        size_t frames);

/* Waits for the device and reports a device-side error (WLDPC_ERR_TIMEOUT)
 * recorded by earlier launches of this decoder. */
WLDPC_API int wldpc_decoder_synchronize(wldpc_decoder* dec);

/* No counterpart in the reference (it has no device waits): a test hook that
 * sets how long (device time, microseconds) the decode kernel waits for the
 * barrier of its frame staging copy before giving up (default
 * WLDPC_WAIT_LIMIT_DEFAULT_US, one second). With 0 every launch gives up at
 * once: it records a timeout, waits (with the default bound) for its copy
 * to land and exits, and the next synchronising call returns
 * WLDPC_ERR_TIMEOUT with the context intact. Outputs of such a launch are
 * undefined. */
#define WLDPC_WAIT_LIMIT_DEFAULT_US 1000000u
WLDPC_API int wldpc_decoder_set_wait_limit(wldpc_decoder* dec, unsigned limit_us);
/* No counterpart in the reference: measures the kernels' wait bound. One GPU
 * thread runs the bounded wait with limit limit_us (at most ten times the
 * default) on an mbarrier phase that never completes, and *elapsed_ns
 * receives the device time until it gave up. Synchronous, default stream. */
WLDPC_API int wldpc_wait_bound_ns(unsigned limit_us, uint64_t* elapsed_ns);

/* ---------------------------------------------------------------- encoder */

typedef struct wldpc_encoder wldpc_encoder;

/* Replaces ldpc_encoder::ldpc_encoder(rate, z, num_threads) (reference
 * include/ldpc_encoder.h:21, lib/ldpc_encoder.cc:9-17). Like the reference
 * class, rate 3/4B is accepted; its output is whatever the dual-diagonal
 * recursion yields (the reference's tools refuse 3/4B, README.md:25). */
WLDPC_API int wldpc_encoder_create(int rate, unsigned z, unsigned num_threads, wldpc_encoder** out);
WLDPC_API int wldpc_encoder_destroy(wldpc_encoder* enc);

/* Replaces void ldpc_encoder::encode_data(uint8_t* infoword, uint8_t* codeword)
 * (reference include/ldpc_encoder.h:24, lib/ldpc_encoder.cc:50-105): k input
 * bytes (non-zero = 1), n output bytes, systematic part copied verbatim. */
WLDPC_API int wldpc_encoder_encode(wldpc_encoder* enc, const uint8_t* infoword, uint8_t* codeword);

/* Batched encode of host buffers (frames x k in, frames x n out). Synchronous. */
WLDPC_API int wldpc_encode_batch_host(wldpc_encoder* enc, const uint8_t* info, uint8_t* codeword, size_t frames);

/* Batched encode on device memory (frames x k in, frames x n out, both
 * 4-byte aligned), asynchronous on stream (NULL = the CUDA default stream). */
WLDPC_API int wldpc_encode_batch_device(wldpc_encoder* enc, const uint8_t* info, uint8_t* codeword, size_t frames,
                              void* stream);

/* --------------------------------------------------------- frame generator */

/* Seeded synthetic frames on device (the GPU stand-in for BER_runner's frame
 * generation, reference lib/BER_runner.cc:162-191): info bits from Philox4x32-10
 * (key = seed, counter = (block, frame, stream)), the encoder above, BPSK
 * bit*2-1, AWGN with sigma^2 = 1/(2 R Eb/N0), LLR = 2y/sigma^2 (positive = 1).
 * Eb/N0 in dB is drawn per frame uniformly in [ebno_lo_db, ebno_hi_db].
 * first_frame offsets the frame counter so that shards of one job draw
 * disjoint frames. Any of info (frames x k), codeword (frames x n), llr
 * (frames x n, 16-byte aligned) and ebno_db (frames) may be NULL. Rate 3/4B
 * has no encoder and returns WLDPC_ERR_UNSUPPORTED. Asynchronous on stream. */
WLDPC_API int wldpc_framegen_device(int rate, unsigned z, uint64_t seed, uint64_t first_frame, size_t frames,
                          float ebno_lo_db, float ebno_hi_db, uint8_t* info, uint8_t* codeword, float* llr,
                          float* ebno_db, void* stream);

/* ----------------------------------------------------- learned min-sum */

/* The learned (neural) normalized/offset min-sum decoder. It generalises the
 * reference's compile-time NMS/OMS constants (reference
 * lib/ldpc_decoder.cc:17-21,220-231) to a scale a and an offset b per
 * (iteration, layer, base column): message = s * max(a*min - b, 0), fp32,
 * same layered schedule and stopping rule, at most 8 iterations. Weights are
 * trained on the GPU by the library's own forward/backward kernels and Adam.
 * Weight tables are float[2][T][12][24]: a then b, [iteration][layer][column];
 * entries of all-zero blocks are ignored (returned as 0). Supported codes:
 * all 114 (every rate, z = 24..96 step 4); a table trained at one z applies
 * to every z of its rate, since it is indexed by base column. 3/4B trains on
 * null-space codewords. A new handle starts at a = 0.815, b = 0. */
typedef struct wldpc_lms wldpc_lms;
WLDPC_API int wldpc_lms_create(int rate, unsigned z, unsigned iterations, wldpc_lms** out);
WLDPC_API int wldpc_lms_destroy(wldpc_lms* h);
WLDPC_API int wldpc_lms_set_weights(wldpc_lms* h, const float* table);
WLDPC_API int wldpc_lms_get_weights(wldpc_lms* h, float* table);
/* Iteration cap of decoding (default: the trained iterations T); iterations
 * past T use the weights of iteration T-1. */
WLDPC_API int wldpc_lms_set_cap(wldpc_lms* h, unsigned cap);
/* Inference arithmetic of the learned decoder (no counterpart in the
 * reference, whose decoder has fixed constants). WLDPC_LMS_F32, the default,
 * decodes in fp32. WLDPC_LMS_F16X2 decodes two frames per thread in packed
 * IEEE binary16, about half the instructions per frame: every operation
 * rounds to binary16, input LLRs are clamped to +-2048 and row minima to
 * 2048, weights are rounded to binary16, and the posteriors returned are the
 * exact float values of the binary16 results. A frame's outputs do not depend
 * on the other frames of the batch. F16X2 needs |a| <= 2 and 0 <= b <= 1024
 * for every weight (finite sums; zero messages for a stopped frame whose
 * partner decodes on); otherwise this call, or a
 * decode after training moved a weight out of range, returns WLDPC_ERR_ARG.
 * Training always runs in fp32. */
#define WLDPC_LMS_F32 0
#define WLDPC_LMS_F16X2 1
WLDPC_API int wldpc_lms_set_precision(wldpc_lms* h, int precision);
/* Decode on device buffers (layout and status as wldpc_decode_batch_device). */
WLDPC_API int wldpc_lms_decode_device(wldpc_lms* h, const float* llr, int8_t* decoded, float* posterior,
                                      int32_t* status, size_t frames, void* stream);
/* Decode host buffers (posterior written back; num_errors = syndrome failed). */
WLDPC_API int wldpc_lms_decode_host(wldpc_lms* h, float* rx_codewords, int8_t* decoded, uint32_t* num_errors,
                                    int32_t* status, size_t frames);
/* The same without the posterior (llr read only; hard decisions, num_errors
 * and status back), as wldpc_decode_batch_host_hard. */
WLDPC_API int wldpc_lms_decode_host_hard(wldpc_lms* h, const float* llr, int8_t* decoded, uint32_t* num_errors,
                                         int32_t* status, size_t frames);
/* Training loss (mean BCE over iterations, bits and frames; positive LLR =
 * bit 1) and its gradient table for host frames (llr, transmitted codeword
 * bits 0/1). Synchronous. */
WLDPC_API int wldpc_lms_loss_grad(wldpc_lms* h, const float* llr, const uint8_t* codeword, size_t frames,
                                  float* grad_table, double* loss);
/* `steps` Adam steps (lr, beta 0.9 / 0.999) on batches of `batch` frames
 * generated on the device (wldpc_framegen_device, or
 * wldpc_framegen_nullspace_device for 3/4B; Eb/N0 uniform in
 * [ebno_lo_db, ebno_hi_db], frame counter first_frame + step * batch).
 * loss_history (nullable) receives the batch loss of every step. */
WLDPC_API int wldpc_lms_train(wldpc_lms* h, unsigned steps, unsigned batch, float ebno_lo_db, float ebno_hi_db,
                              uint64_t seed, uint64_t first_frame, float lr, float* loss_history);
/* One training step split in two, for data-parallel training over several
 * GPUs (no counterpart in the reference): wldpc_lms_step_grad generates
 * `batch` frames from counter first_frame as wldpc_lms_train does, runs the
 * forward and backward passes and writes the batch's gradient (float[nw] on
 * the device, compact [2][T][blocks] layout, nw from wldpc_lms_grad_size)
 * and its loss (float on the device, nullable) without changing the weights;
 * wldpc_lms_apply_grad applies one Adam step (as wldpc_lms_train) with a
 * given device gradient, e.g. the mean of the ranks' gradients after an
 * all-reduce. Both start after the work queued on `stream` and return when
 * their results are complete. Calls on one handle must not overlap. */
WLDPC_API int wldpc_lms_grad_size(wldpc_lms* h, size_t* nw);
WLDPC_API int wldpc_lms_step_grad(wldpc_lms* h, unsigned batch, float ebno_lo_db, float ebno_hi_db, uint64_t seed,
                                  uint64_t first_frame, float* grad, float* loss, void* stream);
WLDPC_API int wldpc_lms_apply_grad(wldpc_lms* h, const float* grad, float lr, void* stream);

/* ------------------------------------------------- allocation-free decode */

/* Size of the static device scratch used by wldpc_decode_host_noalloc. */
#define WLDPC_NOALLOC_SCRATCH_BYTES (1u << 20)

/* No counterpart in the reference: an allocation-free form of the batched
 * host decode, for callers that cannot call cudaMalloc -- hosts whose device
 * memory is owned by another allocator, real-time threads where an
 * allocation's device synchronisation is not allowed, and calls that cannot
 * keep a decoder handle alive. It creates no handle and allocates nothing:
 * its device scratch is a static 1 MiB array (held by every GPU that loads
 * the library until the process exits). Semantics are those of
 * wldpc_decode_batch_host with WLDPC_MODE_NMS: rx_codewords (frames x n host
 * floats) receives the posterior, decoded the hard bits, num_errors (nullable)
 * the per-frame reference return values. The staging must fit the scratch
 * (about 5n bytes per frame: at most 90 frames at z=96, 363 at z=24); larger requests
 * return WLDPC_ERR_SCRATCH. Every call looks up the scratch's device address
 * (which allocates nothing), so a device reset between calls is harmless; the
 * first call on a device also loads the module there and should come before
 * any stream capture. All calls share the scratch: calls that overlap on the
 * GPU race and must be serialised. Runs on the default stream and returns
 * when the results are in host memory; on a CUDA error it first waits for the
 * copies it queued. */
WLDPC_API int wldpc_decode_host_noalloc(int rate, unsigned z, unsigned max_iter, float* rx_codewords,
                                        int8_t* decoded, uint32_t* num_errors, size_t frames);

/* Replaces BER_runner's info-bit source (reference lib/BER_runner.cc:124-146:
 * LFSR x^31 + x^28 + 1 from 0xdeadbeef, restarted every 115200 bits) on the
 * device: out[j] = bit first_bit + j of that stream (0/1 bytes). A
 * BER_runner's frame f uses bits [f*k, (f+1)*k). Asynchronous on stream. */
WLDPC_API int wldpc_lfsr_bits_device(uint64_t first_bit, size_t nbits, uint8_t* out, void* stream);

/* Seeded random codewords of any code, 3/4B included (which has no
 * dual-diagonal encoder): uniform over the null space of H (free bits from
 * Philox stream 0 of (seed, frame), pivot bits from the reduced row-echelon
 * form computed once per (rate, z) on the host), then the same BPSK / AWGN /
 * LLR model as wldpc_framegen_device. codeword (frames x n) and llr
 * (frames x n, 16-byte aligned) and ebno_db may be NULL. Asynchronous. */
WLDPC_API int wldpc_framegen_nullspace_device(int rate, unsigned z, uint64_t seed, uint64_t first_frame,
                                              size_t frames, float ebno_lo_db, float ebno_hi_db, uint8_t* codeword,
                                              float* llr, float* ebno_db, void* stream);

/* --------------------------------------------- mixed-code persistent decode */

/* Code index used by the mixed decoder: rate * 19 + (z - 24) / 4, or
 * WLDPC_ERR_CODE. */
WLDPC_API int wldpc_variant(int rate, unsigned z);

/* A batch whose frames use different codes (any rate, any z), decoded by one
 * persistent launch: frames are binned by code on the device, CTAs take work
 * items (up to `chunk` frames of one code) from a queue and refill a frame
 * slot as soon as its frame stops (early-exit compaction). Arithmetic, outputs
 * and status are those of wldpc_decode_batch_device with WLDPC_MODE_NMS
 * (bit-exact with the reference). The binning and decode launches are
 * captured in a CUDA graph on the first call and replayed by later calls with
 * the same pointers, frame count and configuration. No counterpart in the
 * reference, whose decoder object handles one code. */
typedef struct wldpc_mixed wldpc_mixed;
WLDPC_API int wldpc_mixed_create(unsigned max_iter, wldpc_mixed** out);
WLDPC_API int wldpc_mixed_destroy(wldpc_mixed* h);
/* variant[f]: code of frame f; offset[f]: element offset of frame f's n values
 * in llr / decoded / posterior (frames may be in any order), a multiple of 4
 * so that every frame starts 16-byte aligned (frames of n = 24z values packed
 * back to back satisfy it); llr and posterior 16-byte aligned, decoded 4.
 * Asynchronous on stream (ordered with it through events). */
WLDPC_API int wldpc_mixed_decode_device(wldpc_mixed* h, const uint8_t* variant, const int64_t* offset,
                                        const float* llr, int8_t* decoded, float* posterior, int32_t* status,
                                        size_t frames, void* stream);
/* Waits for the handle's work; WLDPC_ERR_ARG if a frame had an invalid code
 * or an offset that is not a multiple of 4 (such frames are not decoded). */
WLDPC_API int wldpc_mixed_synchronize(wldpc_mixed* h);
/* The autotuner's knobs: CTA size (96 or 192 threads), expanded rows per
 * thread (1 or 2, i.e. z or z/2 threads per frame: the frame slots per CTA
 * are threads * rows / z), where each thread's compressed messages live
 * (registers, or shared memory: fewer registers and more resident CTAs),
 * frames per work item (1..64) and whether the six per-rate grids run
 * concurrently or one after another. set_tuning and set_config leave the
 * rows per thread as they are; set_config / get_config also leave layout and
 * launch policy. */
#define WLDPC_MIXED_MSG_REGISTERS 0
#define WLDPC_MIXED_MSG_SHARED 1
#define WLDPC_MIXED_CONCURRENT 0
#define WLDPC_MIXED_SERIAL 1
WLDPC_API int wldpc_mixed_set_tuning(wldpc_mixed* h, int threads, int layout, int chunk, int launch);
WLDPC_API int wldpc_mixed_get_tuning(wldpc_mixed* h, int* threads, int* layout, int* chunk, int* launch);
WLDPC_API int wldpc_mixed_set_config(wldpc_mixed* h, int threads, int chunk);
WLDPC_API int wldpc_mixed_get_config(wldpc_mixed* h, int* threads, int* chunk);
/* rows = 1 or 2 expanded rows per thread (WLDPC_ERR_ARG otherwise) */
WLDPC_API int wldpc_mixed_set_rows_per_thread(wldpc_mixed* h, int rows);
WLDPC_API int wldpc_mixed_get_rows_per_thread(wldpc_mixed* h, int* rows);
/* Times every (threads, rows per thread, layout, chunk, launch) candidate on
 * the given batch (repeats launches each) and keeps the fastest; *best_ms
 * (nullable) gets its time. */
WLDPC_API int wldpc_mixed_autotune(wldpc_mixed* h, const uint8_t* variant, const int64_t* offset, const float* llr,
                                   int8_t* decoded, size_t frames, int repeats, float* best_ms);

/* ------------------------------------------------------------- BER runner */

typedef struct wldpc_ber_runner wldpc_ber_runner;

/* Replaces BER_runner::BER_runner(rate, z, num_threads, max_iter) (reference
 * include/BER_runner.h:53-57, lib/BER_runner.cc:15-87): 3/4B returns
 * WLDPC_ERR_UNSUPPORTED where the reference throws. */
WLDPC_API int wldpc_ber_runner_create(int rate, unsigned z, unsigned num_threads, unsigned max_iter,
                            wldpc_ber_runner** out);
WLDPC_API int wldpc_ber_runner_destroy(wldpc_ber_runner* b);
/* Replaces double BER_runner::run_iteration(double EbNo_dB) (reference
 * lib/BER_runner.cc:162-204): one frame with the reference's LFSR info bits,
 * mt19937(0) / normal_distribution<float> noise stream and error count (over
 * all n codeword bits, k added to the bit count); encode and decode run on
 * the GPU. *ber gets the running errors / bits. */
WLDPC_API int wldpc_ber_runner_run_iteration(wldpc_ber_runner* b, double ebno_db, double* ber);
/* Replaces BER_runner::reset_test (reference lib/BER_runner.cc:96-102). */
WLDPC_API int wldpc_ber_runner_reset(wldpc_ber_runner* b);
/* Replaces get_total_num_bits / get_total_num_errors (reference :104-112). */
WLDPC_API int wldpc_ber_runner_totals(wldpc_ber_runner* b, uint64_t* num_bits, uint64_t* num_errors);
/* Replaces get_codeword_len / get_dataword_len (reference :114-122). */
WLDPC_API int wldpc_ber_runner_lengths(wldpc_ber_runner* b, unsigned* codeword_len, unsigned* dataword_len);

#ifdef __cplusplus
}
#endif

#endif
