/*
 * wldpc_oracle: CPU restatement of the reference's WiMAX QC-LDPC codec path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only as the checker. The
 * product library (wimax_ldpc_lib_b200) never links, loads or falls back to it.
 *
 * Pinning: every function here is checked against the reference itself
 * (compiled from its own sources into oracle/_ref by oracle/Makefile) and
 * against golden fixtures generated from it (tests/golden/make_golden.py).
 * The reference ships no tests, known-answer files or golden vectors of its
 * own, so those fixtures are the reference's outputs recorded here.
 *
 * Conventions (reference): positive LLR means bit 1 (BPSK bit*2-1,
 * reference lib/BER_runner.cc:183); the slicer gives 1 for x >= 0 (VOLK
 * volk_32f_binary_slicer_8i at reference lib/ldpc_decoder.cc:130,242).
 * Inputs must be finite: the reference is built with -ffast-math, which
 * assumes no NaN or infinity (reference lib/CMakeLists.txt:6).
 */
#ifndef WLDPC_ORACLE_H
#define WLDPC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WO_MAX_BLOCKS 96
#define WO_NB 24

typedef struct {
    int rate, z;
    int mb, kb;            /* base rows (layers), info block columns */
    int n, m, k;           /* codeword, parity, info bits */
    int D, X;              /* encoder constants (reference include/ldpc.h:43,46) */
    int nblk;              /* non-zero circulant blocks */
    int row_start[13];     /* blocks of base row i: [row_start[i], row_start[i+1]) */
    int blk_col[WO_MAX_BLOCKS];
    int blk_shift[WO_MAX_BLOCKS];
    int max_deg;
} wo_code_t;

enum { WO_NMS = 0, WO_OMS = 1, WO_MS = 2 };

int wo_code(int rate, int z, wo_code_t* c);
/* Expanded check-node table in the reference's layout: int16 [rows][cols],
 * -1 padded (reference lib/matrices/wimax_N_RATE.cc). */
int wo_checknode_table(int rate, int z, int16_t* out, long capacity, int* rows, int* cols);

/* Plain TDMP decoder (reference lib/ldpc_decoder.cc:122-262). llr is updated
 * in place with the posterior. Per frame: ret = reference return value,
 * iters = iterations executed (0 when the sliced input already satisfies the
 * syndrome), synfail = 1 when the final syndrome is not zero. Any of ret,
 * iters, synfail may be NULL. */
int wo_decode_batch(int rate, int z, int max_iter, int mode, long frames, float* llr,
                    int8_t* decoded, uint32_t* ret, int32_t* iters, int32_t* synfail,
                    int threads);
/* Hard-bit input adapter (reference lib/ldpc_decoder.cc:108-118). */
int wo_decode_bits_batch(int rate, int z, int max_iter, long frames, const int8_t* bits,
                         int8_t* decoded, uint32_t* ret, int32_t* iters, int threads);
/* compute_syndrome (reference lib/ldpc_decoder.cc:67-104). */
int wo_syndrome_batch(int rate, int z, long frames, const int8_t* bits, int early_exit,
                      uint32_t* ret);
/* Dual-diagonal encoder (reference lib/ldpc_encoder.cc:29-105). */
int wo_encode_batch(int rate, int z, long frames, const uint8_t* info, uint8_t* cw,
                    int threads);

/* BER_runner info-bit LFSR, x^31 + x^28 + 1, seed 0xdeadbeef, restarted every
 * reset_len bits (reference lib/BER_runner.cc:35-41,124-146). Fills nbits
 * bytes of 0/1 and returns the state through *state / *index. */
void wo_lfsr_fill(uint32_t* state, uint32_t* index, uint32_t start_state,
                  uint32_t reset_len, uint8_t* out, long nbits);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), one block. */
void wo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Synthetic frame generation (the project's own on-device generator,
 * restated in double precision): info bits from Philox stream 0, encoder,
 * BPSK bit*2-1, AWGN from Philox stream 1 by Box-Muller, LLR = 2y/sigma^2 with
 * sigma^2 = 1/(2 R Eb/N0). Eb/N0 per frame is ebno_lo + (ebno_hi-ebno_lo)*u,
 * u from Philox stream 2. Frame f uses global index first_frame + f. */
int wo_framegen(int rate, int z, uint64_t seed, uint64_t first_frame, long frames,
                double ebno_lo_db, double ebno_hi_db, uint8_t* info, uint8_t* cw,
                double* llr, double* ebno_db);

/* Learned min-sum, float inference: decoder with per-(iteration, layer,
 * block column) scale a and offset b, message = s * max(a*mu - b, 0)
 * (fmaf), min tracking from +inf, early exit on syndrome, at most cap
 * iterations (iterations past `iterations` use the last row of weights).
 * w has 2*iterations*12*24 floats: a then b, each [iteration][layer][col]. */
int wo_learned_decode_batch(int rate, int z, int iterations, int cap, const float* w, long frames,
                            float* llr, int8_t* decoded, int32_t* iters, int32_t* synfail,
                            int threads);
/* Learned min-sum in binary16, as the packed-half decoder computes it (one
 * frame at a time; the device's lanes are independent): LLRs clamped to
 * +-2048 and rounded to binary16 (-0 made +0), weights rounded to binary16,
 * every difference, sum and fused multiply-add rounded once to binary16
 * (nearest even), row minima clamped to 2048; post receives the posteriors
 * (binary16 values as floats); llr is not modified. */
int wo_learned16_decode_batch(int rate, int z, int iterations, int cap, const float* w, long frames,
                              const float* llr, float* post, int8_t* decoded, int32_t* iters, int32_t* synfail,
                              int threads);
/* x rounded to the nearest binary16 value (ties to even, overflow to inf),
 * and relu of a*b + c rounded once to binary16. */
double wo_half_round(double x);
double wo_half_fma_relu(double a, double b, double c);
/* Learned min-sum training step reference in double precision: loss
 * (mean BCE over iterations, frames and bits, positive LLR = bit 1) and its
 * gradient with respect to w (same layout as above). */
double wo_learned_loss_grad(int rate, int z, int iterations, const float* w, long frames,
                            const float* llr, const uint8_t* cw, double* grad);

#ifdef __cplusplus
}
#endif
#endif
