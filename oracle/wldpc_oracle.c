/*
 * wldpc_oracle.c -- CPU restatement of the reference codec path.
 *
 * TEST INFRASTRUCTURE ONLY (see wldpc_oracle.h). Built by oracle/Makefile
 * with -ffp-contract=off so that every float / double operation rounds
 * exactly as written (no FMA contraction), which is what the reference's x86
 * build does (no FMA without -march flags, reference lib/CMakeLists.txt:6).
 */
#define _GNU_SOURCE
#include "wldpc_oracle.h"
#include "base_matrices.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

/* ------------------------------------------------------------------ codes */

static int shift_rule(int rate, int p, int z)
{
    if (p <= 0) return p;
    if (rate == 1) return p % z;          /* 2/3A */
    return (p * z) / 96;                  /* floor(p*z/96) */
}

int wo_code(int rate, int z, wo_code_t* c)
{
    if (rate < 0 || rate > 5) return -1;
    if (z < 24 || z > 96 || (z % 4) != 0) return -1;
    memset(c, 0, sizeof(*c));
    c->rate = rate;
    c->z = z;
    c->mb = wo_base_mb[rate];
    c->kb = WO_NB - c->mb;
    c->n = WO_NB * z;
    c->m = c->mb * z;
    c->k = c->n - c->m;
    c->D = shift_rule(rate, wo_base_D96[rate], z);
    c->X = wo_base_X[rate];
    int b = 0;
    for (int i = 0; i < c->mb; i++) {
        c->row_start[i] = b;
        for (int j = 0; j < WO_NB; j++) {
            int p = wo_base[rate][i][j];
            if (p < 0) continue;
            c->blk_col[b] = j;
            c->blk_shift[b] = shift_rule(rate, p, z);
            b++;
        }
        int d = b - c->row_start[i];
        if (d > c->max_deg) c->max_deg = d;
    }
    c->row_start[c->mb] = b;
    c->nblk = b;
    return 0;
}

static inline int var_of(const wo_code_t* c, int blk, int r)
{
    int t = r + c->blk_shift[blk];
    if (t >= c->z) t -= c->z;
    return c->blk_col[blk] * c->z + t;
}

int wo_checknode_table(int rate, int z, int16_t* out, long capacity, int* rows, int* cols)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    *rows = c.m;
    *cols = c.max_deg;
    if ((long)c.m * c.max_deg > capacity) return -2;
    for (int i = 0; i < c.mb; i++)
        for (int r = 0; r < z; r++) {
            int16_t* row = out + (long)(i * z + r) * c.max_deg;
            int e = 0;
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) row[e++] = (int16_t)var_of(&c, b, r);
            for (; e < c.max_deg; e++) row[e] = -1;
        }
    return 0;
}

/* --------------------------------------------------------------- syndrome */

/* Row parity as a byte XOR (the reference XORs int8 values, so non 0/1
 * inputs are folded exactly as it does, reference lib/ldpc_decoder.cc:73-83). */
static unsigned syndrome_one(const wo_code_t* c, const int8_t* bits, int early_exit)
{
    unsigned fails = 0;
    for (int i = 0; i < c->mb; i++)
        for (int r = 0; r < c->z; r++) {
            int8_t x = 0;
            for (int b = c->row_start[i]; b < c->row_start[i + 1]; b++) x ^= bits[var_of(c, b, r)];
            if (x != 0) {
                if (early_exit) return 1;
                fails++;
            }
        }
    return fails;
}

int wo_syndrome_batch(int rate, int z, long frames, const int8_t* bits, int early_exit,
                      uint32_t* ret)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    for (long f = 0; f < frames; f++) ret[f] = syndrome_one(&c, bits + f * c.n, early_exit);
    return 0;
}

static void slice(const float* x, int8_t* out, int n)
{
    for (int i = 0; i < n; i++) out[i] = (x[i] >= 0.0f) ? 1 : 0;
}

/* ---------------------------------------------------------- TDMP decoder */

/* Sign test of the check-node update. The reference writes
 * std::signbit(LNM) (reference lib/ldpc_decoder.cc:172,191), but its release
 * build uses -ffast-math (reference lib/CMakeLists.txt:6), under which GCC
 * evaluates signbit(x) as x < 0: -0.0 counts as non-negative. Pinned against
 * the reference compiled with its own flags on inputs with exact +-0 LLRs
 * (tests/golden: the "zeros" edge case). The restatement follows the
 * reference as built: negative means x < 0. */

/* One frame of the layered decoder. msg holds one float per edge
 * (block-major: edge = block*z + r); it is cleared here, which is what the
 * reference's zeroed slice 0 of m_LMN provides (reference
 * lib/ldpc_decoder.cc:36-38,162). */
static unsigned decode_one(const wo_code_t* c, int max_iter, int mode, float* rx,
                           int8_t* out, float* msg, int32_t* iters, int32_t* synfail)
{
    const int z = c->z;
    slice(rx, out, c->n);
    if (syndrome_one(c, out, 1) == 0) {          /* reference :130-139 */
        if (iters) *iters = 0;
        if (synfail) *synfail = 0;
        return 0;
    }
    memset(msg, 0, sizeof(float) * (size_t)c->nblk * z);
    unsigned num_errors = 0;
    for (int it = 1; it <= max_iter; it++) {      /* reference :141 */
        for (int i = 0; i < c->mb; i++) {          /* layer = base row */
            const int b0 = c->row_start[i], d = c->row_start[i + 1] - b0;
            for (int r = 0; r < z; r++) {          /* the z rows touch disjoint variables */
                float L[WO_NB];
                int v[WO_NB];
                int parity = 1;                    /* reference :148 (sign = true) */
                float m1 = 10000.0f;               /* reference :150 */
                int am = 0;
                for (int e = 0; e < d; e++) {      /* pass 1, reference :164-182 */
                    v[e] = var_of(c, b0 + e, r);
                    L[e] = rx[v[e]] - msg[(b0 + e) * z + r];
                    parity ^= !(L[e] < 0.0f);      /* see ref_negative() */
                    float a = fabsf(L[e]);
                    if (a < m1) { m1 = a; am = e; }
                }
                for (int e = 0; e < d; e++) {      /* pass 2, reference :188-239 */
                    float sgn = (float)((parity ^ !(L[e] < 0.0f)) * -2 + 1);
                    float mn;
                    if (e == am) {
                        mn = 10000.0f;
                        for (int q = 0; q < d; q++)
                            if (q != am) { float a = fabsf(L[q]); if (a < mn) mn = a; }
                    } else {
                        mn = m1;
                    }
                    float* pm = &msg[(b0 + e) * z + r];
                    if (mode == WO_NMS) {          /* fp64 normalization, reference :17-18,220-223 */
                        double t = (double)sgn * ((double)mn * 0.815);
                        *pm = (float)t;
                        rx[v[e]] = (float)((double)L[e] + t);
                    } else if (mode == WO_OMS) {   /* reference :21,227-231 (std::max) */
                        double a = (double)mn - 0.10;
                        double mx = (a < 0.0) ? 0.0 : a;
                        double t = (double)sgn * mx;
                        *pm = (float)t;
                        rx[v[e]] = (float)((double)L[e] + t);
                    } else {                       /* plain min-sum, reference :236-237 */
                        float t = sgn * mn;
                        *pm = t;
                        rx[v[e]] = L[e] + t;
                    }
                }
            }
        }
        slice(rx, out, c->n);                      /* reference :242-251 */
        num_errors = syndrome_one(c, out, 1);
        if (num_errors == 0) {
            if (iters) *iters = it;
            if (synfail) *synfail = 0;
            return 0;
        }
    }
    if (iters) *iters = max_iter;
    if (synfail) *synfail = 1;
    return num_errors;                             /* 0 when max_iter == 0 (reference :124,261) */
}

int wo_decode_batch(int rate, int z, int max_iter, int mode, long frames, float* llr,
                    int8_t* decoded, uint32_t* ret, int32_t* iters, int32_t* synfail,
                    int threads)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    if (max_iter < 0 || mode < 0 || mode > 2) return -1;
    if (threads < 1) threads = 1;
    #pragma omp parallel num_threads(threads)
    {
        float* msg = (float*)malloc(sizeof(float) * (size_t)c.nblk * z);
        #pragma omp for schedule(dynamic, 16)
        for (long f = 0; f < frames; f++) {
            unsigned r = decode_one(&c, max_iter, mode, llr + f * c.n, decoded + f * c.n, msg,
                                    iters ? iters + f : NULL, synfail ? synfail + f : NULL);
            if (ret) ret[f] = r;
        }
        free(msg);
    }
    return 0;
}

int wo_decode_bits_batch(int rate, int z, int max_iter, long frames, const int8_t* bits,
                         int8_t* decoded, uint32_t* ret, int32_t* iters, int threads)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    float* soft = (float*)malloc(sizeof(float) * (size_t)frames * c.n);
    for (long i = 0; i < frames * (long)c.n; i++) soft[i] = (float)(bits[i] * 2.0 - 1.0);
    int rc = wo_decode_batch(rate, z, max_iter, WO_NMS, frames, soft, decoded, ret, iters, NULL, threads);
    free(soft);
    return rc;
}

/* ---------------------------------------------------------------- encoder */

/* Block form of the dual-diagonal recursion of the reference encoder
 * (reference lib/ldpc_encoder.cc:50-105): with V_b the z-bit block b of
 * V = H_info * u, P_{mb-1} = V_{mb-1}; P_b = P_{b-1} ^ V_{b-1} for b = 1..X
 * (starting from zero); P_b = V_b ^ P_{b+1} for b = mb-2 down to X+1;
 * P_0 = V_X ^ P_{X+1} ^ P_X; parity block 0 is P_0 and parity block b >= 1,
 * lane r, is P_b[r] ^ P_0[(r + D) mod z]. */
static void encode_one(const wo_code_t* c, const uint8_t* info, uint8_t* cw)
{
    const int z = c->z, mb = c->mb;
    uint8_t V[12 * 96], P[12 * 96];
    memset(V, 0, sizeof(V));
    memset(P, 0, sizeof(P));
    for (int i = 0; i < mb; i++)
        for (int r = 0; r < z; r++) {
            uint8_t x = 0;
            for (int b = c->row_start[i]; b < c->row_start[i + 1]; b++) {
                if (c->blk_col[b] >= c->kb) continue;   /* info columns only (reference :41) */
                x ^= (info[var_of(c, b, r)] != 0);       /* booleanized (reference :43) */
            }
            V[i * z + r] = x;
        }
    for (int r = 0; r < z; r++) P[(mb - 1) * z + r] = V[(mb - 1) * z + r];
    for (int b = 1; b <= c->X; b++)
        for (int r = 0; r < z; r++) P[b * z + r] = P[(b - 1) * z + r] ^ V[(b - 1) * z + r];
    for (int b = mb - 2; b >= c->X + 1; b--)
        for (int r = 0; r < z; r++) P[b * z + r] = V[b * z + r] ^ P[(b + 1) * z + r];
    for (int r = 0; r < z; r++)
        P[r] = V[c->X * z + r] ^ P[(c->X + 1) * z + r] ^ P[c->X * z + r];
    memcpy(cw, info, (size_t)c->k);                     /* raw bytes (reference :90) */
    for (int r = 0; r < z; r++) cw[c->k + r] = P[r];
    for (int b = 1; b < mb; b++)
        for (int r = 0; r < z; r++) {
            int rr = r + c->D;
            while (rr >= z) rr -= z;
            cw[c->k + b * z + r] = P[b * z + r] ^ P[rr];
        }
}

int wo_encode_batch(int rate, int z, long frames, const uint8_t* info, uint8_t* cw, int threads)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    if (threads < 1) threads = 1;
    #pragma omp parallel for num_threads(threads) schedule(static)
    for (long f = 0; f < frames; f++) encode_one(&c, info + f * c.k, cw + f * c.n);
    return 0;
}

/* ------------------------------------------------------------------- LFSR */

void wo_lfsr_fill(uint32_t* state, uint32_t* index, uint32_t start_state, uint32_t reset_len,
                  uint8_t* out, long nbits)
{
    uint32_t s = *state, idx = *index;
    for (long i = 0; i < nbits; i++) {
        uint32_t bit = (s ^ (s >> 3)) & 1u;   /* taps for x^31 + x^28 + 1 */
        s = (s >> 1) | (bit << 30);
        if (++idx == reset_len) { s = start_state; idx = 0; }
        out[i] = (uint8_t)bit;
    }
    *state = s;
    *index = idx;
}

/* ----------------------------------------------------------------- Philox */

void wo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; round++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void philox_at(uint64_t seed, uint64_t frame, uint32_t word, uint32_t stream, uint32_t out[4])
{
    uint32_t ctr[4] = {word, (uint32_t)frame, (uint32_t)(frame >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    wo_philox4x32_10(ctr, key, out);
}

/* 24-bit uniform in (0, 1): ((x >> 8) + 0.5) * 2^-24, exact in float. */
static double unif24(uint32_t x) { return ((double)(x >> 8) + 0.5) * (1.0 / 16777216.0); }

static double code_rate(const wo_code_t* c) { return (double)c->k / (double)c->n; }

int wo_framegen(int rate, int z, uint64_t seed, uint64_t first_frame, long frames,
                double ebno_lo_db, double ebno_hi_db, uint8_t* info, uint8_t* cw,
                double* llr, double* ebno_out)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    uint8_t* u = (uint8_t*)malloc((size_t)c.k);
    uint8_t* x = (uint8_t*)malloc((size_t)c.n);
    for (long f = 0; f < frames; f++) {
        uint64_t g = first_frame + (uint64_t)f;
        for (int j = 0; j < c.k; j += 128) {
            uint32_t o[4];
            philox_at(seed, g, (uint32_t)(j / 128), 0, o);
            for (int q = 0; q < 128 && j + q < c.k; q++) u[j + q] = (o[q >> 5] >> (q & 31)) & 1u;
        }
        encode_one(&c, u, x);
        uint32_t eo[4];
        philox_at(seed, g, 0, 2, eo);
        /* Eb/N0 in float as the device computes it: lo + (hi - lo) * u */
        float ebno = (float)ebno_lo_db + ((float)ebno_hi_db - (float)ebno_lo_db) * (float)unif24(eo[0]);
        double ebno_lin = pow(10.0, (double)ebno / 10.0);
        double sigma2 = 1.0 / (2.0 * code_rate(&c) * ebno_lin);
        double sigma = sqrt(sigma2);
        double scale = 2.0 / sigma2;
        for (int j = 0; j < c.n; j += 4) {
            uint32_t o[4];
            philox_at(seed, g, (uint32_t)(j / 4), 1, o);
            double nrm[4];
            for (int p = 0; p < 2; p++) {
                double u1 = unif24(o[2 * p]), u2 = unif24(o[2 * p + 1]);
                double rad = sqrt(-2.0 * log(u1));
                nrm[2 * p] = rad * cos(2.0 * M_PI * u2);
                nrm[2 * p + 1] = rad * sin(2.0 * M_PI * u2);
            }
            for (int q = 0; q < 4 && j + q < c.n; q++) {
                double y = (x[j + q] ? 1.0 : -1.0) + sigma * nrm[q];
                if (llr) llr[f * c.n + j + q] = scale * y;
            }
        }
        if (info) memcpy(info + f * c.k, u, (size_t)c.k);
        if (cw) memcpy(cw + f * c.n, x, (size_t)c.n);
        if (ebno_out) ebno_out[f] = (double)ebno;
    }
    free(u);
    free(x);
    return 0;
}

/* ------------------------------------------------------- learned min-sum */

#define WO_L 12

static inline size_t widx(int t, int i, int col) { return ((size_t)t * WO_L + (size_t)i) * WO_NB + (size_t)col; }

static inline float flip_sign(float x, unsigned neg)
{
    union { float f; uint32_t u; } v;
    v.f = x;
    v.u ^= (neg & 1u) << 31;
    return v.f;
}

static unsigned learned_one(const wo_code_t* c, int T, int cap, const float* A, const float* B, float* rx,
                            int8_t* out, float* msg, int32_t* iters, int32_t* synfail)
{
    const int z = c->z;
    slice(rx, out, c->n);
    if (syndrome_one(c, out, 1) == 0) {
        if (iters) *iters = 0;
        if (synfail) *synfail = 0;
        return 0;
    }
    memset(msg, 0, sizeof(float) * (size_t)c->nblk * z);
    for (int it = 0; it < cap; it++) {
        const int t = it < T ? it : T - 1;     /* past T: the last trained iteration's weights */
        for (int i = 0; i < c->mb; i++) {
            const int b0 = c->row_start[i], d = c->row_start[i + 1] - b0;
            for (int r = 0; r < z; r++) {
                float L[WO_NB];
                int v[WO_NB];
                unsigned negpar = 0;
                float m1 = INFINITY, m2 = INFINITY;
                for (int e = 0; e < d; e++) {
                    v[e] = var_of(c, b0 + e, r);
                    L[e] = rx[v[e]] - msg[(b0 + e) * z + r];
                    negpar ^= (unsigned)(signbit(L[e]) != 0);
                    float a = fabsf(L[e]);
                    m2 = fminf(m2, fmaxf(m1, a));
                    m1 = fminf(m1, a);
                }
                for (int e = 0; e < d; e++) {
                    unsigned neg_e = (unsigned)(signbit(L[e]) != 0);
                    /* positive LLR = bit 1: the extrinsic sign flips on odd-degree rows */
                    unsigned negmsg = negpar ^ neg_e ^ (unsigned)(d & 1);
                    float mu = (fabsf(L[e]) == m1) ? m2 : m1;
                    int col = c->blk_col[b0 + e];
                    float mag = fmaf(A[widx(t, i, col)], mu, -B[widx(t, i, col)]);
                    mag = fmaxf(mag, 0.0f);
                    float m = flip_sign(mag, negmsg);
                    msg[(b0 + e) * z + r] = m;
                    rx[v[e]] = L[e] + m;
                }
            }
        }
        slice(rx, out, c->n);
        if (syndrome_one(c, out, 1) == 0) {
            if (iters) *iters = it + 1;
            if (synfail) *synfail = 0;
            return 0;
        }
    }
    if (iters) *iters = cap;
    if (synfail) *synfail = 1;
    return 1;
}

int wo_learned_decode_batch(int rate, int z, int iterations, int cap, const float* w, long frames,
                            float* llr, int8_t* decoded, int32_t* iters, int32_t* synfail,
                            int threads)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    if (iterations < 1 || iterations > 8 || cap < 0) return -1;
    const float* A = w;
    const float* B = w + (size_t)iterations * WO_L * WO_NB;
    if (threads < 1) threads = 1;
    #pragma omp parallel num_threads(threads)
    {
        float* msg = (float*)malloc(sizeof(float) * (size_t)c.nblk * z);
        #pragma omp for schedule(dynamic, 16)
        for (long f = 0; f < frames; f++)
            learned_one(&c, iterations, cap, A, B, llr + f * c.n, decoded + f * c.n, msg,
                        iters ? iters + f : NULL, synfail ? synfail + f : NULL);
        free(msg);
    }
    return 0;
}

/* ------------------------------------- learned min-sum in binary16 lanes */

/* Restates the packed-half learned decoder (wimax_ldpc_lib_b200/csrc/lms16.cuh)
 * one frame at a time: every value is a binary16 number held exactly in a
 * float, and every operation is computed exactly in double and rounded once
 * to binary16 (nearest, ties to even). Sums and differences of two binary16
 * numbers are exact in double; the fused multiply-add uses an exact TwoSum
 * so that its single rounding is exact too. */

static int half_quantum(double ax)            /* exponent of the binary16 ulp at |x| = ax > 0 */
{
    const int e = ilogb(ax);
    return e >= -14 ? e - 10 : -24;
}

double wo_half_round(double x)
{
    if (isnan(x) || x == 0.0) return x;
    const double ax = fabs(x);
    if (ax >= 65520.0) return copysign(INFINITY, x);   /* past the largest finite value's tie */
    const int q = half_quantum(ax);
    return copysign(ldexp(nearbyint(ldexp(ax, -q)), q), x);   /* default mode: ties to even */
}

double wo_half_fma_relu(double a, double b, double c)
{
    const double p = a * b;                   /* exact: two 11-bit significands */
    const double s = p + c;
    const double bb = s - p;
    const double err = (p - (s - bb)) + (c - bb);   /* s + err == p + c exactly */
    double r = wo_half_round(s);
    if (err != 0.0 && isfinite(s)) {
        /* only a value of s exactly on a binary16 tie can round the wrong way:
         * the exact sum lies past the tie on err's side */
        const double as = fabs(s);
        const int q = half_quantum(as < 65504.0 ? as : 65504.0);
        const double sc = ldexp(as, -q), fl = floor(sc);
        if (sc - fl == 0.5) {
            const double mag = ((err > 0) == (s > 0)) ? fl + 1.0 : fl;
            r = copysign(ldexp(mag, q), s);
            if (fabs(r) > 65504.0) r = copysign(INFINITY, s);
        }
    }
    return r < 0.0 ? 0.0 : r;
}

static unsigned learned16_one(const wo_code_t* c, int T, int cap, const float* Ah, const float* NBh,
                              const float* llr, float* P, int8_t* out, float* msg, int32_t* iters,
                              int32_t* synfail)
{
    const int z = c->z, n = c->n;
    for (int v = 0; v < n; v++) {
        const float x = fminf(fmaxf(llr[v], -2048.0f), 2048.0f);
        const double h = wo_half_round((double)x);
        P[v] = h == 0.0 ? 0.0f : (float)h;    /* -0 becomes +0 */
    }
    slice(P, out, n);
    if (syndrome_one(c, out, 1) == 0) {
        if (iters) *iters = 0;
        if (synfail) *synfail = 0;
        return 0;
    }
    memset(msg, 0, sizeof(float) * (size_t)c->nblk * z);
    for (int it = 0; it < cap; it++) {
        const int t = it < T ? it : T - 1;
        for (int i = 0; i < c->mb; i++) {
            const int b0 = c->row_start[i], d = c->row_start[i + 1] - b0;
            for (int r = 0; r < z; r++) {
                float L[WO_NB];
                int v[WO_NB];
                unsigned negpar = 0;
                float m1 = INFINITY, m2 = INFINITY;
                for (int e = 0; e < d; e++) {
                    v[e] = var_of(c, b0 + e, r);
                    L[e] = (float)wo_half_round((double)P[v[e]] - (double)msg[(b0 + e) * z + r]);
                    negpar ^= (unsigned)(signbit(L[e]) != 0);
                    const float a = fabsf(L[e]);
                    m2 = fminf(m2, fmaxf(m1, a));
                    m1 = fminf(m1, a);
                }
                m1 = fminf(m1, 2048.0f);
                m2 = fminf(m2, 2048.0f);
                for (int e = 0; e < d; e++) {
                    const unsigned neg = negpar ^ (unsigned)(signbit(L[e]) != 0) ^ (unsigned)(d & 1);
                    const float mu = (fabsf(L[e]) == m1) ? m2 : m1;
                    const size_t wi = widx(t, i, c->blk_col[b0 + e]);
                    const float mag = (float)wo_half_fma_relu((double)Ah[wi], (double)mu, (double)NBh[wi]);
                    const float m = flip_sign(mag, neg);
                    msg[(b0 + e) * z + r] = m;
                    P[v[e]] = (float)wo_half_round((double)L[e] + (double)m);
                }
            }
        }
        slice(P, out, n);
        if (syndrome_one(c, out, 1) == 0) {
            if (iters) *iters = it + 1;
            if (synfail) *synfail = 0;
            return 0;
        }
    }
    if (iters) *iters = cap;
    if (synfail) *synfail = 1;
    return 1;
}

int wo_learned16_decode_batch(int rate, int z, int iterations, int cap, const float* w, long frames,
                              const float* llr, float* post, int8_t* decoded, int32_t* iters, int32_t* synfail,
                              int threads)
{
    wo_code_t c;
    if (wo_code(rate, z, &c)) return -1;
    if (iterations < 1 || iterations > 8 || cap < 0) return -1;
    const size_t WN = (size_t)iterations * WO_L * WO_NB;
    float* Ah = (float*)malloc(sizeof(float) * 2 * WN);
    if (!Ah) return -1;
    float* NBh = Ah + WN;
    for (size_t j = 0; j < WN; j++) {
        Ah[j] = (float)wo_half_round((double)w[j]);
        NBh[j] = (float)wo_half_round(-(double)w[WN + j]);
    }
    if (threads < 1) threads = 1;
    #pragma omp parallel num_threads(threads)
    {
        float* msg = (float*)malloc(sizeof(float) * (size_t)c.nblk * z);
        #pragma omp for schedule(dynamic, 16)
        for (long f = 0; f < frames; f++)
            learned16_one(&c, iterations, cap, Ah, NBh, llr + f * c.n, post + f * c.n, decoded + f * c.n, msg,
                          iters ? iters + f : NULL, synfail ? synfail + f : NULL);
        free(msg);
    }
    free(Ah);
    return 0;
}

/* log(1 + exp(x)) and the logistic function, both stable for large |x|. */
static double softplus(double x) { return x > 0 ? x + log1p(exp(-x)) : log1p(exp(x)); }
static double sigmoid(double x) { return x >= 0 ? 1.0 / (1.0 + exp(-x)) : exp(x) / (1.0 + exp(x)); }

double wo_learned_loss_grad(int rate, int z, int iterations, const float* w, long frames,
                            const float* llr, const uint8_t* cw, double* grad)
{
    /* Forward in float with exactly the decoder's operations (so that every
     * min / argmin / gate decision equals the device's), tape kept, and the
     * reverse sweep accumulated in double. Subgradients: sign() and the
     * argmin choice are constants; d|x|/dx = sign(x) with signbit; relu'(0) = 0.
     * Routing of the min: i1 = first edge with |L| == min1, i2 = first other
     * edge with |L| == min2; edge e != i1 takes its magnitude from i1, edge i1
     * from i2. */
    wo_code_t c;
    if (wo_code(rate, z, &c)) return NAN;
    const int T = iterations, n = c.n, E = c.nblk * z;
    const size_t WN = (size_t)T * WO_L * WO_NB;
    const float* A = w;
    const float* B = w + WN;
    memset(grad, 0, sizeof(double) * 2 * WN);
    const double inv = 1.0 / ((double)T * (double)n * (double)frames);

    float* P = (float*)malloc(sizeof(float) * n);
    float* msg = (float*)malloc(sizeof(float) * E);
    double* gP = (double*)malloc(sizeof(double) * n);
    double* gm = (double*)malloc(sizeof(double) * E);
    float* Lt = (float*)malloc(sizeof(float) * (size_t)T * E);
    float* mut = (float*)malloc(sizeof(float) * (size_t)T * E);
    int* srct = (int*)malloc(sizeof(int) * (size_t)T * E);
    signed char* st = (signed char*)malloc((size_t)T * E);
    signed char* gt = (signed char*)malloc((size_t)T * E);
    float* Pt = (float*)malloc(sizeof(float) * (size_t)T * n);
    double loss = 0.0;

    for (long f = 0; f < frames; f++) {
        const float* lf = llr + f * n;
        const uint8_t* cf = cw + f * n;
        memcpy(P, lf, sizeof(float) * n);
        memset(msg, 0, sizeof(float) * E);
        for (int t = 0; t < T; t++) {
            for (int i = 0; i < c.mb; i++) {
                const int b0 = c.row_start[i], d = c.row_start[i + 1] - b0;
                for (int r = 0; r < z; r++) {
                    float L[WO_NB] = {0};
                    int v[WO_NB];
                    unsigned negpar = 0;
                    float m1 = INFINITY, m2 = INFINITY;
                    for (int e = 0; e < d; e++) {
                        v[e] = var_of(&c, b0 + e, r);
                        L[e] = P[v[e]] - msg[(b0 + e) * z + r];
                        negpar ^= (unsigned)(signbit(L[e]) != 0);
                        float a = fabsf(L[e]);
                        m2 = fminf(m2, fmaxf(m1, a));
                        m1 = fminf(m1, a);
                    }
                    int i1 = 0, i2 = -1;
                    while (fabsf(L[i1]) != m1) i1++;
                    for (int e = 0; e < d; e++)
                        if (e != i1 && fabsf(L[e]) == m2) { i2 = e; break; }
                    for (int e = 0; e < d; e++) {
                        const int eg = (b0 + e) * z + r;
                        const int col = c.blk_col[b0 + e];
                        const unsigned neg = negpar ^ (unsigned)(signbit(L[e]) != 0) ^ (unsigned)(d & 1);
                        const float mu = (fabsf(L[e]) == m1) ? m2 : m1;
                        const float pre = fmaf(A[widx(t, i, col)], mu, -B[widx(t, i, col)]);
                        const float mag = fmaxf(pre, 0.0f);
                        const float m = flip_sign(mag, neg);
                        const size_t k = (size_t)t * E + eg;
                        Lt[k] = L[e];
                        mut[k] = mu;
                        srct[k] = (b0 + ((e == i1) ? i2 : i1)) * z + r;
                        st[k] = (signed char)(neg ? -1 : 1);
                        gt[k] = (signed char)(pre > 0.0f);
                        msg[eg] = m;
                        P[v[e]] = L[e] + m;
                    }
                }
            }
            for (int v = 0; v < n; v++) {
                Pt[(size_t)t * n + v] = P[v];
                const double sg = cf[v] ? -1.0 : 1.0;      /* loss = softplus(sg * P) */
                loss += softplus(sg * (double)P[v]) * inv;
            }
        }
        memset(gP, 0, sizeof(double) * n);
        memset(gm, 0, sizeof(double) * E);
        for (int t = T - 1; t >= 0; t--) {
            for (int v = 0; v < n; v++) {
                const double sg = cf[v] ? -1.0 : 1.0;
                gP[v] += sg * sigmoid(sg * (double)Pt[(size_t)t * n + v]) * inv;
            }
            for (int i = c.mb - 1; i >= 0; i--) {
                const int b0 = c.row_start[i], d = c.row_start[i + 1] - b0;
                for (int r = 0; r < z; r++) {
                    double gL[WO_NB];
                    int v[WO_NB];
                    for (int e = 0; e < d; e++) {
                        v[e] = var_of(&c, b0 + e, r);
                        gL[e] = gP[v[e]];
                    }
                    for (int e = 0; e < d; e++) {
                        const int eg = (b0 + e) * z + r;
                        const size_t k = (size_t)t * E + eg;
                        if (!gt[k]) continue;
                        const int col = c.blk_col[b0 + e];
                        const double G = gP[v[e]] + gm[eg];
                        const double s = (double)st[k];
                        grad[widx(t, i, col)] += G * s * (double)mut[k];
                        grad[WN + widx(t, i, col)] += -G * s;
                        const double gmu = G * s * (double)A[widx(t, i, col)];
                        const int src = srct[k];
                        const int se = src / z - b0;
                        const float Ls = Lt[(size_t)t * E + src];
                        gL[se] += gmu * (signbit(Ls) ? -1.0 : 1.0);
                    }
                    for (int e = 0; e < d; e++) {
                        gP[v[e]] = gL[e];
                        gm[(b0 + e) * z + r] = -gL[e];
                    }
                }
            }
        }
    }
    free(P); free(msg); free(gP); free(gm);
    free(Lt); free(mut); free(srct); free(st); free(gt); free(Pt);
    return loss;
}
