/*
 * C-ABI harness around the UNMODIFIED reference classes
 * (wimax_ldpc_lib::ldpc_decoder / ldpc_encoder / BER_runner, reference
 * include/ldpc_decoder.h:24-33, include/ldpc_encoder.h:21-24,
 * include/BER_runner.h:52-68). It is compiled together with the reference's own
 * lib/*.cc sources by oracle/Makefile into oracle/_ref/libwldpc_ref*.so.
 *
 * TEST INFRASTRUCTURE ONLY. Tests, the smoke check and bench.py's CPU
 * baseline load it to pin the C restatement (wldpc_oracle.c), to generate the
 * golden fixtures under tests/golden/ and to time the reference's own OpenMP
 * CPU decoder. The product library never links or calls it.
 *
 * Every function returns a negative value when the reference constructor
 * throws (invalid rate / z, reference lib/ldpc.cc:46-57,1198-1202).
 */
#include <stdint.h>
#include <string.h>
#include <omp.h>
#include <vector>
#include <exception>
#include <random>

#include "ldpc_decoder.h"
#include "ldpc_encoder.h"
#include "BER_runner.h"

using namespace wimax_ldpc_lib;

namespace {
/* Exposes the protected code description of the reference base class
 * (reference include/ldpc.h:41-51). */
struct code_probe : public ldpc {
    code_probe(coderate r, unsigned z) : ldpc(r, z, 1) {}
    void info(int* o) const {
        o[0] = (int)m_N; o[1] = (int)m_M; o[2] = (int)m_z;
        o[3] = (int)m_row_size; o[4] = (int)m_col_size;
        o[5] = (int)m_D; o[6] = (int)m_X;
    }
    const int16_t* table() const { return m_checknode_array; }
};
}  // namespace

extern "C" {

/* out[7] = {N, M, z, rows, cols, D, X}. */
int ref_code_info(int rate, int z, int* out)
{
    try {
        code_probe p((coderate)rate, (unsigned)z);
        p.info(out);
        return 0;
    } catch (...) { return -1; }
}

/* Copies the expanded check-node table (rows x cols int16, -1 padded). */
int ref_checknode_table(int rate, int z, int16_t* out, long capacity)
{
    try {
        code_probe p((coderate)rate, (unsigned)z);
        int o[7]; p.info(o);
        long cnt = (long)o[3] * o[4];
        if (cnt > capacity) return -2;
        memcpy(out, p.table(), sizeof(int16_t) * cnt);
        return 0;
    } catch (...) { return -1; }
}

/* decode(float*, int8_t*) over a batch: one decoder object per OpenMP thread,
 * `omp parallel for` over frames (the reference lib/decode_example.cc:76,128-135
 * pattern). llr is updated in place with the posterior (reference semantics). */
int ref_decode_batch(int rate, int z, int max_iter, long frames, float* llr,
                     int8_t* decoded, uint32_t* ret, int threads)
{
    if (threads < 1) threads = 1;
    std::vector<ldpc_decoder*> dec(threads, nullptr);
    int n = 0;
    try {
        for (int t = 0; t < threads; t++)
            dec[t] = new ldpc_decoder((coderate)rate, (unsigned)z, (unsigned)max_iter, 1);
        int o[7]; code_probe((coderate)rate, (unsigned)z).info(o); n = o[0];
    } catch (...) {
        for (auto d : dec) delete d;
        return -1;
    }
    #pragma omp parallel for num_threads(threads) schedule(static)
    for (long f = 0; f < frames; f++) {
        int t = omp_get_thread_num();
        ret[f] = dec[t]->decode(llr + f * n, decoded + f * n);
    }
    for (auto d : dec) delete d;
    return 0;
}

/* decode(int8_t*, int8_t*): hard-bit input adapter (reference
 * lib/ldpc_decoder.cc:108-118). */
int ref_decode_bits_batch(int rate, int z, int max_iter, long frames, int8_t* bits,
                          int8_t* decoded, uint32_t* ret, int threads)
{
    if (threads < 1) threads = 1;
    std::vector<ldpc_decoder*> dec(threads, nullptr);
    int n = 0;
    try {
        for (int t = 0; t < threads; t++)
            dec[t] = new ldpc_decoder((coderate)rate, (unsigned)z, (unsigned)max_iter, 1);
        int o[7]; code_probe((coderate)rate, (unsigned)z).info(o); n = o[0];
    } catch (...) {
        for (auto d : dec) delete d;
        return -1;
    }
    #pragma omp parallel for num_threads(threads) schedule(static)
    for (long f = 0; f < frames; f++) {
        int t = omp_get_thread_num();
        ret[f] = dec[t]->decode(bits + f * n, decoded + f * n);
    }
    for (auto d : dec) delete d;
    return 0;
}

/* compute_syndrome(int8_t*, bool) per frame (reference lib/ldpc_decoder.cc:67-104). */
int ref_syndrome_batch(int rate, int z, long frames, int8_t* bits, int early_exit,
                       uint32_t* ret)
{
    try {
        ldpc_decoder d((coderate)rate, (unsigned)z, 1, 1);
        int o[7]; code_probe((coderate)rate, (unsigned)z).info(o);
        for (long f = 0; f < frames; f++)
            ret[f] = d.compute_syndrome(bits + f * o[0], early_exit != 0);
        return 0;
    } catch (...) { return -1; }
}

/* Iteration count by the rebuild-with-smaller-cap recipe: the first k
 * iterations of decode() do not depend on max_iter (messages of slice i are
 * written before they are read, reference lib/ldpc_decoder.cc:36-38,162,184),
 * so iterations = smallest k in [1, cap] whose decoder returns 0, 0 when the
 * sliced input already satisfies the syndrome, and cap+1 when none does. */
int ref_iterations(int rate, int z, int cap, long frames, const float* llr,
                   int32_t* iters, int threads)
{
    if (threads < 1) threads = 1;
    int n;
    try { int o[7]; code_probe((coderate)rate, (unsigned)z).info(o); n = o[0]; }
    catch (...) { return -1; }
    std::vector<std::vector<ldpc_decoder*>> dec(threads);
    for (int t = 0; t < threads; t++)
        for (int k = 0; k <= cap; k++)
            dec[t].push_back(new ldpc_decoder((coderate)rate, (unsigned)z, (unsigned)k, 1));
    #pragma omp parallel for num_threads(threads) schedule(dynamic, 4)
    for (long f = 0; f < frames; f++) {
        int t = omp_get_thread_num();
        std::vector<float> buf(n);
        std::vector<int8_t> hard(n);
        for (int i = 0; i < n; i++) hard[i] = llr[f * n + i] >= 0.0f;
        if (dec[t][0]->compute_syndrome(hard.data(), true) == 0) { iters[f] = 0; continue; }
        int found = cap + 1;
        for (int k = 1; k <= cap; k++) {
            memcpy(buf.data(), llr + f * n, sizeof(float) * n);
            if (dec[t][k]->decode(buf.data(), hard.data()) == 0) { found = k; break; }
        }
        iters[f] = found;
    }
    for (auto& v : dec) for (auto d : v) delete d;
    return 0;
}

/* encode_data over a batch (reference lib/ldpc_encoder.cc:50-105). The
 * encoder forks OpenMP internally with its num_threads (reference
 * lib/ldpc_encoder.cc:34); it is given 1 thread here and frames run in parallel. */
int ref_encode_batch(int rate, int z, long frames, const uint8_t* info, uint8_t* cw,
                     int threads)
{
    if (threads < 1) threads = 1;
    int o[7];
    try { code_probe((coderate)rate, (unsigned)z).info(o); } catch (...) { return -1; }
    int n = o[0], k = o[0] - o[1];
    std::vector<ldpc_encoder*> enc(threads, nullptr);
    try {
        for (int t = 0; t < threads; t++) enc[t] = new ldpc_encoder((coderate)rate, (unsigned)z, 1);
    } catch (...) {
        for (auto e : enc) delete e;
        return -1;
    }
    #pragma omp parallel for num_threads(threads) schedule(static)
    for (long f = 0; f < frames; f++) {
        int t = omp_get_thread_num();
        std::vector<uint8_t> in(info + f * k, info + (f + 1) * k);
        enc[t]->encode_data(in.data(), cw + f * n);
    }
    for (auto e : enc) delete e;
    return 0;
}

/* BER_runner (reference lib/BER_runner.cc). */
void* ref_ber_create(int rate, int z, int threads, int max_iter)
{
    try { return new BER_runner((coderate)rate, (unsigned)z, (unsigned)threads, (unsigned)max_iter); }
    catch (...) { return nullptr; }
}
double ref_ber_run_iteration(void* h, double ebno_db) { return ((BER_runner*)h)->run_iteration(ebno_db); }
void ref_ber_reset(void* h) { ((BER_runner*)h)->reset_test(); }
uint64_t ref_ber_bits(void* h) { return ((BER_runner*)h)->get_total_num_bits(); }
uint64_t ref_ber_errors(void* h) { return ((BER_runner*)h)->get_total_num_errors(); }
unsigned ref_ber_codeword_len(void* h) { return ((BER_runner*)h)->get_codeword_len(); }
unsigned ref_ber_dataword_len(void* h) { return ((BER_runner*)h)->get_dataword_len(); }
void ref_ber_destroy(void* h) { delete (BER_runner*)h; }

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
