/*
 * C++ facade: the reference's public classes (wimax_ldpc_lib::ldpc,
 * ldpc_decoder, ldpc_encoder, BER_runner) re-created over the C ABI, so that
 * code written against the reference headers compiles and runs unchanged.
 * Error behaviour follows the reference: an invalid rate or z prints a
 * message and throws std::exception (reference lib/ldpc.cc:46-57,1198-1202);
 * a failure of the GPU path throws std::runtime_error.
 */
#include <chrono>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "wimax_ldpc_b200.h"
#include "wimax_ldpc_lib/BER_runner.h"
#include "wimax_ldpc_lib/ldpc.h"
#include "wimax_ldpc_lib/ldpc_decoder.h"
#include "wimax_ldpc_lib/ldpc_encoder.h"

namespace wimax_ldpc_lib {

static void throw_gpu(const char* what, int rc)
{
    throw std::runtime_error(std::string(what) + ": " + wldpc_strerror(rc));
}

ldpc::ldpc()
    : m_checknode_array(nullptr), m_D(0), m_N(0), m_M(0), m_X(0), m_z(0), m_col_size(0), m_row_size(0),
      m_num_threads(0), m_rate(HALFRATE)
{
}

ldpc::ldpc(coderate rate, unsigned int z_factor, unsigned int num_threads) : ldpc()
{
    wldpc_code_info ci;
    const int rc = wldpc_code_info_get((int)rate, z_factor, &ci);
    if (rc != WLDPC_OK) {
        if ((int)rate < 0 || (int)rate > 5)
            printf("[!]ldpc_encoder - Invalid Coderate: %d\n", (int)rate);
        else
            printf("[!]ldpc_encoder - Invalid Z factor: %d\n", (int)z_factor);
        throw std::exception();
    }
    m_rate = rate;
    m_num_threads = num_threads;
    m_z = z_factor;
    m_N = (unsigned)ci.n;
    m_M = (unsigned)ci.m;
    m_D = (unsigned)ci.D;
    m_X = (unsigned)ci.X;
    m_row_size = (unsigned)ci.rows;
    m_col_size = (unsigned)ci.cols;
    m_checknode_array = new int16_t[(size_t)m_row_size * m_col_size];
    wldpc_checknode_table((int)rate, z_factor, m_checknode_array, (size_t)m_row_size * m_col_size);
}

ldpc::~ldpc() { delete[] m_checknode_array; }

uint64_t ldpc::get_nanoseconds()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::high_resolution_clock::now().time_since_epoch())
        .count();
}

/* ------------------------------------------------------------ decoder */

ldpc_decoder::ldpc_decoder() : ldpc(), m_max_iter(0), m_handle(nullptr), m_last_iterations(0) {}

ldpc_decoder::ldpc_decoder(coderate rate, unsigned int z_factor, unsigned int max_iter, unsigned int num_threads)
    : ldpc(rate, z_factor, num_threads), m_max_iter(max_iter), m_handle(nullptr), m_last_iterations(0)
{
    const int rc = wldpc_decoder_create((int)rate, z_factor, max_iter, num_threads, WLDPC_MODE_NMS, &m_handle);
    if (rc != WLDPC_OK) throw_gpu("ldpc_decoder", rc);
}

ldpc_decoder::~ldpc_decoder()
{
    if (m_handle) wldpc_decoder_destroy(m_handle);
}

unsigned int ldpc_decoder::compute_syndrome(int8_t* rx_codeword, bool exit_early)
{
    unsigned ne = 0;
    const int rc = wldpc_decoder_compute_syndrome(m_handle, rx_codeword, exit_early ? 1 : 0, &ne);
    if (rc != WLDPC_OK) throw_gpu("compute_syndrome", rc);
    return ne;
}

unsigned int ldpc_decoder::decode(int8_t* rx_codeword, int8_t* decoded)
{
    unsigned ne = 0;
    const int rc = wldpc_decoder_decode_bits(m_handle, rx_codeword, decoded, &ne);
    if (rc != WLDPC_OK) throw_gpu("decode", rc);
    return ne;
}

unsigned int ldpc_decoder::decode(float* rx_codeword, int8_t* decoded)
{
    unsigned ne = 0;
    const int rc = wldpc_decoder_decode(m_handle, rx_codeword, decoded, &ne, &m_last_iterations);
    if (rc != WLDPC_OK) throw_gpu("decode", rc);
    return ne;
}

void ldpc_decoder::decode_batch(float* rx_codewords, int8_t* decoded, size_t frames, uint32_t* num_errors)
{
    const int rc = wldpc_decode_batch_host(m_handle, rx_codewords, decoded, num_errors, nullptr, frames);
    if (rc != WLDPC_OK) throw_gpu("decode_batch", rc);
}

void ldpc_decoder::decode_device(const float* llr, int8_t* decoded, float* posterior, int32_t* status,
                                 size_t frames, void* stream)
{
    const int rc = wldpc_decode_batch_device(m_handle, llr, decoded, posterior, status, frames, stream);
    if (rc != WLDPC_OK) throw_gpu("decode_device", rc);
}

/* ------------------------------------------------------------ encoder */

ldpc_encoder::ldpc_encoder(coderate rate, unsigned int z_factor, unsigned int num_threads)
    : ldpc(rate, z_factor, num_threads), m_handle(nullptr)
{
    const int rc = wldpc_encoder_create((int)rate, z_factor, num_threads, &m_handle);
    if (rc != WLDPC_OK) throw_gpu("ldpc_encoder", rc);
}

ldpc_encoder::~ldpc_encoder()
{
    if (m_handle) wldpc_encoder_destroy(m_handle);
}

void ldpc_encoder::encode_data(uint8_t* infoword, uint8_t* codeword)
{
    const int rc = wldpc_encoder_encode(m_handle, infoword, codeword);
    if (rc != WLDPC_OK) throw_gpu("encode_data", rc);
}

void ldpc_encoder::encode_device(const uint8_t* info, uint8_t* codeword, size_t frames, void* stream)
{
    const int rc = wldpc_encode_batch_device(m_handle, info, codeword, frames, stream);
    if (rc != WLDPC_OK) throw_gpu("encode_device", rc);
}

/* --------------------------------------------------------- BER runner */

BER_runner::BER_runner() : ldpc(), m_handle(nullptr) {}

BER_runner::BER_runner(coderate rate, unsigned int z_factor, unsigned int num_threads, unsigned int max_iter)
    : ldpc(rate, z_factor, num_threads), m_handle(nullptr)
{
    const int rc = wldpc_ber_runner_create((int)rate, z_factor, num_threads, max_iter, &m_handle);
    if (rc == WLDPC_ERR_UNSUPPORTED) {
        printf("[!]ber_runner - 3/4B Not Implemented\n");   /* reference lib/BER_runner.cc:66-71 */
        throw std::exception();
    }
    if (rc != WLDPC_OK) throw_gpu("BER_runner", rc);
}

BER_runner::~BER_runner()
{
    if (m_handle) wldpc_ber_runner_destroy(m_handle);
}

void BER_runner::reset_test() { wldpc_ber_runner_reset(m_handle); }

double BER_runner::run_iteration(double EbNo_dB)
{
    double ber = 0.0;
    const int rc = wldpc_ber_runner_run_iteration(m_handle, EbNo_dB, &ber);
    if (rc != WLDPC_OK) throw_gpu("run_iteration", rc);
    return ber;
}

uint64_t BER_runner::get_total_num_bits()
{
    uint64_t b = 0;
    wldpc_ber_runner_totals(m_handle, &b, nullptr);
    return b;
}

uint64_t BER_runner::get_total_num_errors()
{
    uint64_t e = 0;
    wldpc_ber_runner_totals(m_handle, nullptr, &e);
    return e;
}

unsigned int BER_runner::get_codeword_len()
{
    unsigned c = 0;
    wldpc_ber_runner_lengths(m_handle, &c, nullptr);
    return c;
}

unsigned int BER_runner::get_dataword_len()
{
    unsigned d = 0;
    wldpc_ber_runner_lengths(m_handle, nullptr, &d);
    return d;
}

}  // namespace wimax_ldpc_lib
