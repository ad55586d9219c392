/*
 * Drop-in for the reference's wimax_ldpc_lib::ldpc_decoder (reference
 * include/ldpc_decoder.h:11-34): same constructor and methods, decoding on a
 * B200 through the C ABI in wimax_ldpc_b200.h. The batch methods are
 * additions; they have no counterpart in the reference.
 */
#ifndef LDPC_DECODER_H
#define LDPC_DECODER_H

#include <stddef.h>
#include <stdint.h>

#include "enums.h"
#include "ldpc.h"

struct wldpc_decoder;

namespace wimax_ldpc_lib {

class WIMAX_LDPC_LIB_API ldpc_decoder : public ldpc
{
private:
    unsigned int m_max_iter;
    wldpc_decoder* m_handle;
    int m_last_iterations;

public:
    ldpc_decoder();
    ldpc_decoder(coderate rate, unsigned int z_factor, unsigned int max_iter, unsigned int num_threads);
    ~ldpc_decoder();

    unsigned int compute_syndrome(int8_t* rx_codeword, bool exit_early);
    unsigned int decode(int8_t* rx_codeword, int8_t* decoded);
    unsigned int decode(float* rx_codeword, int8_t* decoded);

    /* additions */
    /* iterations executed by the last decode(float*) call */
    int last_iterations() const { return m_last_iterations; }
    /* frames x n host buffers; rx_codewords receives the posteriors;
     * num_errors (nullable) gets the per-frame return values of decode() */
    void decode_batch(float* rx_codewords, int8_t* decoded, size_t frames, uint32_t* num_errors = nullptr);
    /* device buffers, asynchronous on stream (a cudaStream_t or nullptr) */
    void decode_device(const float* llr, int8_t* decoded, float* posterior, int32_t* status, size_t frames,
                       void* stream = nullptr);
};

}  // namespace wimax_ldpc_lib

#endif  // LDPC_DECODER_H
