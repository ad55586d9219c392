/*
 * Drop-in for the reference's wimax_ldpc_lib::ldpc_encoder (reference
 * include/ldpc_encoder.h:11-27), encoding on a B200 through the C ABI.
 */
#ifndef LDPC_ENCODER_H
#define LDPC_ENCODER_H

#include <stddef.h>
#include <stdint.h>

#include "enums.h"
#include "ldpc.h"

struct wldpc_encoder;

namespace wimax_ldpc_lib {

class WIMAX_LDPC_LIB_API ldpc_encoder : public ldpc
{
private:
    wldpc_encoder* m_handle;

public:
    ldpc_encoder(coderate rate, unsigned int z_factor, unsigned int num_threads);
    ~ldpc_encoder();

    void encode_data(uint8_t* infoword, uint8_t* codeword);

    /* addition: frames x k -> frames x n device buffers, asynchronous */
    void encode_device(const uint8_t* info, uint8_t* codeword, size_t frames, void* stream = nullptr);
};

}  // namespace wimax_ldpc_lib

#endif  // LDPC_ENCODER_H
