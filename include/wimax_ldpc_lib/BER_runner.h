/*
 * Drop-in for the reference's wimax_ldpc_lib::BER_runner (reference
 * include/BER_runner.h:11-71): same LFSR info bits, mt19937(0) noise stream
 * and error accounting; encoding and decoding run on a B200.
 */
#ifndef BER_RUNNER_H
#define BER_RUNNER_H

#include <stdint.h>

#include "enums.h"
#include "ldpc.h"

struct wldpc_ber_runner;

namespace wimax_ldpc_lib {

class WIMAX_LDPC_LIB_API BER_runner : public ldpc
{
private:
    wldpc_ber_runner* m_handle;

public:
    BER_runner();
    BER_runner(coderate rate, unsigned int z_factor, unsigned int num_threads, unsigned int max_iter);
    ~BER_runner();

    void reset_test();
    double run_iteration(double EbNo_dB);
    uint64_t get_total_num_bits();
    uint64_t get_total_num_errors();
    unsigned int get_codeword_len();
    unsigned int get_dataword_len();
};

}  // namespace wimax_ldpc_lib

#endif  // BER_RUNNER_H
