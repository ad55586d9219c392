/*
 * Base class of the codec objects, mirroring the reference's wimax_ldpc_lib::ldpc
 * (reference include/ldpc.h:35-61): selects the code for (rate, z) and holds
 * its description. Invalid rate or z: printf + throw std::exception(), as the
 * reference does (reference lib/ldpc.cc:46-57,1198-1202).
 */
#ifndef LDPC_H
#define LDPC_H

#include <stdint.h>
#include <stdio.h>
#include <exception>

#include "enums.h"

#define BASE_LDPC_BLOCK_LEN 2304

#if defined(__GNUC__)
#define WIMAX_LDPC_LIB_API __attribute__((visibility("default")))
#else
#define WIMAX_LDPC_LIB_API
#endif

namespace wimax_ldpc_lib {

class WIMAX_LDPC_LIB_API ldpc
{
protected:
    int16_t* m_checknode_array;   /* expanded table [m_row_size][m_col_size], -1 padded */

    unsigned int m_D;
    unsigned int m_N;
    unsigned int m_M;
    unsigned int m_X;
    unsigned int m_z;
    unsigned int m_col_size;
    unsigned int m_row_size;
    unsigned int m_num_threads;
    coderate m_rate;

public:
    ldpc();
    ldpc(coderate rate, unsigned int z_factor, unsigned int num_threads);
    ~ldpc();
    ldpc(const ldpc&) = delete;
    ldpc& operator=(const ldpc&) = delete;

    uint64_t get_nanoseconds();
};

}  // namespace wimax_ldpc_lib

#endif  // LDPC_H
