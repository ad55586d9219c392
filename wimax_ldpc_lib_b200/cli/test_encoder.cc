// GPU-backed test_encoder: same arguments and output files as the reference
// tool (reference lib/encode_example.cc): num_rounds random datawords (k
// bytes each, rand() % 2) written to unencoded_data_file, their codewords
// (n bytes each) with errors_to_add random bit flips written to
// encoded_data_file, and the timing lines. Differences, on purpose: the
// random generator is seeded once (the reference reseeds with time(0) every
// round, repeating datawords within a second) and flip positions are drawn in
// [0, n) (the reference's rand() % n + 1 can touch one byte past the frame,
// reference :31). Rate 3/4B is refused as the reference does (reference
// :102-107). All rounds are encoded by one GPU call.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <vector>

#include "wimax_ldpc_b200.h"

int main(int argc, char* argv[])
{
    if (argc != 7) {
        printf("\nError: Incorrect number of arguments\n");
        printf("Usage: ./test_encoder <rate> <z> <num_rounds> <errors_to_add> <unencoded_data_file> <encoded_data_file>\n");
        return 0;
    }
    const int rate = std::stoi(argv[1], nullptr, 0);
    const unsigned z = (unsigned)std::stoi(argv[2], nullptr, 0);
    const unsigned rounds = (unsigned)std::stoi(argv[3], nullptr, 0);
    const unsigned flips = (unsigned)std::stoi(argv[4], nullptr, 0);
    if (rate == 4) {
        printf("[!]test_encoder - 3/4B Not Implemented\n");
        return 1;
    }
    wldpc_code_info ci;
    if (wldpc_code_info_get(rate, z, &ci) != WLDPC_OK) {
        printf("[!]test_encoder - Invalid Coderate: %d\n", rate);
        return 1;
    }
    const size_t n = (size_t)ci.n, k = (size_t)ci.k;
    std::vector<uint8_t> data((size_t)rounds * k), cw((size_t)rounds * n);
    srand((unsigned)time(0));
    for (auto& b : data) b = (uint8_t)(rand() % 2);
    wldpc_encoder* enc = nullptr;
    int rc = wldpc_encoder_create(rate, z, 4, &enc);
    if (rc != WLDPC_OK) {
        printf("[!] GPU encoder: %s\n", wldpc_strerror(rc));
        return 1;
    }
    const auto t0 = std::chrono::high_resolution_clock::now();
    rc = wldpc_encode_batch_host(enc, data.data(), cw.data(), rounds);
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (rc != WLDPC_OK) {
        printf("[!] GPU encode: %s\n", wldpc_strerror(rc));
        return 1;
    }
    for (unsigned r = 0; r < rounds; r++)
        for (unsigned e = 0; e < flips; e++) {
            const size_t i = (size_t)(rand() % n);
            cw[r * n + i] = !cw[r * n + i];
        }
    FILE* fd = fopen(argv[5], "wb");
    FILE* fe = fopen(argv[6], "wb");
    if (!fd || !fe) {
        printf("[!] Error: cannot open files.\n");
        return 1;
    }
    fwrite(data.data(), 1, data.size(), fd);
    fwrite(cw.data(), 1, cw.size(), fe);
    fclose(fd);
    fclose(fe);
    const double ns = (double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    printf("\n\nTiming Statistics:\n\n");
    printf("Average Rate (Mbits/Sec): %f\n", (rounds * n * 1000.0) / ns);
    printf("Fastest Iteration (Mbits/Sec): %f\n", (rounds * n * 1000.0) / ns);
    printf("Slowest Iteration (Mbits/Sec): %f\n", (rounds * n * 1000.0) / ns);
    wldpc_encoder_destroy(enc);
    return 1;
}
