// GPU-backed test_decoder: same arguments, input and output files as the
// reference tool (reference lib/decode_example.cc): reads num_codewords
// codewords of n bytes (hard bits), decodes them as decode(int8_t*, int8_t*)
// with MAX_ITER 10, writes the first k bytes (the dataword) of every decoded
// frame, and prints the initial / final error counts per frame and the
// timing lines. Like the reference, frames are taken in groups of num_threads
// and a final partial group is not decoded (reference :118). The whole batch
// is one GPU call, so the per-group rate line is printed once for the batch.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "wimax_ldpc_b200.h"

#define MAX_ITER 10

int main(int argc, char* argv[])
{
    if (argc != 7) {
        printf("\nError: Incorrect number of arguments\n");
        printf("Usage: ./test_decoder <num_threads> <rate> <z> <num_codewords> <encoded_data_file> <decoded_data_file>\n");
        return 0;
    }
    const unsigned num_threads = (unsigned)std::stoi(argv[1], nullptr, 0);
    const int rate = std::stoi(argv[2], nullptr, 0);
    const unsigned z = (unsigned)std::stoi(argv[3], nullptr, 0);
    const unsigned num_codewords = (unsigned)std::stoi(argv[4], nullptr, 0);
    wldpc_code_info ci;
    if (wldpc_code_info_get(rate, z, &ci) != WLDPC_OK || num_threads == 0) {
        printf("[!]ldpc_encoder - Invalid Coderate: %d\n", rate);
        return 1;
    }
    const size_t n = (size_t)ci.n, k = (size_t)ci.k;
    std::vector<int8_t> in((size_t)num_codewords * n);
    FILE* fin = fopen(argv[5], "rb");
    FILE* fout = fopen(argv[6], "wb");
    if (!fin || !fout) {
        printf("[!] Error: cannot open files.\n");
        return 1;
    }
    if (fread(in.data(), 1, in.size(), fin) != in.size()) {
        printf("[!] Error: File does not contain enough data.\n");
        return 0;
    }
    fclose(fin);
    const size_t frames = (size_t)(num_codewords / num_threads) * num_threads;
    wldpc_decoder* dec = nullptr;
    int rc = wldpc_decoder_create(rate, z, MAX_ITER, num_threads, WLDPC_MODE_NMS, &dec);
    if (rc != WLDPC_OK) {
        printf("[!] GPU decoder: %s\n", wldpc_strerror(rc));
        return 1;
    }
    std::vector<uint32_t> initial(frames), final_errors(frames);
    std::vector<int8_t> out(frames * n);
    rc = wldpc_syndrome_batch_host(dec, in.data(), 0, initial.data(), frames);
    const auto t0 = std::chrono::high_resolution_clock::now();
    if (rc == WLDPC_OK) rc = wldpc_decode_bits_batch_host(dec, in.data(), out.data(), final_errors.data(), frames);
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (rc != WLDPC_OK) {
        printf("[!] GPU decode: %s\n", wldpc_strerror(rc));
        return 1;
    }
    const double ns = (double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    for (size_t f = 0; f < frames; f++) fwrite(out.data() + f * n, 1, k, fout);
    fclose(fout);
    printf("Rate (Mbits/Sec): %f\n", (frames * n * 1000.0) / ns);
    for (size_t f = 0; f < frames; f++) {
        printf("Initial Number of Errors (%u): %u\n", (unsigned)(f % num_threads), initial[f]);
        printf("Final Number of Errors (%u): %u\n", (unsigned)(f % num_threads), final_errors[f]);
    }
    printf("\nTiming Statistics:\n\n");
    printf("Average Rate (Mbits/Sec): %f\n", (frames * n * 1000.0) / ns);
    printf("Fastest Iteration (Mbits/Sec): %f\n", (frames * n * 1000.0) / ns);
    printf("Slowest Iteration (Mbits/Sec): %f\n", (frames * n * 1000.0) / ns);
    wldpc_decoder_destroy(dec);
    return 1;
}
