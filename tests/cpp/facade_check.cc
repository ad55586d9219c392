// Drives the C++ facade exactly as reference code would use the reference
// classes (reference lib/decode_example.cc:76,128-135, lib/encode_example.cc,
// lib/BER_example.cc), so that the test can compare its outputs with the oracle.
//
//   facade_check decode <rate> <z> <frames> <max_iter> <llr.f32> <out.bin>
//       per frame: ldpc_decoder::decode(float*, int8_t*); writes the posterior
//       (n float32, in place), decoded (n int8) and the return value (uint32)
//   facade_check encode <rate> <z> <frames> <info.u8> <out.u8>
//   facade_check ber <rate> <z> <iters> <ebno>      prints bits errors ber
//   facade_check invalid                             exits 0 if the facade throws
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <vector>

#include <wimax_ldpc_lib/BER_runner.h>
#include <wimax_ldpc_lib/ldpc_decoder.h>
#include <wimax_ldpc_lib/ldpc_encoder.h>

using namespace wimax_ldpc_lib;

static std::vector<char> slurp(const char* path)
{
    FILE* f = fopen(path, "rb");
    if (!f) { perror(path); exit(2); }
    std::vector<char> v;
    char buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + r);
    fclose(f);
    return v;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    if (!strcmp(argv[1], "decode") && argc == 8) {
        coderate rate = (coderate)atoi(argv[2]);
        unsigned z = (unsigned)atoi(argv[3]), frames = (unsigned)atoi(argv[4]), max_iter = (unsigned)atoi(argv[5]);
        ldpc_decoder dec(rate, z, max_iter, 1);
        const unsigned n = (unsigned)((z / 96.0) * BASE_LDPC_BLOCK_LEN);
        std::vector<char> in = slurp(argv[6]);
        float* llr = reinterpret_cast<float*>(in.data());
        FILE* out = fopen(argv[7], "wb");
        std::vector<int8_t> decoded(n);
        for (unsigned f = 0; f < frames; f++) {
            unsigned ret = dec.decode(llr + (size_t)f * n, decoded.data());
            fwrite(llr + (size_t)f * n, sizeof(float), n, out);
            fwrite(decoded.data(), 1, n, out);
            fwrite(&ret, sizeof ret, 1, out);
        }
        fclose(out);
        return 0;
    }
    if (!strcmp(argv[1], "encode") && argc == 7) {
        coderate rate = (coderate)atoi(argv[2]);
        unsigned z = (unsigned)atoi(argv[3]), frames = (unsigned)atoi(argv[4]);
        ldpc_encoder enc(rate, z, 4);
        const unsigned n = (unsigned)((z / 96.0) * BASE_LDPC_BLOCK_LEN);
        std::vector<char> in = slurp(argv[5]);
        const unsigned k = (unsigned)(in.size() / frames);
        FILE* out = fopen(argv[6], "wb");
        std::vector<uint8_t> cw(n);
        for (unsigned f = 0; f < frames; f++) {
            enc.encode_data(reinterpret_cast<uint8_t*>(in.data()) + (size_t)f * k, cw.data());
            fwrite(cw.data(), 1, n, out);
        }
        fclose(out);
        return 0;
    }
    if (!strcmp(argv[1], "ber") && argc == 6) {
        BER_runner b((coderate)atoi(argv[2]), (unsigned)atoi(argv[3]), 1, 10);
        double ber = 0;
        for (int i = 0; i < atoi(argv[4]); i++) ber = b.run_iteration(atof(argv[5]));
        printf("%llu %llu %.17g %u %u\n", (unsigned long long)b.get_total_num_bits(),
               (unsigned long long)b.get_total_num_errors(), ber, b.get_codeword_len(), b.get_dataword_len());
        return 0;
    }
    if (!strcmp(argv[1], "invalid")) {
        int thrown = 0;
        try { ldpc_decoder d((coderate)0, 25, 10, 1); } catch (std::exception&) { thrown++; }
        try { ldpc_encoder e((coderate)9, 96, 1); } catch (std::exception&) { thrown++; }
        try { BER_runner b(THREEQUARTERSB, 96, 1, 10); } catch (std::exception&) { thrown++; }
        printf("thrown %d\n", thrown);
        return thrown == 3 ? 0 : 1;
    }
    return 2;
}
