/*
 * C ABI (include/wimax_ldpc_b200.h) over the sm_100a kernels.
 *
 * Handles own their CUDA stream and device scratch; buffers passed in are the
 * caller's. Single-frame calls keep the reference's synchronous, in-place
 * semantics (reference lib/ldpc_decoder.cc:122-262): copy in, decode on the
 * GPU, copy the posterior and hard bits back.
 */
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <random>
#include <vector>
#include <cuda_runtime.h>

#include "wimax_ldpc_b200.h"
#include "codec_kernels.cuh"

using namespace wldpc;

namespace {

int check_device()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    return WLDPC_OK;
}

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

#define CU(call)                                  \
    do {                                          \
        if ((call) != cudaSuccess) {              \
            cudaGetLastError();                   \
            return WLDPC_ERR_CUDA;                \
        }                                         \
    } while (0)

/* grow-only device buffer */
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t want)
    {
        if (want <= bytes) return WLDPC_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, want) != cudaSuccess) {
            cudaGetLastError();
            return WLDPC_ERR_CUDA;
        }
        bytes = want;
        return WLDPC_OK;
    }
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

/* An error after copies were queued on the host-batch pipeline streams: wait
 * for them (their results are not used) so that none writes into the caller's
 * buffers after the call has returned. */
template <int S>
static int drain_pipe(cudaStream_t (&pipe)[S], int rc)
{
    cudaGetLastError();
    for (cudaStream_t p : pipe)
        if (p) cudaStreamSynchronize(p);
    cudaGetLastError();
    return rc;
}

struct wldpc_decoder {
    int rate, z, mode;
    unsigned max_iter;
    unsigned wait_limit_us = kWaitLimitUs;   /* bound of the kernel's staging wait (test hook) */
    CodeDesc code;
    cudaStream_t stream = nullptr;
    cudaStream_t pipe[kHostStages] = {};
    unsigned* err = nullptr;   /* device error word */
    DevBuf llr, hard, status, bits;
    DevBuf pllr[kHostStages], phard[kHostStages], pstatus[kHostStages];
    /* one frame per call: a device block [error word 4 | pad 12 | posterior 4n
     * | hard n | status 4] and its pinned host image, so a call is one copy in
     * (which also clears the error word), one launch and one copy out, none of
     * them through pageable memory */
    DevBuf one;
    unsigned char* one_host = nullptr;
};

struct wldpc_encoder {
    int rate, z;
    CodeDesc code;
    cudaStream_t stream = nullptr;
    DevBuf info, cw;
    /* one frame per call: a device block [info k | codeword n] and its pinned
     * host image, so a call is one copy each way through pinned memory */
    DevBuf one;
    unsigned char* one_host = nullptr;
};

struct wldpc_ber_runner {
    wldpc_encoder* enc = nullptr;
    wldpc_decoder* dec = nullptr;
    uint64_t num_bits = 0, num_errors = 0;
    unsigned codeword_len = 0, dataword_len = 0;
    float float_rate = 0.f;
    uint32_t lfsr = 0xdeadbeefu, lfsr_start = 0xdeadbeefu;
    unsigned lfsr_index = 0, lfsr_reset_len = 1152 * 100;
    std::mt19937 gen{0};
    std::normal_distribution<float> dist{0.0f, 1.0f};
};

extern "C" {

const char* wldpc_strerror(int code)
{
    switch (code) {
    case WLDPC_OK: return "ok";
    case WLDPC_ERR_ARG: return "invalid argument";
    case WLDPC_ERR_CODE: return "invalid code rate or z factor";
    case WLDPC_ERR_CUDA: return "CUDA error";
    case WLDPC_ERR_NO_DEVICE: return "no CUDA device";
    case WLDPC_ERR_TIMEOUT: return "device-side wait timed out";
    case WLDPC_ERR_UNSUPPORTED: return "operation not supported for this code";
    case WLDPC_ERR_SCRATCH: return "request exceeds the static scratch of the allocation-free entry point";
    default: return "unknown error";
    }
}

int wldpc_version(void) { return 10200; }   /* 1.2.0: hard-decision host decodes, wait-limit hook */

int wldpc_code_info_get(int rate, unsigned z, wldpc_code_info* out)
{
    if (!out) return WLDPC_ERR_ARG;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    const CodeDesc c = make_code_desc(rate, (int)z);
    out->rate = rate;
    out->z = (int)z;
    out->n = c.n;
    out->m = c.m;
    out->k = c.k;
    out->rows = c.m;
    out->cols = max_degree(rate);
    out->D = c.D;
    out->X = c.X;
    out->layers = c.mb;
    out->edges = c.nblk * c.z;
    return WLDPC_OK;
}

int wldpc_checknode_table(int rate, unsigned z, int16_t* out, size_t capacity)
{
    if (!out) return WLDPC_ERR_ARG;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    const CodeDesc c = make_code_desc(rate, (int)z);
    const int cols = max_degree(rate);
    if (capacity < (size_t)c.m * cols) return WLDPC_ERR_ARG;
    for (int i = 0; i < c.mb; i++)
        for (int r = 0; r < c.z; r++) {
            int16_t* row = out + (size_t)(i * c.z + r) * cols;
            int e = 0;
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) {
                int t = r + c.shift[b];
                t = t >= c.z ? t - c.z : t;
                row[e++] = (int16_t)(c.col[b] * c.z + t);
            }
            for (; e < cols; e++) row[e] = -1;
        }
    return WLDPC_OK;
}

/* ------------------------------------------------------------- decoder */

int wldpc_decoder_create(int rate, unsigned z, unsigned max_iter, unsigned num_threads, int mode,
                         wldpc_decoder** out)
{
    (void)num_threads;
    if (!out) return WLDPC_ERR_ARG;
    *out = nullptr;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (mode < WLDPC_MODE_NMS || mode > WLDPC_MODE_MS || max_iter > 0xffff) return WLDPC_ERR_ARG;
    int rc = check_device();
    if (rc) return rc;
    wldpc_decoder* d = new (std::nothrow) wldpc_decoder();
    if (!d) return WLDPC_ERR_ARG;
    d->rate = rate;
    d->z = (int)z;
    d->mode = mode;
    d->max_iter = max_iter;
    d->code = make_code_desc(rate, (int)z);
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d->err, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(d->err, 0, sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        wldpc_decoder_destroy(d);
        return WLDPC_ERR_CUDA;
    }
    *out = d;
    return WLDPC_OK;
}

int wldpc_decoder_destroy(wldpc_decoder* d)
{
    if (!d) return WLDPC_ERR_ARG;
    if (d->stream) cudaStreamSynchronize(d->stream);
    for (auto& s : d->pipe)
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    if (d->stream) cudaStreamDestroy(d->stream);
    if (d->err) cudaFree(d->err);
    if (d->one_host) cudaFreeHost(d->one_host);
    delete d;
    return WLDPC_OK;
}

static int decode_launch(wldpc_decoder* d, const float* llr, int8_t* hard, float* post, int32_t* status,
                         size_t frames, cudaStream_t st, unsigned* err = nullptr)
{
    DecodeArgs a;
    a.llr = llr;
    a.hard = hard;
    a.post = post;
    a.status = status;
    a.err = err ? err : d->err;
    a.frames = (long long)frames;
    a.max_iter = (int)d->max_iter;
    a.wait_limit_us = d->wait_limit_us;
    return launch_tdmp(d->rate, d->z, d->mode, a, st) == cudaSuccess ? WLDPC_OK : WLDPC_ERR_CUDA;
}

static int read_err(wldpc_decoder* d)
{
    unsigned e = 0;
    CU(cudaMemcpy(&e, d->err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) {
        CU(cudaMemset(d->err, 0, sizeof(unsigned)));
        return WLDPC_ERR_TIMEOUT;
    }
    return WLDPC_OK;
}

int wldpc_decode_batch_device(wldpc_decoder* d, const float* llr, int8_t* decoded, float* posterior,
                              int32_t* status, size_t frames, void* stream)
{
    if (!d || (frames && (!llr || !decoded))) return WLDPC_ERR_ARG;
    if (!aligned(llr, 16) || !aligned(decoded, 4) || !aligned(posterior, 16) || !aligned(status, 4))
        return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    return decode_launch(d, llr, decoded, posterior, status, frames, (cudaStream_t)stream);
}

static_assert(kWaitLimitUs == WLDPC_WAIT_LIMIT_DEFAULT_US, "the header's default wait limit is the kernels'");

int wldpc_decoder_set_wait_limit(wldpc_decoder* d, unsigned limit_us)
{
    if (!d) return WLDPC_ERR_ARG;
    d->wait_limit_us = limit_us;
    return WLDPC_OK;
}

int wldpc_wait_bound_ns(unsigned limit_us, uint64_t* elapsed_ns)
{
    if (!elapsed_ns || limit_us > 10u * kWaitLimitUs) return WLDPC_ERR_ARG;
    int rc = check_device();
    if (rc) return rc;
    DevBuf out;
    if ((rc = out.reserve(2 * sizeof(unsigned long long)))) return rc;
    unsigned long long h[2] = {0, 0};
    CU(launch_wait_bound(limit_us, (unsigned long long*)out.p, 0));
    CU(cudaMemcpy(h, out.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (h[1]) return WLDPC_ERR_CUDA;   /* a barrier nobody completes cannot have completed */
    *elapsed_ns = h[0];
    return WLDPC_OK;
}

int wldpc_decoder_synchronize(wldpc_decoder* d)
{
    if (!d) return WLDPC_ERR_ARG;
    CU(cudaDeviceSynchronize());
    return read_err(d);
}

/* One frame (the reference's per-frame decode(float*)): the caller's buffers
 * are usually pageable, so the frame goes through the decoder's pinned block
 * by host memcpy and crosses PCIe in one copy each way. The block starts with
 * the launch's own error word, which the copy in clears, so the copy out
 * brings it back with the results. */
static int decode_one_host(wldpc_decoder* d, float* rx, int8_t* decoded, int32_t* status_host)
{
    const size_t n = (size_t)d->code.n;
    const size_t head = 16;                 /* error word + pad: the posterior stays 16-byte aligned */
    const size_t block = head + 5 * n + 4;  /* 4n and 5n are multiples of 16 (n = 24 z, z a multiple of 4) */
    int rc;
    if ((rc = d->one.reserve(block))) return rc;
    if (!d->one_host) {
        void* h = nullptr;
        if (cudaHostAlloc(&h, block, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return WLDPC_ERR_CUDA;
        }
        d->one_host = (unsigned char*)h;
    }
    unsigned char* dev = (unsigned char*)d->one.p;
    unsigned char* host = d->one_host;
    memset(host, 0, head);
    memcpy(host + head, rx, n * 4);
    CU(cudaMemcpyAsync(dev, host, head + n * 4, cudaMemcpyHostToDevice, d->stream));
    unsigned char* dp = dev + head;
    if ((rc = decode_launch(d, (const float*)dp, (int8_t*)(dp + 4 * n), (float*)dp, (int32_t*)(dp + 5 * n), 1,
                            d->stream, (unsigned*)dev))) {
        cudaStreamSynchronize(d->stream);
        return rc;
    }
    if (cudaMemcpyAsync(host, dev, block, cudaMemcpyDeviceToHost, d->stream) != cudaSuccess) {
        cudaStreamSynchronize(d->stream);
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    CU(cudaStreamSynchronize(d->stream));
    unsigned errword = 0;
    memcpy(&errword, host, 4);
    if (errword) return WLDPC_ERR_TIMEOUT;
    const unsigned char* hp = host + head;
    memcpy(rx, hp, n * 4);
    memcpy(decoded, hp + 4 * n, n);
    memcpy(status_host, hp + 5 * n, 4);
    return WLDPC_OK;
}

static unsigned ref_return(const wldpc_decoder* d, int32_t status)
{
    return d->max_iter == 0 ? 0u : (unsigned)((status >> 16) & 1);
}

int wldpc_decoder_decode(wldpc_decoder* d, float* rx_codeword, int8_t* decoded, unsigned* num_errors,
                         int* iterations)
{
    if (!d || !rx_codeword || !decoded) return WLDPC_ERR_ARG;
    int32_t st = 0;
    int rc = decode_one_host(d, rx_codeword, decoded, &st);
    if (rc) return rc;
    if (num_errors) *num_errors = ref_return(d, st);
    if (iterations) *iterations = st & 0xffff;
    return WLDPC_OK;
}

int wldpc_decoder_decode_bits(wldpc_decoder* d, const int8_t* rx_codeword, int8_t* decoded,
                              unsigned* num_errors)
{
    if (!d || !rx_codeword || !decoded) return WLDPC_ERR_ARG;
    const size_t n = (size_t)d->code.n;
    int rc;
    if ((rc = d->llr.reserve(n * 4)) || (rc = d->hard.reserve(n)) || (rc = d->status.reserve(4)) ||
        (rc = d->bits.reserve(n)))
        return rc;
    CU(cudaMemcpyAsync(d->bits.p, rx_codeword, n, cudaMemcpyHostToDevice, d->stream));
    CU(launch_bits_to_llr((const int8_t*)d->bits.p, (float*)d->llr.p, (long long)n, d->stream));
    if ((rc = decode_launch(d, (const float*)d->llr.p, (int8_t*)d->hard.p, nullptr, (int32_t*)d->status.p, 1,
                            d->stream)))
        return rc;
    int32_t st = 0;
    CU(cudaMemcpyAsync(decoded, d->hard.p, n, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaMemcpyAsync(&st, d->status.p, 4, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaStreamSynchronize(d->stream));
    if ((rc = read_err(d))) return rc;
    if (num_errors) *num_errors = ref_return(d, st);
    return WLDPC_OK;
}

int wldpc_decoder_compute_syndrome(wldpc_decoder* d, const int8_t* rx_codeword, int exit_early,
                                   unsigned* num_errors)
{
    if (!d || !rx_codeword || !num_errors) return WLDPC_ERR_ARG;
    const size_t n = (size_t)d->code.n;
    int rc;
    if ((rc = d->bits.reserve(n)) || (rc = d->status.reserve(4))) return rc;
    CU(cudaMemcpyAsync(d->bits.p, rx_codeword, n, cudaMemcpyHostToDevice, d->stream));
    CU(launch_syndrome(d->code, (const int8_t*)d->bits.p, (uint32_t*)d->status.p, 1, exit_early, d->stream));
    uint32_t v = 0;
    CU(cudaMemcpyAsync(&v, d->status.p, 4, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaStreamSynchronize(d->stream));
    *num_errors = v;
    return WLDPC_OK;
}

/* Batched forms of decode(int8_t*) and compute_syndrome over host buffers. */
int wldpc_decode_bits_batch_host(wldpc_decoder* d, const int8_t* bits, int8_t* decoded, uint32_t* num_errors,
                                 size_t frames)
{
    if (!d || (frames && (!bits || !decoded))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    const size_t n = (size_t)d->code.n;
    int rc;
    if ((rc = d->bits.reserve(frames * n)) || (rc = d->llr.reserve(frames * n * 4)) ||
        (rc = d->hard.reserve(frames * n)) || (rc = d->status.reserve(frames * 4)))
        return rc;
    CU(cudaMemcpyAsync(d->bits.p, bits, frames * n, cudaMemcpyHostToDevice, d->stream));
    CU(launch_bits_to_llr((const int8_t*)d->bits.p, (float*)d->llr.p, (long long)(frames * n), d->stream));
    if ((rc = decode_launch(d, (const float*)d->llr.p, (int8_t*)d->hard.p, nullptr, (int32_t*)d->status.p, frames,
                            d->stream)))
        return rc;
    std::vector<int32_t> st(frames);
    CU(cudaMemcpyAsync(decoded, d->hard.p, frames * n, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaMemcpyAsync(st.data(), d->status.p, frames * 4, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaStreamSynchronize(d->stream));
    if ((rc = read_err(d))) return rc;
    if (num_errors)
        for (size_t f = 0; f < frames; f++) num_errors[f] = ref_return(d, st[f]);
    return WLDPC_OK;
}

int wldpc_syndrome_batch_host(wldpc_decoder* d, const int8_t* bits, int exit_early, uint32_t* counts, size_t frames)
{
    if (!d || (frames && (!bits || !counts))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    const size_t n = (size_t)d->code.n;
    int rc;
    if ((rc = d->bits.reserve(frames * n)) || (rc = d->status.reserve(frames * 4))) return rc;
    CU(cudaMemcpyAsync(d->bits.p, bits, frames * n, cudaMemcpyHostToDevice, d->stream));
    CU(launch_syndrome(d->code, (const int8_t*)d->bits.p, (uint32_t*)d->status.p, (long long)frames, exit_early,
                       d->stream));
    CU(cudaMemcpyAsync(counts, d->status.p, frames * 4, cudaMemcpyDeviceToHost, d->stream));
    CU(cudaStreamSynchronize(d->stream));
    return WLDPC_OK;
}

/* Host batch: chunks of kHostChunk frames rotate over kHostStages streams so
 * that the copy-in of one chunk, the kernel of another and the copy-out of a
 * third overlap. post (nullable) receives the posterior; it may alias rx. */
static int decode_host_pipeline(wldpc_decoder* d, const float* rx, float* post, int8_t* decoded,
                                uint32_t* num_errors, int32_t* status, size_t frames)
{
    if (!d || (frames && (!rx || !decoded))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    const size_t n = (size_t)d->code.n;
    const size_t chunk = frames < kHostChunk ? frames : kHostChunk;
    int rc;
    for (int s = 0; s < kHostStages; s++) {
        if (!d->pipe[s]) CU(cudaStreamCreateWithFlags(&d->pipe[s], cudaStreamNonBlocking));
        if ((rc = d->pllr[s].reserve(chunk * n * 4)) || (rc = d->phard[s].reserve(chunk * n)) ||
            (rc = d->pstatus[s].reserve(chunk * 4)))
            return rc;
    }
    std::vector<int32_t> st_local;
    int32_t* st_host = status;
    if (!st_host && num_errors) {
        st_local.resize(frames);
        st_host = st_local.data();
    }
    size_t idx = 0;
    for (size_t f0 = 0; f0 < frames; f0 += chunk, idx++) {
        const int s = (int)(idx % kHostStages);
        const size_t nf = frames - f0 < chunk ? frames - f0 : chunk;
        cudaStream_t st = d->pipe[s];
        if (cudaMemcpyAsync(d->pllr[s].p, rx + f0 * n, nf * n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return drain_pipe(d->pipe, WLDPC_ERR_CUDA);
        if ((rc = decode_launch(d, (const float*)d->pllr[s].p, (int8_t*)d->phard[s].p,
                                post ? (float*)d->pllr[s].p : nullptr, (int32_t*)d->pstatus[s].p, nf, st)))
            return drain_pipe(d->pipe, rc);
        if ((post &&
             cudaMemcpyAsync(post + f0 * n, d->pllr[s].p, nf * n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
            cudaMemcpyAsync(decoded + f0 * n, d->phard[s].p, nf * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            (st_host &&
             cudaMemcpyAsync(st_host + f0, d->pstatus[s].p, nf * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess))
            return drain_pipe(d->pipe, WLDPC_ERR_CUDA);
    }
    for (int s = 0; s < kHostStages; s++)
        if (cudaStreamSynchronize(d->pipe[s]) != cudaSuccess) return drain_pipe(d->pipe, WLDPC_ERR_CUDA);
    if ((rc = read_err(d))) return rc;
    if (num_errors)
        for (size_t f = 0; f < frames; f++) num_errors[f] = ref_return(d, st_host[f]);
    return WLDPC_OK;
}

int wldpc_decode_batch_host(wldpc_decoder* d, float* rx, int8_t* decoded, uint32_t* num_errors,
                            int32_t* status, size_t frames)
{
    return decode_host_pipeline(d, rx, rx, decoded, num_errors, status, frames);
}

int wldpc_decode_batch_host_hard(wldpc_decoder* d, const float* llr, int8_t* decoded, uint32_t* num_errors,
                                 int32_t* status, size_t frames)
{
    return decode_host_pipeline(d, llr, nullptr, decoded, num_errors, status, frames);
}

/* ------------------------------------------------------------- encoder */

int wldpc_encoder_create(int rate, unsigned z, unsigned num_threads, wldpc_encoder** out)
{
    (void)num_threads;
    if (!out) return WLDPC_ERR_ARG;
    *out = nullptr;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    int rc = check_device();
    if (rc) return rc;
    wldpc_encoder* e = new (std::nothrow) wldpc_encoder();
    if (!e) return WLDPC_ERR_ARG;
    e->rate = rate;
    e->z = (int)z;
    e->code = make_code_desc(rate, (int)z);
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete e;
        return WLDPC_ERR_CUDA;
    }
    *out = e;
    return WLDPC_OK;
}

int wldpc_encoder_destroy(wldpc_encoder* e)
{
    if (!e) return WLDPC_ERR_ARG;
    if (e->stream) {
        cudaStreamSynchronize(e->stream);
        cudaStreamDestroy(e->stream);
    }
    if (e->one_host) cudaFreeHost(e->one_host);
    delete e;
    return WLDPC_OK;
}

int wldpc_encode_batch_host(wldpc_encoder* e, const uint8_t* info, uint8_t* codeword, size_t frames)
{
    if (!e || (frames && (!info || !codeword))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    int rc;
    if ((rc = e->info.reserve(frames * e->code.k)) || (rc = e->cw.reserve(frames * e->code.n))) return rc;
    CU(cudaMemcpyAsync(e->info.p, info, frames * e->code.k, cudaMemcpyHostToDevice, e->stream));
    CU(launch_encode_bytes(e->code, (const uint8_t*)e->info.p, (uint8_t*)e->cw.p, (long long)frames, e->stream));
    CU(cudaMemcpyAsync(codeword, e->cw.p, frames * e->code.n, cudaMemcpyDeviceToHost, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return WLDPC_OK;
}

int wldpc_encode_batch_device(wldpc_encoder* e, const uint8_t* info, uint8_t* codeword, size_t frames,
                              void* stream)
{
    if (!e || (frames && (!info || !codeword))) return WLDPC_ERR_ARG;
    if (!aligned(info, 4) || !aligned(codeword, 4)) return WLDPC_ERR_ARG;
    CU(launch_encode_bytes(e->code, info, codeword, (long long)frames, (cudaStream_t)stream));
    return WLDPC_OK;
}

int wldpc_encoder_encode(wldpc_encoder* e, const uint8_t* infoword, uint8_t* codeword)
{
    if (!e || !infoword || !codeword) return WLDPC_ERR_ARG;
    const size_t k = (size_t)e->code.k, n = (size_t)e->code.n;   /* k and n are multiples of 4 */
    int rc;
    if ((rc = e->one.reserve(k + n))) return rc;
    if (!e->one_host) {
        void* h = nullptr;
        if (cudaHostAlloc(&h, k + n, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return WLDPC_ERR_CUDA;
        }
        e->one_host = (unsigned char*)h;
    }
    unsigned char* dev = (unsigned char*)e->one.p;
    memcpy(e->one_host, infoword, k);
    CU(cudaMemcpyAsync(dev, e->one_host, k, cudaMemcpyHostToDevice, e->stream));
    if (launch_encode_bytes(e->code, dev, dev + k, 1, e->stream) != cudaSuccess ||
        cudaMemcpyAsync(e->one_host + k, dev + k, n, cudaMemcpyDeviceToHost, e->stream) != cudaSuccess) {
        cudaStreamSynchronize(e->stream);
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    CU(cudaStreamSynchronize(e->stream));
    memcpy(codeword, e->one_host + k, n);
    return WLDPC_OK;
}

/* ----------------------------------------------------------- framegen */

int wldpc_framegen_device(int rate, unsigned z, uint64_t seed, uint64_t first_frame, size_t frames,
                          float ebno_lo_db, float ebno_hi_db, uint8_t* info, uint8_t* codeword, float* llr,
                          float* ebno_db, void* stream)
{
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (rate == THREEQUARTERSB) return WLDPC_ERR_UNSUPPORTED;
    if (!aligned(info, 4) || !aligned(codeword, 4) || !aligned(llr, 16) || !aligned(ebno_db, 4))
        return WLDPC_ERR_ARG;
    int rc = check_device();
    if (rc) return rc;
    FramegenArgs a;
    a.seed = seed;
    a.first_frame = first_frame;
    a.frames = (long long)frames;
    a.ebno_lo = ebno_lo_db;
    a.ebno_hi = ebno_hi_db;
    a.info = info;
    a.cw = codeword;
    a.llr = llr;
    a.ebno_out = ebno_db;
    CU(launch_framegen(make_code_desc(rate, (int)z), a, (cudaStream_t)stream));
    return WLDPC_OK;
}

/* --------------------------------------------- null-space frame generator */

namespace {

/* H in reduced row-echelon form over GF(2): pivot columns, free columns and
 * the pivot rows restricted to the free columns, packed; on the device. */
struct Nullspace {
    DevBuf A, piv, fre;
    int rank = 0, nfree = 0, words = 0;
};

std::mutex g_ns_mutex;
std::map<int, Nullspace*> g_ns;

int nullspace_for(int rate, int z, Nullspace** out)
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    const int key = (dev * kRates + rate) * 128 + z;
    std::lock_guard<std::mutex> lock(g_ns_mutex);
    auto it = g_ns.find(key);
    if (it != g_ns.end()) {
        *out = it->second;
        return WLDPC_OK;
    }
    const CodeDesc c = make_code_desc(rate, z);
    const int n = c.n, m = c.m, W = (n + 31) / 32;
    std::vector<uint32_t> H((size_t)m * W, 0u);
    for (int i = 0; i < c.mb; i++)
        for (int r = 0; r < z; r++)
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) {
                int t = r + c.shift[b];
                t = t >= z ? t - z : t;
                const int v = c.col[b] * z + t;
                H[(size_t)(i * z + r) * W + (v >> 5)] ^= 1u << (v & 31);
            }
    std::vector<int> pivots;
    std::vector<char> is_pivot(n, 0);
    int pr = 0;
    for (int col = 0; col < n && pr < m; col++) {
        int sel = -1;
        for (int r = pr; r < m; r++)
            if ((H[(size_t)r * W + (col >> 5)] >> (col & 31)) & 1u) { sel = r; break; }
        if (sel < 0) continue;
        if (sel != pr)
            for (int q = 0; q < W; q++) std::swap(H[(size_t)sel * W + q], H[(size_t)pr * W + q]);
        for (int r = 0; r < m; r++)
            if (r != pr && ((H[(size_t)r * W + (col >> 5)] >> (col & 31)) & 1u))
                for (int q = 0; q < W; q++) H[(size_t)r * W + q] ^= H[(size_t)pr * W + q];
        pivots.push_back(col);
        is_pivot[col] = 1;
        pr++;
    }
    std::vector<unsigned short> fre;
    for (int col = 0; col < n; col++)
        if (!is_pivot[col]) fre.push_back((unsigned short)col);
    Nullspace* ns = new Nullspace();
    ns->rank = pr;
    ns->nfree = (int)fre.size();
    ns->words = (ns->nfree + 31) / 32;
    std::vector<uint32_t> A((size_t)pr * ns->words, 0u);
    for (int i = 0; i < pr; i++)
        for (int j = 0; j < ns->nfree; j++)
            if ((H[(size_t)i * W + (fre[j] >> 5)] >> (fre[j] & 31)) & 1u) A[(size_t)i * ns->words + (j >> 5)] |= 1u << (j & 31);
    std::vector<unsigned short> piv(pivots.begin(), pivots.end());
    if (ns->A.reserve(A.size() * 4 + 4) || ns->piv.reserve(piv.size() * 2 + 2) || ns->fre.reserve(fre.size() * 2 + 2) ||
        cudaMemcpy(ns->A.p, A.data(), A.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ns->piv.p, piv.data(), piv.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ns->fre.p, fre.data(), fre.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        delete ns;
        return WLDPC_ERR_CUDA;
    }
    g_ns[key] = ns;
    *out = ns;
    return WLDPC_OK;
}

}  // namespace

/* null-space frame generation for other parts of the library (learned
 * training); internal, C linkage because it sits in this file's extern "C" block */
int wldpc_internal_nullspace_frames(int rate, int z, const FramegenArgs& a, cudaStream_t st)
{
    Nullspace* ns = nullptr;
    int rc = nullspace_for(rate, z, &ns);
    if (rc) return rc;
    NullspaceArgs na;
    na.A = (const uint32_t*)ns->A.p;
    na.pivot_col = (const unsigned short*)ns->piv.p;
    na.free_col = (const unsigned short*)ns->fre.p;
    na.rank = ns->rank;
    na.nfree = ns->nfree;
    na.words = ns->words;
    return launch_framegen_nullspace(make_code_desc(rate, z), a, na, st) == cudaSuccess ? WLDPC_OK : WLDPC_ERR_CUDA;
}

int wldpc_framegen_nullspace_device(int rate, unsigned z, uint64_t seed, uint64_t first_frame, size_t frames,
                                    float ebno_lo_db, float ebno_hi_db, uint8_t* codeword, float* llr, float* ebno_db,
                                    void* stream)
{
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (!aligned(codeword, 4) || !aligned(llr, 16) || !aligned(ebno_db, 4)) return WLDPC_ERR_ARG;
    int rc = check_device();
    if (rc) return rc;
    Nullspace* ns = nullptr;
    if ((rc = nullspace_for(rate, (int)z, &ns))) return rc;
    FramegenArgs a;
    a.seed = seed;
    a.first_frame = first_frame;
    a.frames = (long long)frames;
    a.ebno_lo = ebno_lo_db;
    a.ebno_hi = ebno_hi_db;
    a.info = nullptr;
    a.cw = codeword;
    a.llr = llr;
    a.ebno_out = ebno_db;
    NullspaceArgs na;
    na.A = (const uint32_t*)ns->A.p;
    na.pivot_col = (const unsigned short*)ns->piv.p;
    na.free_col = (const unsigned short*)ns->fre.p;
    na.rank = ns->rank;
    na.nfree = ns->nfree;
    na.words = ns->words;
    CU(launch_framegen_nullspace(make_code_desc(rate, (int)z), a, na, (cudaStream_t)stream));
    return WLDPC_OK;
}

/* ------------------------------------------------------- LFSR info bits */

int wldpc_lfsr_bits_device(uint64_t first_bit, size_t nbits, uint8_t* out, void* stream)
{
    if (nbits && !out) return WLDPC_ERR_ARG;
    int rc = check_device();
    if (rc) return rc;
    static bool uploaded[64] = {false};   /* per device: the period table is in place */
    static std::mutex upload_mutex;
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return WLDPC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(upload_mutex);
    if (!uploaded[dev]) {
        /* one period of the stream, as BER_runner::lfsr_get_num produces it */
        std::vector<uint32_t> words(115200 / 32, 0u);
        uint32_t s = 0xdeadbeefu;
        for (unsigned i = 0; i < 115200; i++) {
            const uint32_t bit = (s ^ (s >> 3)) & 1u;
            s = (s >> 1) | (bit << 30);
            words[i >> 5] |= bit << (i & 31);
        }
        CU(upload_lfsr_period(words.data()));
        uploaded[dev] = true;
    }
    CU(launch_lfsr_bits((unsigned long long)first_bit, (long long)nbits, out, (cudaStream_t)stream));
    return WLDPC_OK;
}

/* ---------------------------------------------------------- BER runner */

int wldpc_ber_runner_create(int rate, unsigned z, unsigned num_threads, unsigned max_iter,
                            wldpc_ber_runner** out)
{
    if (!out) return WLDPC_ERR_ARG;
    *out = nullptr;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (rate == THREEQUARTERSB) return WLDPC_ERR_UNSUPPORTED;   /* reference lib/BER_runner.cc:66-71 */
    wldpc_ber_runner* b = new (std::nothrow) wldpc_ber_runner();
    if (!b) return WLDPC_ERR_ARG;
    int rc = wldpc_encoder_create(rate, z, num_threads, &b->enc);
    if (!rc) rc = wldpc_decoder_create(rate, z, max_iter, num_threads, WLDPC_MODE_NMS, &b->dec);
    if (rc) {
        wldpc_ber_runner_destroy(b);
        return rc;
    }
    /* lengths and rate as the reference computes them (reference :30,43-77) */
    b->codeword_len = (unsigned)((z / 96.0) * 2304);
    static const float kRate[6] = {0.5f, (float)(2.0 / 3.0), (float)(2.0 / 3.0), (float)(3.0 / 4.0), 0.f,
                                   (float)(5.0 / 6.0)};
    static const unsigned kNum[6] = {1, 2, 2, 3, 0, 5}, kDen[6] = {2, 3, 3, 4, 1, 6};
    b->dataword_len = (b->codeword_len * kNum[rate]) / kDen[rate];
    b->float_rate = kRate[rate];
    *out = b;
    return WLDPC_OK;
}

int wldpc_ber_runner_destroy(wldpc_ber_runner* b)
{
    if (!b) return WLDPC_ERR_ARG;
    if (b->enc) wldpc_encoder_destroy(b->enc);
    if (b->dec) wldpc_decoder_destroy(b->dec);
    delete b;
    return WLDPC_OK;
}

int wldpc_ber_runner_run_iteration(wldpc_ber_runner* b, double ebno_db, double* ber)
{
    if (!b) return WLDPC_ERR_ARG;
    const unsigned n = b->codeword_len, k = b->dataword_len;
    std::vector<uint8_t> data(k), cw(n);
    std::vector<float> buf(n);
    std::vector<int8_t> dec(n);
    const double ebno_lin = pow(10.0, ebno_db / 10.0);
    const float amp = (float)((1.0 / std::sqrt(ebno_lin)) * std::sqrt(1.0 / (b->float_rate * 1)));
    /* info bits: LFSR x^31 + x^28 + 1, restarted every reset_len bits (reference :124-146) */
    for (unsigned i = 0; i < k; i++) {
        const uint32_t bit = ((b->lfsr >> 0) ^ (b->lfsr >> 3)) & 1u;
        b->lfsr = (b->lfsr >> 1) | (bit << 30);
        if (++b->lfsr_index == b->lfsr_reset_len) {
            b->lfsr = b->lfsr_start;
            b->lfsr_index = 0;
        }
        data[i] = (uint8_t)bit;
    }
    int rc = wldpc_encoder_encode(b->enc, data.data(), cw.data());
    if (rc) return rc;
    /* BPSK and the reference's noise stream, in its order and types (reference :181-191) */
    for (unsigned j = 0; j < n; j++) buf[j] = (float)(cw[j] * 2 - 1);
    for (unsigned j = 0; j < n; j++) buf[j] = buf[j] + std::sqrt(0.5) * amp * b->dist(b->gen);
    unsigned ne = 0;
    rc = wldpc_decoder_decode(b->dec, buf.data(), dec.data(), &ne, nullptr);
    if (rc) return rc;
    b->num_bits += k;
    unsigned errors = 0;   /* counted over all n codeword bits (reference :148-160) */
    for (unsigned j = 0; j < n; j++) errors += cw[j] != (uint8_t)dec[j];
    b->num_errors += errors;
    if (ber) *ber = (double)b->num_errors / (double)b->num_bits;
    return WLDPC_OK;
}

int wldpc_ber_runner_reset(wldpc_ber_runner* b)
{
    if (!b) return WLDPC_ERR_ARG;
    b->num_bits = 0;
    b->num_errors = 0;
    return WLDPC_OK;
}

int wldpc_ber_runner_totals(wldpc_ber_runner* b, uint64_t* num_bits, uint64_t* num_errors)
{
    if (!b) return WLDPC_ERR_ARG;
    if (num_bits) *num_bits = b->num_bits;
    if (num_errors) *num_errors = b->num_errors;
    return WLDPC_OK;
}

int wldpc_ber_runner_lengths(wldpc_ber_runner* b, unsigned* codeword_len, unsigned* dataword_len)
{
    if (!b) return WLDPC_ERR_ARG;
    if (codeword_len) *codeword_len = b->codeword_len;
    if (dataword_len) *dataword_len = b->dataword_len;
    return WLDPC_OK;
}

}  // extern "C"
