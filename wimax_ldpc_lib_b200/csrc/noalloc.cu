/*
 * wldpc_decode_host_noalloc: decode frames held in host memory without
 * allocating anything, for callers that cannot call cudaMalloc.
 *
 * Who those callers are: hosts whose device memory is owned and budgeted by
 * another allocator and that forbid libraries from taking device memory of
 * their own; real-time signal-processing threads, where cudaMalloc (which may
 * synchronise the device and take unbounded time) is not allowed on the
 * processing path; and short-lived plugin calls that cannot keep a decoder
 * handle (and its buffers) alive between calls.
 *
 * The device scratch this call needs (error word, per-frame status, LLR /
 * posterior and hard-bit staging) lives in g_noalloc_scratch, a file-scope
 * static __device__ array of WLDPC_NOALLOC_SCRATCH_BYTES (1 MiB). Every GPU
 * that loads the library holds it until the process exits. In host code the
 * array's name is only a host-side stand-in, so every call takes the device
 * address with cudaGetSymbolAddress (with the caller's device current; the
 * lookup allocates nothing). Looking it up on every call rather than caching
 * it keeps the address right after the caller resets the device or recreates
 * its primary context, which can move the array. The first call on a device
 * also loads the module there, so that first call should come before any
 * stream capture. Requests whose staging does not fit return
 * WLDPC_ERR_SCRATCH before touching the GPU. If a copy or the launch fails
 * after work was queued, the call waits for the queued copies to finish
 * before it returns, so nothing writes into the caller's buffers afterwards.
 *
 * Every call shares the one array and leaves the last call's contents in it;
 * the error word is cleared at the start of each call. Calls that overlap on
 * the GPU (for example from two host threads at once) race on the array and
 * must be serialised by the caller.
 */
#include <cstdint>
#include <cuda_runtime.h>

#include "wimax_ldpc_b200.h"
#include "codec_kernels.cuh"

using namespace wldpc;

static __device__ __align__(256) unsigned char g_noalloc_scratch[WLDPC_NOALLOC_SCRATCH_BYTES];

namespace {

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

/* device address of g_noalloc_scratch on the current device */
int scratch_address(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    *out = p;
    return WLDPC_OK;
}

/* error after work was queued on st: let the queued copies finish (their
 * result is not needed) so that none lands in the caller's buffers later */
int fail_after_enqueue(cudaStream_t st)
{
    cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaGetLastError();
    return WLDPC_ERR_CUDA;
}

}  // namespace

extern "C" WLDPC_API int wldpc_decode_host_noalloc(int rate, unsigned z, unsigned max_iter, float* rx_codewords,
                                                   int8_t* decoded, uint32_t* num_errors, size_t frames)
{
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (max_iter > 0xffff) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    if (!rx_codewords || !decoded) return WLDPC_ERR_ARG;
    const size_t n = (size_t)kNB * z;
    /* scratch layout: error word | status | LLR and posterior | hard bits */
    const size_t off_status = 256;
    const size_t off_llr = off_status + round256(frames * 4);
    const size_t off_hard = off_llr + round256(frames * n * 4);
    const size_t need = off_hard + round256(frames * n);
    if (frames > WLDPC_NOALLOC_SCRATCH_BYTES || need > WLDPC_NOALLOC_SCRATCH_BYTES) return WLDPC_ERR_SCRATCH;

    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices <= 0) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char* s = static_cast<unsigned char*>(base);
    unsigned* err = reinterpret_cast<unsigned*>(s);
    int32_t* status = reinterpret_cast<int32_t*>(s + off_status);
    float* llr = reinterpret_cast<float*>(s + off_llr);
    int8_t* hard = reinterpret_cast<int8_t*>(s + off_hard);
    const cudaStream_t st = 0;

    if (cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess ||
        cudaMemcpyAsync(llr, rx_codewords, frames * n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return fail_after_enqueue(st);
    DecodeArgs a;
    a.llr = llr;
    a.hard = hard;
    a.post = llr;
    a.status = status;
    a.err = err;
    a.frames = (long long)frames;
    a.max_iter = (int)max_iter;
    if (launch_tdmp(rate, (int)z, kNms, a, st) != cudaSuccess) return fail_after_enqueue(st);
    unsigned errword = 0;
    if (cudaMemcpyAsync(rx_codewords, llr, frames * n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(decoded, hard, frames * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        (num_errors &&
         cudaMemcpyAsync(num_errors, status, frames * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
        cudaMemcpyAsync(&errword, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail_after_enqueue(st);
    if (errword) return WLDPC_ERR_TIMEOUT;
    /* status words -> the reference's return values, in place */
    if (num_errors)
        for (size_t f = 0; f < frames; f++)
            num_errors[f] = max_iter == 0 ? 0u : ((num_errors[f] >> 16) & 1u);
    return WLDPC_OK;
}
