/*
 * C ABI of the learned min-sum decoder (include/wimax_ldpc_b200.h,
 * wldpc_lms_*): handle with its weights, inference, gradient and training.
 * The weight table the ABI exchanges is float[2][T][12][24]: scales a, then
 * offsets b, each [iteration][layer][base column]; entries of all-zero blocks
 * are ignored on input and returned as 0.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "wimax_ldpc_b200.h"
#include "codec_kernels.cuh"
#include "lms_dispatch.cuh"

using namespace wldpc;

extern "C" int wldpc_internal_nullspace_frames(int rate, int z, const wldpc::FramegenArgs& a, cudaStream_t st);

namespace wldpc {
/* dispatch rows defined by the 12 compilations of lms_instances.cuh */
#define WLDPC_LMS_HALVES(R)                             \
    extern const LmsLaunch kLms_r##R##_h0[kLmsHalf0]; \
    extern const LmsLaunch kLms_r##R##_h1[kNumZ - kLmsHalf0];
WLDPC_LMS_HALVES(0)
WLDPC_LMS_HALVES(1)
WLDPC_LMS_HALVES(2)
WLDPC_LMS_HALVES(3)
WLDPC_LMS_HALVES(4)
WLDPC_LMS_HALVES(5)
#undef WLDPC_LMS_HALVES

/* Column sums of the per-frame gradients in frame order (deterministic),
 * the batch loss, then Adam; one thread per weight. */
__global__ void lms_reduce_adam_kernel(const __grid_constant__ AdamArgs a)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0 && a.loss_out) {
        float s = 0.0f;
        for (long long f = 0; f < a.frames; f++) s += a.loss_part[f];
        *a.loss_out = s;
    }
    if (j >= a.nw) return;
    float g = 0.0f;
    for (long long f = 0; f < a.frames; f++) g += a.gpart[f * a.nw + j];
    a.grad[j] = g;
    if (!a.apply) return;
    const float m = a.beta1 * a.m[j] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * a.v[j] + (1.0f - a.beta2) * g * g;
    a.m[j] = m;
    a.v[j] = v;
    const float mh = m / (1.0f - powf(a.beta1, (float)a.step));
    const float vh = v / (1.0f - powf(a.beta2, (float)a.step));
    a.w[j] -= a.lr * mh / (sqrtf(vh) + a.eps);
}

const LmsLaunch* lms_entry(int rate, int z)
{
    static const LmsLaunch* const t[kRates][2] = {{kLms_r0_h0, kLms_r0_h1}, {kLms_r1_h0, kLms_r1_h1},
                                                  {kLms_r2_h0, kLms_r2_h1}, {kLms_r3_h0, kLms_r3_h1},
                                                  {kLms_r4_h0, kLms_r4_h1}, {kLms_r5_h0, kLms_r5_h1}};
    if (!valid_rate(rate) || !valid_z(z)) return nullptr;
    const int zi = z_index(z);
    const LmsLaunch* e = zi < kLmsHalf0 ? &t[rate][0][zi] : &t[rate][1][zi - kLmsHalf0];
    return e->z == z ? e : nullptr;
}
}  // namespace wldpc

namespace {

#define CU(call)                     \
    do {                             \
        if ((call) != cudaSuccess) { \
            cudaGetLastError();      \
            return WLDPC_ERR_CUDA;   \
        }                            \
    } while (0)

struct Buf {
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
    ~Buf()
    {
        if (p) cudaFree(p);
    }
};

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace

struct wldpc_lms {
    int rate, z, T, nblk;
    int cap;                 /* decoding iteration cap (>= 1); iterations past T reuse row T-1 */
    int precision = WLDPC_LMS_F32;   /* inference arithmetic (training is always fp32) */
    CodeDesc code;
    const LmsLaunch* k;
    LmsWeights w;            /* host copy, compact [T][nblk], used by inference launches */
    bool host_stale = false; /* device weights changed by training */
    cudaStream_t stream = nullptr;
    unsigned* err = nullptr;
    Buf wdev, mdev, vdev, grad, loss;                  /* training state: [2][T][nblk] */
    Buf ckp, ckm, gpart, lpart, tllr, tcw;             /* training scratch */
    Buf pllr[kHostStages], phard[kHostStages], pstat[kHostStages];                   /* host-batch pipeline staging */
    cudaStream_t pipe[kHostStages] = {};
    cudaEvent_t ev_user = nullptr;                     /* orders the handle's stream after a caller's */
    int adam_step = 0;
};

static int lms_sync_host_weights(wldpc_lms* h)
{
    if (!h->host_stale) return WLDPC_OK;
    std::vector<float> buf((size_t)2 * h->T * h->nblk);
    CU(cudaMemcpy(buf.data(), h->wdev.p, buf.size() * 4, cudaMemcpyDeviceToHost));
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++) {
            h->w.a[t][b] = buf[(size_t)t * h->nblk + b];
            h->w.b[t][b] = buf[(size_t)(h->T + t) * h->nblk + b];
        }
    h->host_stale = false;
    return WLDPC_OK;
}

static int lms_push_device_weights(wldpc_lms* h)
{
    std::vector<float> buf((size_t)2 * h->T * h->nblk);
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++) {
            buf[(size_t)t * h->nblk + b] = h->w.a[t][b];
            buf[(size_t)(h->T + t) * h->nblk + b] = h->w.b[t][b];
        }
    CU(cudaMemcpy(h->wdev.p, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice));
    return WLDPC_OK;
}

extern "C" {

int wldpc_lms_create(int rate, unsigned z, unsigned iterations, wldpc_lms** out)
{
    if (!out) return WLDPC_ERR_ARG;
    *out = nullptr;
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    if (iterations < 1 || iterations > (unsigned)kLmsMaxIter) return WLDPC_ERR_ARG;
    const LmsLaunch* k = lms_entry(rate, (int)z);
    if (!k) return WLDPC_ERR_UNSUPPORTED;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    wldpc_lms* h = new (std::nothrow) wldpc_lms();
    if (!h) return WLDPC_ERR_ARG;
    h->rate = rate;
    h->z = (int)z;
    h->T = (int)iterations;
    h->cap = (int)iterations;
    h->code = make_code_desc(rate, (int)z);
    h->nblk = h->code.nblk;
    h->k = k;
    memset(&h->w, 0, sizeof(h->w));
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++) h->w.a[t][b] = 0.815f;   /* start as normalized min-sum */
    const size_t nw = (size_t)2 * h->T * h->nblk;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->err, sizeof(unsigned)) != cudaSuccess || cudaMemset(h->err, 0, 4) != cudaSuccess ||
        h->wdev.reserve(nw * 4) || h->mdev.reserve(nw * 4) || h->vdev.reserve(nw * 4) ||
        h->grad.reserve(nw * 4) || cudaMemset(h->mdev.p, 0, nw * 4) != cudaSuccess ||
        cudaMemset(h->vdev.p, 0, nw * 4) != cudaSuccess || lms_push_device_weights(h)) {
        cudaGetLastError();
        wldpc_lms_destroy(h);
        return WLDPC_ERR_CUDA;
    }
    *out = h;
    return WLDPC_OK;
}

int wldpc_lms_destroy(wldpc_lms* h)
{
    if (!h) return WLDPC_ERR_ARG;
    if (h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
    }
    for (auto& ps : h->pipe)
        if (ps) {
            cudaStreamSynchronize(ps);
            cudaStreamDestroy(ps);
        }
    if (h->err) cudaFree(h->err);
    if (h->ev_user) cudaEventDestroy(h->ev_user);
    delete h;
    return WLDPC_OK;
}

int wldpc_lms_set_weights(wldpc_lms* h, const float* table)
{
    if (!h || !table) return WLDPC_ERR_ARG;
    const CodeDesc& c = h->code;
    for (int t = 0; t < h->T; t++)
        for (int i = 0; i < c.mb; i++)
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) {
                const size_t o = ((size_t)t * kMaxMb + i) * kNB + c.col[b];
                h->w.a[t][b] = table[o];
                h->w.b[t][b] = table[(size_t)h->T * kMaxMb * kNB + o];
            }
    h->host_stale = false;
    h->adam_step = 0;
    const size_t nw = (size_t)2 * h->T * h->nblk;
    CU(cudaMemset(h->mdev.p, 0, nw * 4));
    CU(cudaMemset(h->vdev.p, 0, nw * 4));
    return lms_push_device_weights(h);
}

int wldpc_lms_get_weights(wldpc_lms* h, float* table)
{
    if (!h || !table) return WLDPC_ERR_ARG;
    int rc = lms_sync_host_weights(h);
    if (rc) return rc;
    const CodeDesc& c = h->code;
    memset(table, 0, sizeof(float) * 2 * h->T * kMaxMb * kNB);
    for (int t = 0; t < h->T; t++)
        for (int i = 0; i < c.mb; i++)
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) {
                const size_t o = ((size_t)t * kMaxMb + i) * kNB + c.col[b];
                table[o] = h->w.a[t][b];
                table[(size_t)h->T * kMaxMb * kNB + o] = h->w.b[t][b];
            }
    return WLDPC_OK;
}

/* the packed-half decoder accepts |a| <= 2 and 0 <= b <= 1024: the bounds keep
 * every binary16 sum of the decode finite, and b >= 0 is what lets a stopped
 * frame's lane produce zero messages (lms16.cuh) */
static bool lms16_weights_ok(const wldpc_lms* h)
{
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++)
            if (!(fabsf(h->w.a[t][b]) <= kLms16MaxScale) || !(h->w.b[t][b] >= 0.0f && h->w.b[t][b] <= kLms16MaxOffset))
                return false;
    return true;
}

static uint32_t half_pair_bits(float x)
{
    const __half v = __float2half_rn(x);
    const uint32_t u = __half_as_ushort(v);
    return u | (u << 16);
}

static int lms16_launch_decode(wldpc_lms* h, const float* llr, int8_t* hard, float* post, int32_t* status,
                               size_t frames, cudaStream_t st)
{
    if (!lms16_weights_ok(h)) return WLDPC_ERR_ARG;
    Lms16Args a;
    a.llr = llr;
    a.hard = hard;
    a.post = post;
    a.status = status;
    a.frames = (long long)frames;
    a.iters = h->cap;
    a.wrows = h->T;
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++)
            a.wab[t][b] = make_uint2(half_pair_bits(h->w.a[t][b]), half_pair_bits(-h->w.b[t][b]));
    const LmsLaunch* k = h->k;
    const long long ctas = ((long long)frames + k->frames16 - 1) / k->frames16;
    k->decode16<<<(unsigned)ctas, k->threads16, 0, st>>>(a);
    CU(cudaGetLastError());
    return WLDPC_OK;
}

static int lms_launch_decode(wldpc_lms* h, const float* llr, int8_t* hard, float* post, int32_t* status,
                             size_t frames, cudaStream_t st)
{
    int rc = lms_sync_host_weights(h);
    if (rc) return rc;
    if (h->precision == WLDPC_LMS_F16X2) return lms16_launch_decode(h, llr, hard, post, status, frames, st);
    LmsArgs a;
    a.llr = llr;
    a.hard = hard;
    a.post = post;
    a.status = status;
    a.err = h->err;
    a.frames = (long long)frames;
    a.iters = h->cap;
    a.wrows = h->T;
    for (int t = 0; t < h->T; t++)
        for (int b = 0; b < h->nblk; b++) a.wab[t][b] = make_float2(h->w.a[t][b], h->w.b[t][b]);
    const LmsLaunch* k = h->k;
    if (k->smem > 48 * 1024)
        CU(cudaFuncSetAttribute(k->decode, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem));
    const long long ctas = ((long long)frames + k->frames_per_cta - 1) / k->frames_per_cta;
    k->decode<<<(unsigned)ctas, k->threads, k->smem, st>>>(a);
    CU(cudaGetLastError());
    return WLDPC_OK;
}

int wldpc_lms_decode_device(wldpc_lms* h, const float* llr, int8_t* decoded, float* posterior, int32_t* status,
                            size_t frames, void* stream)
{
    if (!h || (frames && (!llr || !decoded))) return WLDPC_ERR_ARG;
    if (!aligned(llr, 16) || !aligned(decoded, 4) || !aligned(posterior, 16) || !aligned(status, 4))
        return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    return lms_launch_decode(h, llr, decoded, posterior, status, frames, (cudaStream_t)stream);
}

int wldpc_lms_set_precision(wldpc_lms* h, int precision)
{
    if (!h || (precision != WLDPC_LMS_F32 && precision != WLDPC_LMS_F16X2)) return WLDPC_ERR_ARG;
    if (precision == WLDPC_LMS_F16X2) {
        int rc = lms_sync_host_weights(h);
        if (rc) return rc;
        if (!lms16_weights_ok(h)) return WLDPC_ERR_ARG;
    }
    h->precision = precision;
    return WLDPC_OK;
}

int wldpc_lms_set_cap(wldpc_lms* h, unsigned cap)
{
    if (!h || cap < 1 || cap > 0xffff) return WLDPC_ERR_ARG;
    h->cap = (int)cap;
    return WLDPC_OK;
}

/* Host batch: chunks rotate over kHostStages streams so that copies and
 * kernels of neighbouring chunks overlap (as wldpc_decode_batch_host). post
 * (nullable) receives the posterior; it may alias rx. */
static int lms_decode_host_pipeline(wldpc_lms* h, const float* rx, float* post, int8_t* decoded,
                                    uint32_t* num_errors, int32_t* status, size_t frames)
{
    if (!h || (frames && (!rx || !decoded))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    const size_t n = (size_t)h->code.n;
    const size_t chunk = frames < kHostChunk ? frames : kHostChunk;
    int rc;
    for (int s = 0; s < kHostStages; s++) {
        if (!h->pipe[s]) CU(cudaStreamCreateWithFlags(&h->pipe[s], cudaStreamNonBlocking));
        if ((rc = h->pllr[s].reserve(chunk * n * 4)) || (rc = h->phard[s].reserve(chunk * n)) ||
            (rc = h->pstat[s].reserve(chunk * 4)))
            return rc;
    }
    std::vector<int32_t> st_local;
    int32_t* st = status;
    if (!st && num_errors) {
        st_local.resize(frames);
        st = st_local.data();
    }
    /* an error after copies were queued: wait for them (results unused) so
     * that none writes into the caller's buffers after the call returns */
    auto drain = [h](int code) {
        cudaGetLastError();
        for (cudaStream_t p : h->pipe)
            if (p) cudaStreamSynchronize(p);
        cudaGetLastError();
        return code;
    };
    size_t idx = 0;
    for (size_t f0 = 0; f0 < frames; f0 += chunk, idx++) {
        const int s = (int)(idx % kHostStages);
        const size_t nf = frames - f0 < chunk ? frames - f0 : chunk;
        cudaStream_t ps = h->pipe[s];
        if (cudaMemcpyAsync(h->pllr[s].p, rx + f0 * n, nf * n * 4, cudaMemcpyHostToDevice, ps) != cudaSuccess)
            return drain(WLDPC_ERR_CUDA);
        if ((rc = lms_launch_decode(h, (const float*)h->pllr[s].p, (int8_t*)h->phard[s].p,
                                    post ? (float*)h->pllr[s].p : nullptr, (int32_t*)h->pstat[s].p, nf, ps)))
            return drain(rc);
        if ((post &&
             cudaMemcpyAsync(post + f0 * n, h->pllr[s].p, nf * n * 4, cudaMemcpyDeviceToHost, ps) != cudaSuccess) ||
            cudaMemcpyAsync(decoded + f0 * n, h->phard[s].p, nf * n, cudaMemcpyDeviceToHost, ps) != cudaSuccess ||
            (st && cudaMemcpyAsync(st + f0, h->pstat[s].p, nf * 4, cudaMemcpyDeviceToHost, ps) != cudaSuccess))
            return drain(WLDPC_ERR_CUDA);
    }
    for (int s = 0; s < kHostStages; s++)
        if (cudaStreamSynchronize(h->pipe[s]) != cudaSuccess) return drain(WLDPC_ERR_CUDA);
    unsigned e = 0;
    CU(cudaMemcpy(&e, h->err, 4, cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(h->err, 0, 4);
        return WLDPC_ERR_TIMEOUT;
    }
    if (num_errors)
        for (size_t f = 0; f < frames; f++) num_errors[f] = (uint32_t)((st[f] >> 16) & 1);
    return WLDPC_OK;
}

int wldpc_lms_decode_host(wldpc_lms* h, float* rx, int8_t* decoded, uint32_t* num_errors, int32_t* status,
                          size_t frames)
{
    return lms_decode_host_pipeline(h, rx, rx, decoded, num_errors, status, frames);
}

int wldpc_lms_decode_host_hard(wldpc_lms* h, const float* llr, int8_t* decoded, uint32_t* num_errors,
                               int32_t* status, size_t frames)
{
    return lms_decode_host_pipeline(h, llr, nullptr, decoded, num_errors, status, frames);
}

/* one training forward/backward over `frames` frames already on the device;
 * leaves the per-frame partials in h->gpart / h->lpart */
static int lms_forward_backward(wldpc_lms* h, const float* llr, const uint8_t* cw, size_t frames, cudaStream_t st)
{
    const size_t n = (size_t)h->code.n, E = (size_t)h->nblk * h->z, T = (size_t)h->T;
    const size_t nw = 2 * T * h->nblk;
    int rc;
    if ((rc = h->ckp.reserve(frames * T * n * 4)) || (rc = h->ckm.reserve(frames * (T > 1 ? T - 1 : 1) * E * 4)) ||
        (rc = h->gpart.reserve(frames * nw * 4)) || (rc = h->lpart.reserve(frames * 4)))
        return rc;
    LmsTrainArgs a;
    a.llr = llr;
    a.cw = cw;
    a.ck_post = (float*)h->ckp.p;
    a.ck_msg = (float*)h->ckm.p;
    a.gpart = (float*)h->gpart.p;
    a.loss_part = (float*)h->lpart.p;
    a.wa = (const float*)h->wdev.p;
    a.wb = (const float*)h->wdev.p + T * h->nblk;
    a.frames = (long long)frames;
    a.iters = h->T;
    a.inv_norm = (float)(1.0 / ((double)T * (double)n * (double)frames));
    const LmsLaunch* k = h->k;
    if (k->train_smem > 48 * 1024)
        CU(cudaFuncSetAttribute(k->train, cudaFuncAttributeMaxDynamicSharedMemorySize, k->train_smem));
    k->train<<<(unsigned)frames, h->z, k->train_smem, st>>>(a);
    CU(cudaGetLastError());
    return WLDPC_OK;
}

static int lms_reduce(wldpc_lms* h, size_t frames, int apply, float lr, float* loss_out, cudaStream_t st)
{
    AdamArgs a;
    a.gpart = (const float*)h->gpart.p;
    a.loss_part = (const float*)h->lpart.p;
    a.grad = (float*)h->grad.p;
    a.w = (float*)h->wdev.p;
    a.m = (float*)h->mdev.p;
    a.v = (float*)h->vdev.p;
    a.loss_out = loss_out;
    a.frames = (long long)frames;
    a.nw = 2 * h->T * h->nblk;
    a.step = h->adam_step + 1;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.apply = apply;
    lms_reduce_adam_kernel<<<(a.nw + 127) / 128, 128, 0, st>>>(a);
    CU(cudaGetLastError());
    if (apply) {
        h->adam_step++;
        h->host_stale = true;
    }
    return WLDPC_OK;
}

int wldpc_lms_loss_grad(wldpc_lms* h, const float* llr, const uint8_t* codeword, size_t frames, float* grad_table,
                        double* loss)
{
    if (!h || !llr || !codeword || !grad_table || frames == 0) return WLDPC_ERR_ARG;
    if (h->host_stale == false) {
        int rc = lms_push_device_weights(h);
        if (rc) return rc;
    }
    const size_t n = (size_t)h->code.n;
    int rc;
    if ((rc = h->tllr.reserve(frames * n * 4)) || (rc = h->tcw.reserve(frames * n)) || (rc = h->loss.reserve(4)))
        return rc;
    CU(cudaMemcpyAsync(h->tllr.p, llr, frames * n * 4, cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->tcw.p, codeword, frames * n, cudaMemcpyHostToDevice, h->stream));
    if ((rc = lms_forward_backward(h, (const float*)h->tllr.p, (const uint8_t*)h->tcw.p, frames, h->stream)))
        return rc;
    if ((rc = lms_reduce(h, frames, 0, 0.0f, (float*)h->loss.p, h->stream))) return rc;
    const size_t nw = (size_t)2 * h->T * h->nblk;
    std::vector<float> g(nw);
    float l = 0.0f;
    CU(cudaMemcpyAsync(g.data(), h->grad.p, nw * 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(&l, h->loss.p, 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    const CodeDesc& c = h->code;
    memset(grad_table, 0, sizeof(float) * 2 * h->T * kMaxMb * kNB);
    for (int t = 0; t < h->T; t++)
        for (int i = 0; i < c.mb; i++)
            for (int b = c.row_start[i]; b < c.row_start[i + 1]; b++) {
                const size_t o = ((size_t)t * kMaxMb + i) * kNB + c.col[b];
                grad_table[o] = g[(size_t)t * h->nblk + b];
                grad_table[(size_t)h->T * kMaxMb * kNB + o] = g[(size_t)(h->T + t) * h->nblk + b];
            }
    if (loss) *loss = l;
    return WLDPC_OK;
}

int wldpc_lms_train(wldpc_lms* h, unsigned steps, unsigned batch, float ebno_lo_db, float ebno_hi_db, uint64_t seed,
                    uint64_t first_frame, float lr, float* loss_history)
{
    if (!h || batch == 0) return WLDPC_ERR_ARG;
    if (h->host_stale == false) {
        int rc = lms_push_device_weights(h);
        if (rc) return rc;
    }
    const size_t n = (size_t)h->code.n;
    int rc;
    if ((rc = h->tllr.reserve((size_t)batch * n * 4)) || (rc = h->tcw.reserve((size_t)batch * n)) ||
        (rc = h->loss.reserve((size_t)(steps ? steps : 1) * 4)))
        return rc;
    for (unsigned s = 0; s < steps; s++) {
        FramegenArgs f{};
        f.seed = seed;
        f.first_frame = first_frame + (uint64_t)s * batch;
        f.frames = batch;
        f.ebno_lo = ebno_lo_db;
        f.ebno_hi = ebno_hi_db;
        f.cw = (uint8_t*)h->tcw.p;
        f.llr = (float*)h->tllr.p;
        if (h->rate == THREEQUARTERSB) {   /* no dual-diagonal encoder: null-space codewords */
            if ((rc = wldpc_internal_nullspace_frames(h->rate, h->z, f, h->stream))) return rc;
        } else {
            CU(launch_framegen(h->code, f, h->stream));
        }
        if ((rc = lms_forward_backward(h, (const float*)h->tllr.p, (const uint8_t*)h->tcw.p, batch, h->stream)))
            return rc;
        if ((rc = lms_reduce(h, batch, 1, lr, (float*)h->loss.p + s, h->stream))) return rc;
    }
    if (loss_history && steps) CU(cudaMemcpyAsync(loss_history, h->loss.p, (size_t)steps * 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return lms_sync_host_weights(h);
}

/* the handle's stream waits for the work the caller queued on `user` */
static int lms_after_user_stream(wldpc_lms* h, cudaStream_t user)
{
    if (!h->ev_user) CU(cudaEventCreateWithFlags(&h->ev_user, cudaEventDisableTiming));
    CU(cudaEventRecord(h->ev_user, user));
    CU(cudaStreamWaitEvent(h->stream, h->ev_user, 0));
    return WLDPC_OK;
}

int wldpc_lms_grad_size(wldpc_lms* h, size_t* nw)
{
    if (!h || !nw) return WLDPC_ERR_ARG;
    *nw = (size_t)2 * h->T * h->nblk;
    return WLDPC_OK;
}

int wldpc_lms_step_grad(wldpc_lms* h, unsigned batch, float ebno_lo_db, float ebno_hi_db, uint64_t seed,
                        uint64_t first_frame, float* grad, float* loss, void* stream)
{
    if (!h || batch == 0 || !grad) return WLDPC_ERR_ARG;
    if (h->host_stale == false) {
        int rc = lms_push_device_weights(h);
        if (rc) return rc;
    }
    const size_t n = (size_t)h->code.n, nw = (size_t)2 * h->T * h->nblk;
    int rc;
    if ((rc = h->tllr.reserve((size_t)batch * n * 4)) || (rc = h->tcw.reserve((size_t)batch * n)) ||
        (rc = h->loss.reserve(4)))
        return rc;
    if ((rc = lms_after_user_stream(h, (cudaStream_t)stream))) return rc;
    FramegenArgs f{};
    f.seed = seed;
    f.first_frame = first_frame;
    f.frames = batch;
    f.ebno_lo = ebno_lo_db;
    f.ebno_hi = ebno_hi_db;
    f.cw = (uint8_t*)h->tcw.p;
    f.llr = (float*)h->tllr.p;
    if (h->rate == THREEQUARTERSB) {
        if ((rc = wldpc_internal_nullspace_frames(h->rate, h->z, f, h->stream))) return rc;
    } else {
        CU(launch_framegen(h->code, f, h->stream));
    }
    if ((rc = lms_forward_backward(h, (const float*)h->tllr.p, (const uint8_t*)h->tcw.p, batch, h->stream)))
        return rc;
    if ((rc = lms_reduce(h, batch, 0, 0.0f, (float*)h->loss.p, h->stream))) return rc;
    CU(cudaMemcpyAsync(grad, h->grad.p, nw * 4, cudaMemcpyDeviceToDevice, h->stream));
    if (loss) CU(cudaMemcpyAsync(loss, h->loss.p, 4, cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return WLDPC_OK;
}

int wldpc_lms_apply_grad(wldpc_lms* h, const float* grad, float lr, void* stream)
{
    if (!h || !grad) return WLDPC_ERR_ARG;
    if (h->host_stale == false) {
        int rc = lms_push_device_weights(h);
        if (rc) return rc;
    }
    int rc;
    if ((rc = lms_after_user_stream(h, (cudaStream_t)stream))) return rc;
    AdamArgs a;
    a.gpart = grad;            /* one "frame": the given gradient */
    a.loss_part = nullptr;
    a.grad = (float*)h->grad.p;
    a.w = (float*)h->wdev.p;
    a.m = (float*)h->mdev.p;
    a.v = (float*)h->vdev.p;
    a.loss_out = nullptr;
    a.frames = 1;
    a.nw = 2 * h->T * h->nblk;
    a.step = h->adam_step + 1;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.apply = 1;
    lms_reduce_adam_kernel<<<(a.nw + 127) / 128, 128, 0, h->stream>>>(a);
    CU(cudaGetLastError());
    h->adam_step++;
    h->host_stale = true;
    CU(cudaStreamSynchronize(h->stream));
    return WLDPC_OK;
}

}  // extern "C"
