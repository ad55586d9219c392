/*
 * Mixed-code persistent decoder (see mixed.cuh): binning kernels, CUDA-graph
 * capture, autotuning, and the C ABI (wldpc_mixed_*). The decode kernels are
 * in mixed_kernel.cuh, instantiated per rate by mixed_instances.cuh.
 */
#include <chrono>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include <cuda_runtime.h>

#include "wimax_ldpc_b200.h"
#include "codec_kernels.cuh"
#include "mixed_kernel.cuh"

namespace wldpc {

/* ---- binning: counts, plan (prefix sums and work items), scatter ---- */

__global__ void mixed_count_kernel(const uint8_t* __restrict__ variant, const long long* __restrict__ offset,
                                   int* __restrict__ counts, int* __restrict__ rank, long long frames, unsigned* err)
{
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < frames;
         f += (long long)gridDim.x * blockDim.x) {
        const int v = variant[f];
        /* a frame must start 16-byte aligned (its bulk copy and vector stores) */
        if (v >= kVariants || (offset[f] & 3) != 0 || offset[f] < 0) {
            atomicOr(err, kErrBadArgument);
            rank[f] = -1;
            continue;
        }
        rank[f] = atomicAdd(&counts[v], 1);
    }
}

__global__ void mixed_plan_kernel(const int* __restrict__ counts, int* __restrict__ base, MixedItem* __restrict__ items,
                                  int* __restrict__ num_items, int* __restrict__ queue, int chunk, long long per_rate)
{
    const int rate = threadIdx.x;
    if (blockIdx.x != 0 || rate >= kRates) return;
    /* frame list: rates in order, z descending within a rate (long items first) */
    int acc = 0;
    for (int q = 0; q < rate; q++)
        for (int zi = 0; zi < kNumZ; zi++) acc += counts[q * kNumZ + zi];
    int k = 0;
    MixedItem* it = items + (long long)rate * per_rate;
    for (int zi = kNumZ - 1; zi >= 0; zi--) {
        const int v = rate * kNumZ + zi;
        base[v] = acc;
        for (int s = 0; s < counts[v]; s += chunk) {
            it[k].variant = v;
            it[k].start = acc + s;
            it[k].count = counts[v] - s < chunk ? counts[v] - s : chunk;
            k++;
        }
        acc += counts[v];
    }
    num_items[rate] = k;
    queue[rate] = 0;
}

__global__ void mixed_scatter_kernel(const uint8_t* __restrict__ variant, const int* __restrict__ rank,
                                     const int* __restrict__ base, int* __restrict__ perm, long long frames)
{
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < frames;
         f += (long long)gridDim.x * blockDim.x) {
        if (rank[f] < 0) continue;
        perm[base[variant[f]] + rank[f]] = (int)f;
    }
}

}  // namespace wldpc

using namespace wldpc;

namespace {

constexpr int kThreadChoices[2] = {96, 192};

struct MBuf {
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
    ~MBuf()
    {
        if (p) cudaFree(p);
    }
};

inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace

namespace wldpc {
/* [threads 96 | 192][layout registers | shared][rows per thread 1 | 2], per
 * rate (mixed_instances.cuh) */
extern const MixedKernel kMixed_r0[2][2][2];
extern const MixedKernel kMixed_r1[2][2][2];
extern const MixedKernel kMixed_r2[2][2][2];
extern const MixedKernel kMixed_r3[2][2][2];
extern const MixedKernel kMixed_r4[2][2][2];
extern const MixedKernel kMixed_r5[2][2][2];
}  // namespace wldpc

static MixedKernel mixed_kernel(int ti, int layout, int rows, int rate)
{
    static const MixedKernel (*const t[kRates])[2][2] = {kMixed_r0, kMixed_r1, kMixed_r2,
                                                          kMixed_r3, kMixed_r4, kMixed_r5};
    return t[rate][ti][layout][rows - 1];
}

struct wldpc_mixed {
    unsigned max_iter;
    int threads = 96, layout = kMsgRegisters, chunk = 16;
    int rows = 1;                          /* expanded rows per thread: z / rows threads per frame */
    int launch = WLDPC_MIXED_CONCURRENT;   /* the six rate grids: concurrent or one after another */
    MixedCode codes[kVariants];            /* every code, by variant */
    int sms = 148;
    int per_sm[2][2][2][kRates] = {};   /* resident CTAs per SM, [96 | 192 threads][layout][rows - 1][rate] */
    cudaStream_t stream = nullptr;
    cudaStream_t rs[kRates] = {};
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr, ev_join[kRates] = {};
    unsigned* err = nullptr;
    MBuf counts, base, rank, perm, items, nitems, queue;
    /* captured graph and the arguments it was captured for */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Key {
        const void *variant, *offset, *llr, *hard, *post, *status;
        size_t frames;
        int threads, layout, chunk, launch, rows;
        bool operator==(const Key& o) const { return memcmp(this, &o, sizeof(Key)) == 0; }
    } key{};
};

static int mixed_enqueue(wldpc_mixed* h, const uint8_t* variant, const long long* offset, const float* llr,
                         int8_t* hard, float* post, int32_t* status, size_t frames, cudaStream_t st)
{
    const int chunk = h->chunk;
    const long long nf = (long long)frames;
    const long long per_rate = nf / chunk + kNumZ + 1;
    if (cudaMemsetAsync(h->counts.p, 0, sizeof(int) * kVariants, st) != cudaSuccess) return WLDPC_ERR_CUDA;
    const unsigned gb = (unsigned)((nf + 255) / 256 < 4096 ? (nf + 255) / 256 : 4096);
    mixed_count_kernel<<<gb, 256, 0, st>>>(variant, offset, (int*)h->counts.p, (int*)h->rank.p, nf, h->err);
    mixed_plan_kernel<<<1, 32, 0, st>>>((const int*)h->counts.p, (int*)h->base.p, (MixedItem*)h->items.p,
                                       (int*)h->nitems.p, (int*)h->queue.p, chunk, per_rate);
    mixed_scatter_kernel<<<gb, 256, 0, st>>>(variant, (const int*)h->rank.p, (const int*)h->base.p,
                                            (int*)h->perm.p, nf);
    MixedArgs a;
    a.variant = variant;
    a.offset = offset;
    a.llr = llr;
    a.hard = hard;
    a.post = post;
    a.status = status;
    a.perm = (const int*)h->perm.p;
    a.items = (const MixedItem*)h->items.p;
    a.num_items = (const int*)h->nitems.p;
    a.queue = (int*)h->queue.p;
    a.items_per_rate = per_rate;
    a.err = h->err;
    a.frames = nf;
    a.max_iter = (int)h->max_iter;
    const int T = h->threads;
    const int ti = T == 96 ? 0 : 1;
    if (cudaGetLastError() != cudaSuccess) return WLDPC_ERR_CUDA;
    if (h->launch == WLDPC_MIXED_SERIAL) {
        /* one rate after another on st, each grid with the whole GPU */
        for (int rate = 0; rate < kRates; rate++) {
            memcpy(a.codes, h->codes + rate * kNumZ, sizeof(a.codes));
            mixed_kernel(ti, h->layout, h->rows, rate)<<<h->sms * h->per_sm[ti][h->layout][h->rows - 1][rate], T,
                                                         mixed_smem_bytes(T, h->layout, rate, h->rows), st>>>(a);
            if (cudaGetLastError() != cudaSuccess) return WLDPC_ERR_CUDA;
        }
        return WLDPC_OK;
    }
    /* fork: the six rate kernels run concurrently, then join back on st */
    if (cudaEventRecord(h->ev_fork, st) != cudaSuccess) return WLDPC_ERR_CUDA;
    /* every forked stream is joined back even when a step fails, so that a
     * capture in progress always ends with all its streams joined */
    int rc = WLDPC_OK;
    for (int rate = 0; rate < kRates; rate++) {
        const MixedKernel k = mixed_kernel(ti, h->layout, h->rows, rate);
        const int per_sm = h->per_sm[ti][h->layout][h->rows - 1][rate];
        if (cudaStreamWaitEvent(h->rs[rate], h->ev_fork, 0) != cudaSuccess) {
            rc = WLDPC_ERR_CUDA;
            break;
        }
        memcpy(a.codes, h->codes + rate * kNumZ, sizeof(a.codes));
        k<<<h->sms * per_sm, T, mixed_smem_bytes(T, h->layout, rate, h->rows), h->rs[rate]>>>(a);
        if (cudaGetLastError() != cudaSuccess) rc = WLDPC_ERR_CUDA;
        if (cudaEventRecord(h->ev_join[rate], h->rs[rate]) != cudaSuccess ||
            cudaStreamWaitEvent(st, h->ev_join[rate], 0) != cudaSuccess) {
            rc = WLDPC_ERR_CUDA;
            break;
        }
    }
    return rc;
}

extern "C" {

int wldpc_variant(int rate, unsigned z)
{
    if (!valid_rate(rate) || !valid_z((int)z)) return WLDPC_ERR_CODE;
    return rate * kNumZ + z_index((int)z);
}

int wldpc_mixed_create(unsigned max_iter, wldpc_mixed** out)
{
    if (!out) return WLDPC_ERR_ARG;
    *out = nullptr;
    if (max_iter > 0xffff) return WLDPC_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    wldpc_mixed* h = new (std::nothrow) wldpc_mixed();
    if (!h) return WLDPC_ERR_ARG;
    h->max_iter = max_iter;
    for (int rate = 0; rate < kRates; rate++)
        for (int zi = 0; zi < kNumZ; zi++) {
            const int z = kZMin + kZStep * zi;
            const CodeDesc c = make_code_desc(rate, z);
            MixedCode& m = h->codes[rate * kNumZ + zi];
            memset(&m, 0, sizeof(m));
            m.z = (unsigned short)z;
            m.n = (unsigned short)c.n;
            for (int b = 0; b < c.nblk; b++) {
                m.colz[b] = (unsigned short)(c.col[b] * z);
                m.shift[b] = (unsigned char)c.shift[b];
            }
        }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev);
    /* shared-memory limit and occupancy of every decode kernel, once, outside any capture */
    for (int ti = 0; ti < 2; ti++)
        for (int layout = 0; layout < 2; layout++)
            for (int rows = 1; rows <= 2; rows++)
                for (int rate = 0; rate < kRates; rate++) {
                    const int T = kThreadChoices[ti];
                    const int smem = mixed_smem_bytes(T, layout, rate, rows);
                    const MixedKernel k = mixed_kernel(ti, layout, rows, rate);
                    int per = 0;
                    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
                        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, smem) != cudaSuccess) {
                        cudaGetLastError();
                        delete h;
                        return WLDPC_ERR_CUDA;
                    }
                    h->per_sm[ti][layout][rows - 1][rate] = per > 0 ? per : 1;
                }
    bool ok = true;
    for (int r = 0; r < kRates; r++)
        ok = ok && cudaStreamCreateWithFlags(&h->rs[r], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->ev_join[r], cudaEventDisableTiming) == cudaSuccess;
    if (!ok || cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&h->err, sizeof(unsigned)) != cudaSuccess || cudaMemset(h->err, 0, 4) != cudaSuccess ||
        h->counts.reserve(sizeof(int) * kVariants) || h->base.reserve(sizeof(int) * kVariants) ||
        h->nitems.reserve(sizeof(int) * kRates) || h->queue.reserve(sizeof(int) * kRates)) {
        cudaGetLastError();
        wldpc_mixed_destroy(h);
        return WLDPC_ERR_CUDA;
    }
    *out = h;
    return WLDPC_OK;
}

int wldpc_mixed_destroy(wldpc_mixed* h)
{
    if (!h) return WLDPC_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->stream) cudaStreamDestroy(h->stream);
    for (int r = 0; r < kRates; r++) {
        if (h->rs[r]) cudaStreamDestroy(h->rs[r]);
        if (h->ev_join[r]) cudaEventDestroy(h->ev_join[r]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_in) cudaEventDestroy(h->ev_in);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->err) cudaFree(h->err);
    delete h;
    return WLDPC_OK;
}

int wldpc_mixed_set_tuning(wldpc_mixed* h, int threads, int layout, int chunk, int launch)
{
    if (!h || chunk < 1 || chunk > kMixedMaxChunk) return WLDPC_ERR_ARG;
    if (threads != 96 && threads != 192) return WLDPC_ERR_ARG;
    if (layout != WLDPC_MIXED_MSG_REGISTERS && layout != WLDPC_MIXED_MSG_SHARED) return WLDPC_ERR_ARG;
    if (launch != WLDPC_MIXED_CONCURRENT && launch != WLDPC_MIXED_SERIAL) return WLDPC_ERR_ARG;
    h->threads = threads;
    h->layout = layout;
    h->chunk = chunk;
    h->launch = launch;
    return WLDPC_OK;
}

int wldpc_mixed_get_tuning(wldpc_mixed* h, int* threads, int* layout, int* chunk, int* launch)
{
    if (!h) return WLDPC_ERR_ARG;
    if (threads) *threads = h->threads;
    if (layout) *layout = h->layout;
    if (chunk) *chunk = h->chunk;
    if (launch) *launch = h->launch;
    return WLDPC_OK;
}

int wldpc_mixed_set_rows_per_thread(wldpc_mixed* h, int rows)
{
    if (!h || (rows != 1 && rows != 2)) return WLDPC_ERR_ARG;
    h->rows = rows;
    return WLDPC_OK;
}

int wldpc_mixed_get_rows_per_thread(wldpc_mixed* h, int* rows)
{
    if (!h || !rows) return WLDPC_ERR_ARG;
    *rows = h->rows;
    return WLDPC_OK;
}

int wldpc_mixed_set_config(wldpc_mixed* h, int threads, int chunk)
{
    if (!h) return WLDPC_ERR_ARG;
    return wldpc_mixed_set_tuning(h, threads, h->layout, chunk, h->launch);
}

int wldpc_mixed_get_config(wldpc_mixed* h, int* threads, int* chunk)
{
    return wldpc_mixed_get_tuning(h, threads, nullptr, chunk, nullptr);
}

int wldpc_mixed_decode_device(wldpc_mixed* h, const uint8_t* variant, const int64_t* offset, const float* llr,
                              int8_t* decoded, float* posterior, int32_t* status, size_t frames, void* stream)
{
    if (!h || (frames && (!variant || !offset || !llr || !decoded))) return WLDPC_ERR_ARG;
    if (!aligned(llr, 16) || !aligned(decoded, 4) || !aligned(posterior, 16) || !aligned(status, 4) ||
        !aligned(offset, 8))
        return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    if (frames > 0x7fffffff) return WLDPC_ERR_ARG;
    int rc;
    const size_t max_items = kRates * (frames / (size_t)h->chunk + kNumZ + 1);
    if ((rc = h->rank.reserve(frames * sizeof(int))) || (rc = h->perm.reserve(frames * sizeof(int))) ||
        (rc = h->items.reserve(max_items * sizeof(MixedItem))))
        return rc;
    wldpc_mixed::Key key{variant,  offset,     llr,       decoded,  posterior, status,
                         frames,   h->threads, h->layout, h->chunk, h->launch, h->rows};
    const cudaStream_t user = (cudaStream_t)stream;
    if (cudaEventRecord(h->ev_in, user) != cudaSuccess || cudaStreamWaitEvent(h->stream, h->ev_in, 0) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    if (!h->exec || !(h->key == key)) {
        if (h->exec) cudaGraphExecDestroy(h->exec);
        if (h->graph) cudaGraphDestroy(h->graph);
        h->exec = nullptr;
        h->graph = nullptr;
        if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return WLDPC_ERR_CUDA;
        }
        rc = mixed_enqueue(h, variant, (const long long*)offset, llr, decoded, posterior, status, frames, h->stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc || e != cudaSuccess || !g) {
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            return rc ? rc : WLDPC_ERR_CUDA;
        }
        if (cudaGraphInstantiate(&h->exec, g, 0) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphDestroy(g);
            return WLDPC_ERR_CUDA;
        }
        h->graph = g;
        h->key = key;
    }
    if (cudaGraphLaunch(h->exec, h->stream) != cudaSuccess || cudaEventRecord(h->ev_out, h->stream) != cudaSuccess ||
        cudaStreamWaitEvent(user, h->ev_out, 0) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    return WLDPC_OK;
}

int wldpc_mixed_synchronize(wldpc_mixed* h)
{
    if (!h) return WLDPC_ERR_ARG;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    unsigned e = 0;
    if (cudaMemcpy(&e, h->err, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    if (e) {
        cudaMemset(h->err, 0, 4);
        return (e & kErrBadArgument) ? WLDPC_ERR_ARG : WLDPC_ERR_TIMEOUT;
    }
    return WLDPC_OK;
}

int wldpc_mixed_autotune(wldpc_mixed* h, const uint8_t* variant, const int64_t* offset, const float* llr,
                         int8_t* decoded, size_t frames, int repeats, float* best_ms)
{
    if (!h || repeats < 1) return WLDPC_ERR_ARG;
    static const int chunks[4] = {8, 16, 32, 64};
    float best = 1e30f;
    int bt = h->threads, bl = h->layout, bc = h->chunk, bp = h->launch, br = h->rows;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    auto restore = [&]() {
        h->threads = bt;
        h->layout = bl;
        h->chunk = bc;
        h->launch = bp;
        h->rows = br;
    };
    /* CTA size x rows per thread x message layout x frames per work item x
     * launch policy, timed on the caller's batch */
    for (int ti = 0; ti < 2; ti++)
        for (int rows = 1; rows <= 2; rows++)
            for (int layout = 0; layout < 2; layout++)
                for (int ci = 0; ci < 4; ci++)
                    for (int lp = 0; lp < 2; lp++) {
                        h->threads = kThreadChoices[ti];
                        h->rows = rows;
                        h->layout = layout;
                        h->chunk = chunks[ci];
                        h->launch = lp;
                        int rc = wldpc_mixed_decode_device(h, variant, offset, llr, decoded, nullptr, nullptr,
                                                           frames, h->stream);
                        if (!rc && cudaEventRecord(e0, h->stream) != cudaSuccess) rc = WLDPC_ERR_CUDA;
                        for (int k = 0; k < repeats && !rc; k++)
                            rc = wldpc_mixed_decode_device(h, variant, offset, llr, decoded, nullptr, nullptr,
                                                           frames, h->stream);
                        if (!rc && (cudaEventRecord(e1, h->stream) != cudaSuccess ||
                                    cudaEventSynchronize(e1) != cudaSuccess))
                            rc = WLDPC_ERR_CUDA;
                        if (rc) {
                            cudaGetLastError();
                            cudaEventDestroy(e0);
                            cudaEventDestroy(e1);
                            restore();
                            return rc;
                        }
                        float ms = 0.f;
                        cudaEventElapsedTime(&ms, e0, e1);
                        ms /= repeats;
                        if (ms < best) {
                            best = ms;
                            bt = h->threads;
                            bl = h->layout;
                            bc = h->chunk;
                            bp = h->launch;
                            br = h->rows;
                        }
                    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    restore();
    if (best_ms) *best_ms = best;
    return wldpc_mixed_synchronize(h);
}

}  // extern "C"
