/*
 * Mixed-code persistent decoder (see mixed.cuh): kernels, binning, CUDA-graph
 * capture, autotuning, and the C ABI (wldpc_mixed_*).
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
#include "mixed.cuh"

namespace wldpc {

__constant__ MixedCode c_codes[kVariants];

struct MixedSlots {
    int frame[32];
    int next;
    unsigned fresh, fail;
    int item;
};

/* Each thread's edge addresses for the current code, [block][thread] in
 * shared memory, computed once per work item: one 16-bit load per edge. */
template <int R, int I, int E, int THREADS>
__device__ __forceinline__ int mixed_var(const unsigned short* A)
{
    constexpr int b = block_index(R, I, E);
    return A[b * THREADS + threadIdx.x];
}

template <int R, int THREADS>
__device__ __forceinline__ void mixed_run_item(const MixedArgs& a, const MixedItem item, float* sp,
                                               unsigned short* A, MixedSlots& S)
{
    constexpr int MB = kMb[R];
    constexpr int NBLK = num_blocks(R);
    const MixedCode& code = c_codes[item.variant];
    const int z = code.z, n = code.n;
    const int G = THREADS / z;
    const int tid = threadIdx.x;
    const int g = tid / z;
    const int r = tid - g * z;
    const bool in_slot = g < G;
    float* P = sp + (in_slot ? g : 0) * n;
    for (int b = 0; b < NBLK; b++) {
        int t = r + (int)code.shift[b];
        t = t >= z ? t - z : t;
        A[b * THREADS + tid] = in_slot ? (unsigned short)(code.colz[b] + t) : (unsigned short)0;
    }

    float M1[MB], M2[MB];
    uint32_t NEG[MB];
    int frame = -1, iters = 0;
    long long off = 0;
    bool need_check = false;

    if (tid == 0) {
        S.next = 0;
        for (int q = 0; q < G; q++) S.frame[q] = -1;
    }
    __syncthreads();
    while (true) {
        /* refill empty slots with the item's next frames */
        if (tid == 0) {
            unsigned fresh = 0;
            for (int q = 0; q < G; q++)
                if (S.frame[q] < 0 && S.next < item.count) {
                    S.frame[q] = a.perm[item.start + S.next++];
                    fresh |= 1u << q;
                }
            S.fresh = fresh;
            S.fail = 0;
        }
        __syncthreads();
        if (in_slot && ((S.fresh >> g) & 1u)) {
            frame = S.frame[g];
            off = a.offset[frame];
            iters = 0;
            need_check = true;
            for (int c = 0; c < kNB; c++) P[c * z + r] = a.llr[off + c * z + r];
#pragma unroll
            for (int i = 0; i < MB; i++) { M1[i] = 0.0f; M2[i] = 0.0f; NEG[i] = 0u; }
        }
        __syncthreads();
        /* syndrome of the slots loaded or iterated since their last check */
        if (in_slot && frame >= 0 && need_check) {
            unsigned fail = 0;
            static_for<MB>([&](auto I) {
                constexpr int d = layer_degree(R, I);
                bool odd = (d & 1) != 0;   /* parity of the hard bits: d minus the negatives */
                static_for<d>([&](auto E_) {
                    odd = odd != (P[mixed_var<R, I, E_, THREADS>(A)] < 0.0f);
                });
                fail |= odd ? 1u : 0u;
            });
            if (fail) atomicOr(&S.fail, 1u << g);
        }
        __syncthreads();
        if (in_slot && frame >= 0 && need_check) {
            need_check = false;
            const bool failed = (S.fail >> g) & 1u;
            if (!failed || iters >= a.max_iter) {
                for (int c = 0; c < kNB; c++) {
                    const float p = P[c * z + r];
                    a.hard[off + c * z + r] = p >= 0.0f ? 1 : 0;
                    if (a.post) a.post[off + c * z + r] = p;
                }
                if (r == 0) {
                    if (a.status) a.status[frame] = iters | ((failed ? 1 : 0) << 16);
                    S.frame[g] = -1;
                }
                frame = -1;
            }
        }
        __syncthreads();
        bool any_empty = false, all_empty = true;
        for (int q = 0; q < G; q++) {
            any_empty |= S.frame[q] < 0;
            all_empty &= S.frame[q] < 0;
        }
        const bool more = S.next < item.count;
        __syncthreads();
        if (all_empty && !more) break;
        if (any_empty && more) continue;

        /* one iteration of every occupied slot (all of them failed their check) */
        const bool active = in_slot && frame >= 0;
        static_for<MB>([&](auto I) {
            constexpr int d = layer_degree(R, I);
            if (active) {
                float L[d];
                uint32_t LC[d];
                uint32_t sgn = 0;
                float m1, m2;
                const float oM1 = M1[I], oM2 = M2[I];
                const uint32_t oNeg = NEG[I];
                const int oIdx = (int)(oNeg >> 27);
                /* the layer's edge addresses, loaded once for both passes */
                int ad[d];
                static_for<d>([&](auto E_) { ad[decltype(E_)::value] = mixed_var<R, I, decltype(E_)::value, THREADS>(A); });
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    const float x = P[ad[e]];
                    const float mag = (oIdx == e) ? oM2 : oM1;
                    const uint32_t sb = (oNeg << (32 - d + e)) & 0x80000000u;
                    const float l = __fsub_rn(x, __uint_as_float(__float_as_uint(mag) | sb));
                    L[e] = l;
                    LC[e] = __float_as_uint(canon(l));
                    sgn = __funnelshift_l(LC[e], sgn, 1);
                });
                /* the two smallest |L| from 10000.0f (reference lib/ldpc_decoder.cc:150,198) */
                two_min_abs<0, d>(L, m1, m2);
                m1 = fminf(m1, 10000.0f);
                m2 = fminf(m2, 10000.0f);
                const uint32_t flip = (uint32_t)((d & 1) ^ (__popc(sgn) & 1));
                const uint32_t dmask = (d >= 32) ? 0xffffffffu : ((1u << d) - 1u);
                const double D1 = __dmul_rn((double)m1, 0.815);
                const double D2 = __dmul_rn((double)m2, 0.815);
                const uint32_t fb = flip << 31;
                const int h1 = __double2hiint(D1) ^ (int)fb, l1 = __double2loint(D1);
                const int h2 = __double2hiint(D2) ^ (int)fb, l2 = __double2loint(D2);
                int nIdx = 0;
                static_for<d>([&](auto E_) {
                    constexpr int e = decltype(E_)::value;
                    const float l = L[e];
                    const bool is_min = fabsf(l) == m1;
                    nIdx = is_min ? e : nIdx;
                    int hi = is_min ? h2 : h1;
                    const int lo = is_min ? l2 : l1;
                    hi ^= (int)(LC[e] & 0x80000000u);
                    P[ad[e]] = __double2float_rn(__dadd_rn((double)l, __hiloint2double(hi, lo)));
                });
                M1[I] = __double2float_rn(D1);
                M2[I] = __double2float_rn(D2);
                NEG[I] = ((sgn ^ (flip ? dmask : 0u)) & dmask) | ((uint32_t)nIdx << 27);
            }
            __syncthreads();
        });
        if (active) {
            iters++;
            need_check = true;
        }
    }
}

/* One persistent kernel per rate: it takes work items of its rate from its
 * own queue until none are left. The register cap (80 per thread: 8 CTAs of
 * 96 or 4 of 192 threads per SM) trades a few spills in the 5/6 kernels for
 * more resident warps; the kernel is latency-bound, and this measured 18.6
 * against 16.2 info Gbit/s uncapped on the mixed batch. */
template <int R, int THREADS>
__global__ void __launch_bounds__(THREADS, (THREADS == 96 ? 8 : 4)) mixed_decode_kernel(const __grid_constant__ MixedArgs a)
{
    extern __shared__ __align__(16) float smem_mixed[];   /* posteriors, then the address table */
    __shared__ MixedSlots S;
    unsigned short* A = reinterpret_cast<unsigned short*>(smem_mixed + 24 * THREADS);
    const MixedItem* items = a.items + (long long)R * a.items_per_rate;
    while (true) {
        if (threadIdx.x == 0) S.item = atomicAdd(&a.queue[R], 1);
        __syncthreads();
        const int k = S.item;
        __syncthreads();
        if (k >= a.num_items[R]) break;
        mixed_run_item<R, THREADS>(a, items[k], smem_mixed, A, S);
        __syncthreads();
    }
}

/* ---- binning: counts, plan (prefix sums and work items), scatter ---- */

__global__ void mixed_count_kernel(const uint8_t* __restrict__ variant, int* __restrict__ counts,
                                   int* __restrict__ rank, long long frames, unsigned* err)
{
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < frames;
         f += (long long)gridDim.x * blockDim.x) {
        const int v = variant[f];
        if (v >= kVariants) {
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

/* per device: the code table has been copied into c_codes */
bool g_codes_uploaded[64] = {false};
std::mutex g_codes_mutex;

int upload_codes()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= 64) return WLDPC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_codes_mutex);
    if (g_codes_uploaded[dev]) return WLDPC_OK;
    std::vector<MixedCode> t(kVariants);
    for (int rate = 0; rate < kRates; rate++)
        for (int zi = 0; zi < kNumZ; zi++) {
            const int z = kZMin + kZStep * zi;
            const CodeDesc c = make_code_desc(rate, z);
            MixedCode& m = t[rate * kNumZ + zi];
            memset(&m, 0, sizeof(m));
            m.z = (unsigned short)z;
            m.n = (unsigned short)c.n;
            for (int b = 0; b < c.nblk; b++) {
                m.colz[b] = (unsigned short)(c.col[b] * z);
                m.shift[b] = c.shift[b];
            }
        }
    if (cudaMemcpyToSymbol(c_codes, t.data(), sizeof(MixedCode) * kVariants) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    g_codes_uploaded[dev] = true;
    return WLDPC_OK;
}

}  // namespace

struct wldpc_mixed {
    unsigned max_iter;
    int threads = 96, chunk = 32;
    int sms = 148;
    int per_sm[2][kRates] = {};   /* resident CTAs per SM, [96 | 192 threads][rate] */
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
        int threads, chunk;
        bool operator==(const Key& o) const { return memcmp(this, &o, sizeof(Key)) == 0; }
    } key{};
};

using MixedKernel = void (*)(const MixedArgs);
/* dynamic shared memory of a CTA: posteriors (24 floats per thread) and the
 * 16-bit address table (96 blocks per thread) */
static int mixed_smem(int threads) { return 24 * threads * 4 + 96 * threads * 2; }
template <int T>
struct MixedKernels {
    static constexpr MixedKernel k[kRates] = {&mixed_decode_kernel<0, T>, &mixed_decode_kernel<1, T>,
                                             &mixed_decode_kernel<2, T>, &mixed_decode_kernel<3, T>,
                                             &mixed_decode_kernel<4, T>, &mixed_decode_kernel<5, T>};
};

static int mixed_enqueue(wldpc_mixed* h, const uint8_t* variant, const long long* offset, const float* llr,
                         int8_t* hard, float* post, int32_t* status, size_t frames, cudaStream_t st)
{
    const int chunk = h->chunk;
    const long long nf = (long long)frames;
    const long long per_rate = nf / chunk + kNumZ + 1;
    if (cudaMemsetAsync(h->counts.p, 0, sizeof(int) * kVariants, st) != cudaSuccess) return WLDPC_ERR_CUDA;
    const unsigned gb = (unsigned)((nf + 255) / 256 < 4096 ? (nf + 255) / 256 : 4096);
    mixed_count_kernel<<<gb, 256, 0, st>>>(variant, (int*)h->counts.p, (int*)h->rank.p, nf, h->err);
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
    const int smem = mixed_smem(T);
    /* fork: the six rate kernels run concurrently, then join back on st */
    if (cudaGetLastError() != cudaSuccess || cudaEventRecord(h->ev_fork, st) != cudaSuccess) return WLDPC_ERR_CUDA;
    /* every forked stream is joined back even when a step fails, so that a
     * capture in progress always ends with all its streams joined */
    int rc = WLDPC_OK;
    for (int rate = 0; rate < kRates; rate++) {
        const MixedKernel k = ti == 0 ? MixedKernels<96>::k[rate] : MixedKernels<192>::k[rate];
        const int per_sm = h->per_sm[ti][rate];
        if (cudaStreamWaitEvent(h->rs[rate], h->ev_fork, 0) != cudaSuccess) {
            rc = WLDPC_ERR_CUDA;
            break;
        }
        k<<<h->sms * per_sm, T, smem, h->rs[rate]>>>(a);
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
    int rc = upload_codes();
    if (rc) return rc;
    wldpc_mixed* h = new (std::nothrow) wldpc_mixed();
    if (!h) return WLDPC_ERR_ARG;
    h->max_iter = max_iter;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, dev);
    /* shared-memory limit and occupancy of every decode kernel, once, outside any capture */
    for (int ti = 0; ti < 2; ti++)
        for (int rate = 0; rate < kRates; rate++) {
            const int T = ti == 0 ? 96 : 192;
            const MixedKernel k = ti == 0 ? MixedKernels<96>::k[rate] : MixedKernels<192>::k[rate];
            int per = 0;
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, mixed_smem(T)) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, mixed_smem(T)) != cudaSuccess) {
                cudaGetLastError();
                delete h;
                return WLDPC_ERR_CUDA;
            }
            h->per_sm[ti][rate] = per > 0 ? per : 1;
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

int wldpc_mixed_set_config(wldpc_mixed* h, int threads, int chunk)
{
    if (!h || chunk < 1 || chunk > (1 << 20)) return WLDPC_ERR_ARG;
    if (threads != 96 && threads != 192) return WLDPC_ERR_ARG;
    h->threads = threads;
    h->chunk = chunk;
    return WLDPC_OK;
}

int wldpc_mixed_get_config(wldpc_mixed* h, int* threads, int* chunk)
{
    if (!h) return WLDPC_ERR_ARG;
    if (threads) *threads = h->threads;
    if (chunk) *chunk = h->chunk;
    return WLDPC_OK;
}

int wldpc_mixed_decode_device(wldpc_mixed* h, const uint8_t* variant, const int64_t* offset, const float* llr,
                              int8_t* decoded, float* posterior, int32_t* status, size_t frames, void* stream)
{
    if (!h || (frames && (!variant || !offset || !llr || !decoded))) return WLDPC_ERR_ARG;
    if (frames == 0) return WLDPC_OK;
    if (frames > 0x7fffffff) return WLDPC_ERR_ARG;
    int rc;
    const size_t max_items = kRates * (frames / (size_t)h->chunk + kNumZ + 1);
    if ((rc = h->rank.reserve(frames * sizeof(int))) || (rc = h->perm.reserve(frames * sizeof(int))) ||
        (rc = h->items.reserve(max_items * sizeof(MixedItem))))
        return rc;
    wldpc_mixed::Key key{variant, offset, llr, decoded, posterior, status, frames, h->threads, h->chunk};
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
    int bt = h->threads, bc = h->chunk;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return WLDPC_ERR_CUDA;
    }
    for (int ti = 0; ti < 2; ti++)
        for (int ci = 0; ci < 4; ci++) {
            h->threads = kThreadChoices[ti];
            h->chunk = chunks[ci];
            int rc = wldpc_mixed_decode_device(h, variant, offset, llr, decoded, nullptr, nullptr, frames, h->stream);
            if (!rc && cudaEventRecord(e0, h->stream) != cudaSuccess) rc = WLDPC_ERR_CUDA;
            for (int k = 0; k < repeats && !rc; k++)
                rc = wldpc_mixed_decode_device(h, variant, offset, llr, decoded, nullptr, nullptr, frames, h->stream);
            if (!rc && (cudaEventRecord(e1, h->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
                rc = WLDPC_ERR_CUDA;
            if (rc) {
                cudaGetLastError();
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                h->threads = bt;
                h->chunk = bc;
                return rc;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= repeats;
            if (ms < best) {
                best = ms;
                bt = h->threads;
                bc = h->chunk;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->threads = bt;
    h->chunk = bc;
    if (best_ms) *best_ms = best;
    return WLDPC_OK;
}

}  // extern "C"
