// Functional delivery op: fold a batch of synaptic arrivals into conductance
// arrays in the reference's delivery order, on the device.
//
// The reference CPU models add each arriving weight straight into the target's
// conductance as the event is processed (NeuronModel::ProcessInputSpike,
// src/neuron_model/LIFTimeDrivenModel.cpp:77-83), i.e. per target in order of
// arrival time, ties in event order (src/spike/PropagatedSpikeGroup.cpp:112-149);
// its GPU models instead sum a step's arrivals on the host into AuxState
// (src/neuron_model/LIFTimeDrivenModel_GPU_C_INTERFACE.cu:66-70).  This op gives
// a host-driven engine the CPU models' rounding on the GPU: arrivals are grouped
// per target (count, scan, scatter -- integer atomics only), sorted per target by
// (time, position in the batch), and added in that order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "edlut_b200.h"
#include "eb_runtime.h"

using namespace eb;

namespace {

struct FoldRec {
    double t;
    uint32_t i;
    uint32_t pad;
};

__device__ __forceinline__ bool fold_less(const FoldRec &a, const FoldRec &b) {
    return a.t < b.t || (a.t == b.t && a.i < b.i);
}

__global__ void k_fold_count(int64_t n, const int32_t *target, uint32_t *cnt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + target[i], 1u);
}

// Exclusive scan of cnt[0..m) into offs[0..m], two levels: per 1024-element
// block (offs, block totals), then the block totals (single block), then add.
constexpr int kScanBlock = 1024;

__global__ void k_scan_blocks(int64_t m, const uint32_t *cnt, uint32_t *offs, uint32_t *totals) {
    __shared__ uint32_t s[kScanBlock];
    const int64_t base = (int64_t)blockIdx.x * kScanBlock;
    const int t = threadIdx.x;
    s[t] = (base + t < m) ? cnt[base + t] : 0u;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        uint32_t v = t >= o ? s[t - o] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    if (base + t < m) offs[base + t] = s[t] - ((base + t < m) ? cnt[base + t] : 0u);
    if (t == kScanBlock - 1) totals[blockIdx.x] = s[t];
}

__global__ void k_scan_totals(int nb, uint32_t *totals) {
    __shared__ uint32_t s[kScanBlock];
    const int t = threadIdx.x;
    s[t] = t < nb ? totals[t] : 0u;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        uint32_t v = t >= o ? s[t - o] : 0u;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    if (t < nb) totals[t] = s[t] - (t < nb ? totals[t] : 0u);
}

__global__ void k_scan_add(int64_t m, uint32_t *offs, const uint32_t *totals) {
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < m) offs[i] += totals[blockIdx.x];
}

__global__ void k_fold_scatter(int64_t n, const int32_t *target, const double *time, const uint32_t *offs,
                               uint32_t *fill, FoldRec *rec) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t t = target[i];
        const uint32_t p = atomicAdd(fill + t, 1u);
        FoldRec r;
        r.t = time ? time[i] : 0.0;
        r.i = (uint32_t)i;
        r.pad = 0;
        rec[offs[t] + p] = r;
    }
}

// Restore the heap property below node j of the max-heap r[0..c) by (time, index).
__device__ __forceinline__ void sift_down(FoldRec *r, uint32_t j, uint32_t c) {
    const FoldRec v = r[j];
    for (;;) {
        uint32_t ch = 2 * j + 1;
        if (ch >= c) break;
        if (ch + 1 < c && fold_less(r[ch], r[ch + 1])) ++ch;
        if (!fold_less(v, r[ch])) break;
        r[j] = r[ch];
        j = ch;
    }
    r[j] = v;
}

// Sort r[0..c) by (time, index) in place: insertion sort for the few arrivals a
// target usually gets, heapsort (O(c log c), no extra memory) beyond, so a batch
// that sends every arrival to one target stays bounded.  The keys are distinct
// (the index), so both give the same order.
constexpr uint32_t kFoldInsertionMax = 32;

__device__ __forceinline__ void fold_sort(FoldRec *r, uint32_t c) {
    if (c <= kFoldInsertionMax) {
        for (uint32_t a = 1; a < c; ++a) {
            FoldRec v = r[a];
            int b = (int)a - 1;
            while (b >= 0 && fold_less(v, r[b])) { r[b + 1] = r[b]; --b; }
            r[b + 1] = v;
        }
        return;
    }
    for (uint32_t j = c / 2; j-- > 0;) sift_down(r, j, c);
    for (uint32_t e = c - 1; e > 0; --e) {
        const FoldRec top = r[0];
        r[0] = r[e];
        r[e] = top;
        sift_down(r, 0, e);
    }
}

// One thread per target: sort its arrivals by (time, index) in place, then add
// the weights in that order.
__global__ void k_fold_apply(int64_t m, const uint32_t *cnt, const uint32_t *offs, FoldRec *rec,
                             const int8_t *type, const float *weight, float *g_exc, float *g_inh, float *g_nmda) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const uint32_t c = cnt[t];
    if (!c) return;
    FoldRec *r = rec + offs[t];
    fold_sort(r, c);
    float ge = g_exc ? g_exc[t] : 0.0f, gi = g_inh ? g_inh[t] : 0.0f, gn = g_nmda ? g_nmda[t] : 0.0f;
    for (uint32_t a = 0; a < c; ++a) {
        const uint32_t i = r[a].i;
        const int ty = type[i];
        const float w = weight[i];
        if (ty == 0) ge += w;
        else if (ty == 1) gi += w;
        else gn += w;
    }
    if (g_exc) g_exc[t] = ge;
    if (g_inh) g_inh[t] = gi;
    if (g_nmda) g_nmda[t] = gn;
}

// Scratch layout shared by the entry points: cnt, fill, offs (m+1 each, uint32),
// block totals, then the records (16-byte aligned).
size_t fold_scratch_bytes(int64_t n, int64_t m) {
    size_t words = 3 * (size_t)(m + 1) + kScanBlock;
    size_t b = (words * sizeof(uint32_t) + 255) & ~(size_t)255;
    return b + (size_t)n * sizeof(FoldRec);
}

int fold_enqueue(cudaStream_t st, void *scratch, int64_t n, const int32_t *target, const int8_t *type,
                 const float *weight, const double *time, int64_t m, float *g_exc, float *g_inh, float *g_nmda) {
    uint32_t *cnt = (uint32_t *)scratch;
    uint32_t *fill = cnt + (m + 1);
    uint32_t *offs = fill + (m + 1);
    uint32_t *totals = offs + (m + 1);
    size_t words = 3 * (size_t)(m + 1) + kScanBlock;
    FoldRec *rec = (FoldRec *)((char *)scratch + ((words * sizeof(uint32_t) + 255) & ~(size_t)255));
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * 2 * (size_t)(m + 1), st);
    if (e != cudaSuccess) { set_error("cudaMemsetAsync: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
    if (n == 0) return EB_OK;
    const int nb = (int)((m + kScanBlock - 1) / kScanBlock);
    const int gb = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_fold_count<<<gb, 256, 0, st>>>(n, target, cnt);
    k_scan_blocks<<<nb, kScanBlock, 0, st>>>(m, cnt, offs, totals);
    k_scan_totals<<<1, kScanBlock, 0, st>>>(nb, totals);
    k_scan_add<<<nb, kScanBlock, 0, st>>>(m, offs, totals);
    k_fold_scatter<<<gb, 256, 0, st>>>(n, target, time, offs, fill, rec);
    k_fold_apply<<<(int)((m + 255) / 256), 256, 0, st>>>(m, cnt, offs, rec, type, weight, g_exc, g_inh, g_nmda);
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_error("fold kernels: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
    return EB_OK;
}

int fold_check(int64_t n, const int32_t *target, const int8_t *type, const float *weight, int64_t m) {
    if (n < 0 || m <= 0 || (n > 0 && (!target || !type || !weight))) { set_error("bad fold arguments"); return EB_ERR_ARG; }
    if (m > (int64_t)kScanBlock * kScanBlock) { set_error("fold: more than %d targets", kScanBlock * kScanBlock); return EB_ERR_ARG; }
    if (n >= (int64_t)UINT32_MAX) { set_error("fold: too many arrivals"); return EB_ERR_ARG; }
    return EB_OK;
}

}  // namespace

extern "C" int eb_fold_arrivals(void *stream, int64_t n, const int32_t *target, const int8_t *type,
                                const float *weight, const double *time, int64_t n_targets, float *g_exc,
                                float *g_inh, float *g_nmda) {
    int rc = fold_check(n, target, type, weight, n_targets);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    void *scratch = nullptr;
    const size_t bytes = fold_scratch_bytes(n, n_targets);
    cudaError_t e = cudaMallocAsync(&scratch, bytes, st);
    if (e != cudaSuccess) { set_error("cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e)); return EB_ERR_NOMEM; }
    rc = fold_enqueue(st, scratch, n, target, type, weight, time, n_targets, g_exc, g_inh, g_nmda);
    cudaFreeAsync(scratch, st);
    return rc;
}

// ------------------------------------------------------ allocation-free form --
// Some callers cannot allocate device memory while they run: a closed-loop
// (real-time) controller whose step deadline must not contain allocator calls,
// or a host engine that claims all device memory for itself at start-up.  This
// form of the op takes its scratch from a fixed array in the library's device
// image instead.  Every GPU that loads the library holds that array (about
// 7 MiB) until the process exits; it bounds one call to kNoAllocMaxArrivals
// arrivals and kNoAllocMaxTargets targets.  All calls share the one array and
// it keeps the previous call's contents: the counters that must start at zero
// are cleared at the start of every call, and two calls whose work overlaps on
// the GPU (different streams, or different host threads on the same device)
// race on it.
namespace {

constexpr int64_t kNoAllocMaxArrivals = 1 << 18;
constexpr int64_t kNoAllocMaxTargets = 1 << 18;
constexpr size_t kNoAllocScratchBytes =
    (((3 * (size_t)(kNoAllocMaxTargets + 1) + kScanBlock) * sizeof(uint32_t) + 255) & ~(size_t)255) +
    (size_t)kNoAllocMaxArrivals * sizeof(FoldRec);

static __device__ __align__(256) unsigned char g_fold_scratch[kNoAllocScratchBytes];

// The array's device address on each device, looked up once per device (with
// that device current); in host code g_fold_scratch only names a host-side
// stand-in, never the device memory.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices] = {};

int scratch_for_current_device(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error("cudaGetDevice: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
    if (dev < 0 || dev >= kMaxDevices) { set_error("device index %d above %d", dev, kMaxDevices - 1); return EB_ERR_ARG; }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fold_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(e));
            return EB_ERR_CUDA;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return EB_OK;
}

}  // namespace

extern "C" int eb_fold_arrivals_noalloc(void *stream, int64_t n, const int32_t *target, const int8_t *type,
                                        const float *weight, const double *time, int64_t n_targets,
                                        float *g_exc, float *g_inh, float *g_nmda) {
    int rc = fold_check(n, target, type, weight, n_targets);
    if (rc) return rc;
    if (n > kNoAllocMaxArrivals || n_targets > kNoAllocMaxTargets) {
        set_error("eb_fold_arrivals_noalloc: %lld arrivals / %lld targets exceed its fixed scratch "
                  "(at most %lld arrivals and %lld targets per call); use eb_fold_arrivals",
                  (long long)n, (long long)n_targets, (long long)kNoAllocMaxArrivals, (long long)kNoAllocMaxTargets);
        return EB_ERR_ARG;
    }
    void *scratch = nullptr;
    if ((rc = scratch_for_current_device(&scratch))) return rc;
    return fold_enqueue((cudaStream_t)stream, scratch, n, target, type, weight, time, n_targets, g_exc, g_inh,
                        g_nmda);
}
