// dmolp_metrics_noalloc: the fused edge-cut / balance reduction for callers that cannot let a library
// allocate device memory -- for instance a process whose GPU memory is owned by another allocator (a
// framework's caching pool, or a server that reserves all memory at start-up) and where cudaMalloc /
// cudaFree from a library call are not allowed.  The caller passes its graph and labels as device
// pointers and receives the results in host memory; the only scratch (per-part counters, the cut counter
// and an error flag) is the file-scope device array below, of fixed size.
//
// Every GPU that loads the library holds that array until the process exits.  All calls on a device
// share it and it keeps the last call's contents: each call clears it before use, and calls that overlap
// on the GPU (different host threads or streams at the same time) race on it.  The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) with that device current; make that first
// call before any stream capture.  The address is cached for the life of the process: a cudaDeviceReset
// after the first call on a device is not supported.  The caller's current device is restored on return.
// A neighbour id outside [0, nv) or a row whose end offset is below its start is flagged by the kernel and
// skipped (DMOLP_ERR_ARG), never read; offsets[nv] itself cannot be checked (the call has no arc count).
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dmolp_b200.h"
#include "common.cuh"

namespace dmolp {
void set_last_error(const std::string &msg);  // dmolp_cabi.cu
}

namespace {

constexpr int kMaxDevices = 64;
constexpr unsigned long long kBadLabel = 1ull, kBadGraph = 2ull;  // flag bits

// [0, K): vertex counts, [K, 2K): intra-part arcs, [2K]: cut arcs, [2K+1]: flags (kBadLabel | kBadGraph)
static __device__ __align__(256) unsigned long long g_noalloc_scratch[2 * DMOLP_NOALLOC_MAX_K + 2];

unsigned long long *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

int fail(int code, const std::string &msg) {
    dmolp::set_last_error(msg);  // read back with dmolp_last_error()
    return code;
}

// Puts the caller's current device back when the call returns.
struct DeviceRestore {
    int dev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    }
    ~DeviceRestore() {
        if (dev >= 0) cudaSetDevice(dev);
    }
};

// Warp per vertex: label count of the vertex, same-label and different-label arcs of its row.
__global__ void k_metrics_noalloc(const int64_t *__restrict__ off, const int32_t *__restrict__ col,
                                  const int32_t *__restrict__ label, int64_t nv, int k,
                                  unsigned long long *__restrict__ scratch) {
    extern __shared__ unsigned long long sacc[];  // [2k]
    for (int p = threadIdx.x; p < 2 * k; p += blockDim.x) sacc[p] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long cut = 0;
    bool bad = false, bad_graph = false;
    for (int64_t v = gw; v < nv; v += nw) {
        const int lv = label[v];
        unsigned int same = 0, diff = 0;
        const int64_t s = off[v], e = off[v + 1];
        bad_graph |= e < s;  // such a row is skipped (the loop below does not run)
        for (int64_t j = s + lane; j < e; j += 32) {
            const int u = col[j];
            if ((unsigned long long)(unsigned)u >= (unsigned long long)nv) {  // flagged, never read
                bad_graph = true;
                continue;
            }
            const int lu = label[u];
            bad |= (unsigned)lu >= (unsigned)k;
            same += (lu == lv);
            diff += (lu != lv);
        }
        for (int o = 16; o > 0; o >>= 1) {
            same += __shfl_xor_sync(DMOLP_FULL_MASK, same, o);
            diff += __shfl_xor_sync(DMOLP_FULL_MASK, diff, o);
        }
        if (lane == 0) {
            cut += diff;
            if ((unsigned)lv < (unsigned)k) {
                atomicAdd(&sacc[lv], 1ull);
                if (same) atomicAdd(&sacc[k + lv], (unsigned long long)same);
            } else {
                bad = true;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) cut += __shfl_xor_sync(DMOLP_FULL_MASK, cut, o);
    if (lane == 0 && cut) atomicAdd(&scratch[2 * k], cut);
    const bool any_bad = __any_sync(DMOLP_FULL_MASK, bad), any_graph = __any_sync(DMOLP_FULL_MASK, bad_graph);
    if (lane == 0 && (any_bad || any_graph))
        atomicOr(&scratch[2 * k + 1], (any_bad ? kBadLabel : 0ull) | (any_graph ? kBadGraph : 0ull));
    __syncthreads();
    for (int p = threadIdx.x; p < 2 * k; p += blockDim.x)
        if (sacc[p]) atomicAdd(&scratch[p], sacc[p]);
}

}  // namespace

extern "C" {

int dmolp_metrics_noalloc(int device, int64_t nv, const int64_t *offsets_device, const int32_t *indices_device,
                          const int32_t *labels_device, int k, void *stream, int64_t *edge_cut,
                          int64_t *vertex_counts, int64_t *edge_counts) {
    if (k < 1 || k > DMOLP_NOALLOC_MAX_K)
        return fail(DMOLP_ERR_ARG, "k must be in [1, " + std::to_string(DMOLP_NOALLOC_MAX_K) +
                                       "]: the no-allocation scratch array holds that many parts");
    if (nv < 0 || nv >= (1ll << 31) || (nv > 0 && (!offsets_device || !indices_device || !labels_device)) ||
        !edge_cut)
        return fail(DMOLP_ERR_ARG, "bad sizes or null pointers");
    if (device < 0 || device >= kMaxDevices) return fail(DMOLP_ERR_ARG, "device index out of range");
    const DeviceRestore restore;  // the caller's current device comes back on every return path
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    unsigned long long *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[device]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(DMOLP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_addr[device] = (unsigned long long *)p;
        }
        scratch = g_scratch_addr[device];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t used = (2 * (size_t)k + 2) * sizeof(unsigned long long);
    e = cudaMemsetAsync(scratch, 0, used, s);  // the array keeps the previous call's counts
    if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    if (nv > 0) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        k_metrics_noalloc<<<sms * 4, 256, 2 * k * sizeof(unsigned long long), s>>>(
            offsets_device, indices_device, labels_device, nv, k, scratch);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    unsigned long long host[2 * DMOLP_NOALLOC_MAX_K + 2];
    e = cudaMemcpyAsync(host, scratch, used, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(DMOLP_ERR_CUDA, std::string("copy back: ") + cudaGetErrorString(e));
    const unsigned long long arcs = host[2 * k];
    *edge_cut = (int64_t)(arcs >> 1);
    for (int p = 0; p < k; ++p) {
        if (vertex_counts) vertex_counts[p] = (int64_t)host[p];
        if (edge_counts) edge_counts[p] = (int64_t)(host[k + p] / 2);
    }
    if (host[2 * k + 1] & kBadGraph)
        return fail(DMOLP_ERR_ARG, "neighbour id outside [0, nv) or a row whose end offset is below its start");
    if (host[2 * k + 1] || (arcs & 1ull))
        return fail(DMOLP_ERR_BAD_LABELS, "label outside [0,k) or odd cut-arc count");
    return DMOLP_OK;
}

}  // extern "C"
