// dem_sort.cu -- RadixSort(pData0, pData1, elements, keybits): the stable
// key/value radix sort that dempacking.cu:553-555 takes from the CUDA SDK
// (radixsort.cu, not in the reference).  LSD, 8-bit digits, ping-pong between
// the two buffers, result in pData0.  Per pass: block digit histograms ->
// device-wide scan (digit-major) -> stable scatter.  Stability inside a tile
// comes from processing the tile in 8 rounds of 256 items in index order and
// ranking equal digits with __match_any_sync inside each warp.
#include <mutex>
#include <vector>
#include "dem_common.cuh"
#include "dem_compat_state.h"

namespace dem {

namespace {
constexpr int kRsThreads = 256;
constexpr int kRsRounds = 8;
constexpr int kRsTile = kRsThreads * kRsRounds;
constexpr int kRsWarps = kRsThreads / 32;

__global__ void __launch_bounds__(kRsThreads) k_radix_hist(const uint2* __restrict__ in, uint n, int shift,
                                                           uint* __restrict__ hist, uint nb) {
    __shared__ uint cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint base = blockIdx.x * kRsTile;
#pragma unroll
    for (int e = 0; e < kRsRounds; e++) {
        uint idx = base + e * kRsThreads + threadIdx.x;
        if (idx < n) atomicAdd(&cnt[(in[idx].x >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * nb + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) k_radix_scatter(const uint2* __restrict__ in, uint2* __restrict__ out,
                                                              uint n, int shift, const uint* __restrict__ hist,
                                                              uint nb) {
    __shared__ uint run[256];
    __shared__ uint wc[kRsWarps][256];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    run[t] = hist[(size_t)t * nb + blockIdx.x];
    const uint lt = (1u << lane) - 1u;
    const uint base = blockIdx.x * kRsTile;
    for (int e = 0; e < kRsRounds; e++) {
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) wc[w][t] = 0;
        __syncthreads();
        const uint idx = base + e * kRsThreads + t;
        const bool valid = idx < n;
        uint2 kv = make_uint2(0u, 0u);
        uint d = 256u;
        if (valid) { kv = in[idx]; d = (kv.x >> shift) & 255u; }
        const uint peers = __match_any_sync(0xffffffffu, d);
        const uint rank = __popc(peers & lt);
        if (valid && lane == __ffs(peers) - 1) wc[warp][d] = __popc(peers);
        __syncthreads();
        uint acc = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) { uint c = wc[w][t]; wc[w][t] = acc; acc += c; }
        __syncthreads();
        if (valid) out[run[d] + wc[warp][d] + rank] = kv;
        __syncthreads();
        run[t] += acc;
        __syncthreads();
    }
}
}  // namespace

size_t radix_scratch_words(uint n) {
    uint nb = (n + kRsTile - 1) / kRsTile;
    if (nb < 1) nb = 1;
    return (size_t)256 * nb + scan_scratch_words((long long)256 * nb);
}

// Sort with caller-provided scratch of radix_scratch_words(n) uint32.
int radix_sort_pairs(uint2* d0, uint2* d1, uint n, uint keybits, uint* scratch, cudaStream_t s) {
    if (n <= 1) return DEM_OK;
    if (keybits == 0) return DEM_OK;
    if (keybits > 32) keybits = 32;
    const uint nb = (n + kRsTile - 1) / kRsTile;
    uint* hist = scratch;
    uint* tmp = scratch + (size_t)256 * nb;
    const int passes = (int)((keybits + 7) / 8);
    uint2* src = d0;
    uint2* dst = d1;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        k_radix_hist<<<nb, kRsThreads, 0, s>>>(src, n, shift, hist, nb);
        DEM_LAUNCH_CHECK();
        int rc = exclusive_scan_u32(hist, hist, (long long)256 * nb, nullptr, tmp, s);
        if (rc) return rc;
        k_radix_scatter<<<nb, kRsThreads, 0, s>>>(src, dst, n, shift, hist, nb);
        DEM_LAUNCH_CHECK();
        uint2* t = src; src = dst; dst = t;
    }
    if (src != d0) DEM_CUDA_TRY(cudaMemcpyAsync(d0, src, (size_t)n * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
    return DEM_OK;
}

}  // namespace dem

extern "C" int RadixSort(KeyValuePair* pData0, KeyValuePair* pData1, unsigned int elements, unsigned int keybits) {
    if (elements > 1 && (!pData0 || !pData1)) return dem::fail(DEM_ERR_ARG, "RadixSort: null buffer");
    if (elements <= 1) return DEM_OK;
    dem::CompatDevice* cd = nullptr;
    int rc = dem::compat_device(&cd);
    if (rc) return rc;
    uint* scratch = nullptr;
    rc = dem::compat_scratch(cd, dem::radix_scratch_words(elements), &scratch);
    if (rc) return rc;
    return dem::radix_sort_pairs(reinterpret_cast<uint2*>(pData0), reinterpret_cast<uint2*>(pData1), elements, keybits,
                                 scratch, dem::compat_stream());
}

// ---------------------------------------------------------------------------
// RadixSortNoAlloc: the same stable sort for callers that must not allocate
// device memory, e.g. a host loop that owns all of HBM through its own pool
// allocator, or a latency-critical loop in which a first-call cudaMalloc (and
// the device synchronisation it may cause) is not acceptable.  Its scratch
// (digit histograms and scan carries) lives in the fixed device array below,
// sized for at most kNoAllocMaxRecords records (about 2 MiB); every GPU that
// loads this library holds that array until the process exits.
//
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress while that device is current (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory).  Under
// CUDA's lazy module loading that call may be the one that loads this
// library's device code, which reserves device memory: make the first call
// during set-up, before any stream capture; later calls allocate nothing.  All calls share the one array,
// which keeps the contents of the last call: every histogram word is written
// before it is read, so nothing needs clearing, but two calls that overlap on
// the GPU (different streams, or different host threads on the same device)
// race on it and must be serialised by the caller.
namespace dem {
namespace {
constexpr unsigned kNoAllocMaxRecords = 1u << 22;                        // 4,194,304
constexpr size_t kNoAllocHistWords = (size_t)256 * (kNoAllocMaxRecords / kRsTile);
constexpr size_t kNoAllocWords = kNoAllocHistWords + kNoAllocHistWords / 4096 + 256;
__device__ __align__(256) unsigned int g_noalloc_scratch[kNoAllocWords];

std::mutex g_noalloc_mu;
std::vector<std::pair<int, uint*>> g_noalloc_addr;   // (device, device address of g_noalloc_scratch)

int noalloc_scratch(uint** out) {
    int dev = 0;
    DEM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    for (auto& e : g_noalloc_addr)
        if (e.first == dev) { *out = e.second; return DEM_OK; }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    g_noalloc_addr.emplace_back(dev, (uint*)p);
    *out = (uint*)p;
    return DEM_OK;
}
}  // namespace
}  // namespace dem

extern "C" int RadixSortNoAlloc(KeyValuePair* pData0, KeyValuePair* pData1, unsigned int elements,
                                unsigned int keybits) {
    if (elements > dem::kNoAllocMaxRecords)
        return dem::fail(DEM_ERR_ARG, "RadixSortNoAlloc: %u records exceed the fixed scratch limit of %u records",
                         elements, dem::kNoAllocMaxRecords);
    if (elements > 1 && (!pData0 || !pData1)) return dem::fail(DEM_ERR_ARG, "RadixSortNoAlloc: null buffer");
    if (elements <= 1) return DEM_OK;
    if (dem::radix_scratch_words(elements) > dem::kNoAllocWords)
        return dem::fail(DEM_ERR_ARG, "RadixSortNoAlloc: scratch sizing error");
    uint* scratch = nullptr;
    int rc = dem::noalloc_scratch(&scratch);
    if (rc) return rc;
    return dem::radix_sort_pairs(reinterpret_cast<uint2*>(pData0), reinterpret_cast<uint2*>(pData1), elements, keybits,
                                 scratch, dem::compat_stream());
}
