// dem_scan.cu -- device-wide exclusive prefix sum of uint32 (cell counts,
// per-particle pair counts, radix digit histograms).  Three launches:
// tile reduce -> scan of tile sums (one CTA per array) -> tile scan + offset.
// 256 threads x 16 items per tile; items are loaded as uint4 when aligned.
// Up to three arrays of the same length are scanned by the same three
// launches (blockIdx.y selects the array).
#include "dem_common.cuh"

namespace dem {

namespace {
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint warp_incl_scan(uint v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total.
__device__ __forceinline__ uint block_excl_scan(uint v, uint* smem_warp, uint& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint inc = warp_incl_scan(v);
    if (lane == 31) smem_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint w = lane < (kScanThreads / 32) ? smem_warp[lane] : 0u;
        uint wi = warp_incl_scan(w);
        if (lane < (kScanThreads / 32)) smem_warp[lane] = wi - w;
        if (lane == (kScanThreads / 32) - 1) smem_warp[kScanThreads / 32] = wi;
    }
    __syncthreads();
    uint r = smem_warp[warp] + inc - v;
    total = smem_warp[kScanThreads / 32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ void load_items(const uint* in, long long n, long long base, uint (&it)[kScanItems]) {
    const long long b = base + (long long)threadIdx.x * kScanItems;
    if (b + kScanItems <= n && ((reinterpret_cast<uintptr_t>(in + b) & 15) == 0)) {
        const uint4* p = reinterpret_cast<const uint4*>(in + b);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) {
            uint4 v = p[q];
            it[4 * q] = v.x; it[4 * q + 1] = v.y; it[4 * q + 2] = v.z; it[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < kScanItems; q++) it[q] = (b + q < n) ? in[b + q] : 0u;
    }
}

constexpr int kMaxArrays = 3;
struct ScanSet {
    const uint* in[kMaxArrays];
    uint* out[kMaxArrays];
    uint* total[kMaxArrays];
    uint* sums[kMaxArrays];
};

__global__ void __launch_bounds__(kScanThreads) k_tile_reduce(ScanSet a, long long n) {
    __shared__ uint sw[kScanThreads / 32 + 1];
    pdl_wait();
    pdl_trigger();
    const int y = blockIdx.y;
    uint it[kScanItems];
    load_items(a.in[y], n, (long long)blockIdx.x * kScanTile, it);
    uint s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; q++) s += it[q];
    uint tot;
    block_excl_scan(s, sw, tot);
    if (threadIdx.x == 0) a.sums[y][blockIdx.x] = tot;
}

// One CTA per array scans its tile sums in chunks of 256.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(ScanSet a, long long nt) {
    __shared__ uint sw[kScanThreads / 32 + 1];
    pdl_wait();
    pdl_trigger();
    uint* sums = a.sums[blockIdx.y];
    uint carry = 0;
    for (long long base = 0; base < nt; base += kScanThreads) {
        long long i = base + threadIdx.x;
        uint v = i < nt ? sums[i] : 0u;
        uint tot;
        uint e = block_excl_scan(v, sw, tot);
        if (i < nt) sums[i] = e + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && a.total[blockIdx.y]) *a.total[blockIdx.y] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_scan(ScanSet a, long long n) {
    __shared__ uint sw[kScanThreads / 32 + 1];
    pdl_wait();
    pdl_trigger();
    const int y = blockIdx.y;
    const uint* in = a.in[y];
    uint* out = a.out[y];
    uint it[kScanItems];
    const long long base = (long long)blockIdx.x * kScanTile;
    load_items(in, n, base, it);
    uint s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; q++) s += it[q];
    uint tot;
    uint run = block_excl_scan(s, sw, tot) + a.sums[y][blockIdx.x];
    const long long b = base + (long long)threadIdx.x * kScanItems;
    uint o[kScanItems];
#pragma unroll
    for (int q = 0; q < kScanItems; q++) { o[q] = run; run += it[q]; }
    if (b + kScanItems <= n && ((reinterpret_cast<uintptr_t>(out + b) & 15) == 0)) {
        uint4* p = reinterpret_cast<uint4*>(out + b);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) p[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < kScanItems; q++)
            if (b + q < n) out[b + q] = o[q];
    }
}

// pdl: the three launches are programmatic (each kernel waits for its
// predecessor before it touches memory, so only the launch latency overlaps);
// for a scan that follows a kernel on the stream
int scan_set(ScanSet a, int narr, long long n, cudaStream_t s, bool pdl) {
    const long long nt = (n + kScanTile - 1) / kScanTile;
    DEM_CUDA_TRY(launch_ex(k_tile_reduce, dim3((unsigned)nt, narr), dim3(kScanThreads), s, pdl, a, n));
    DEM_CUDA_TRY(launch_ex(k_scan_sums, dim3(1, narr), dim3(kScanThreads), s, pdl, a, nt));
    DEM_CUDA_TRY(launch_ex(k_tile_scan, dim3((unsigned)nt, narr), dim3(kScanThreads), s, pdl, a, n));
    return DEM_OK;
}
}  // namespace

size_t scan_scratch_words(long long n) {
    long long nt = (n + kScanTile - 1) / kScanTile;
    return (size_t)(nt < 1 ? 1 : nt) + 4;
}

int exclusive_scan_u32(const uint* in, uint* out, long long n, uint* total, uint* tmp, cudaStream_t s, bool pdl) {
    const uint* ins[1] = {in};
    uint* outs[1] = {out};
    uint* tots[1] = {total};
    return exclusive_scan_multi_u32(1, ins, outs, tots, n, tmp, s, pdl);
}

int exclusive_scan_multi_u32(int narr, const uint* const* in, uint* const* out, uint* const* total, long long n,
                             uint* tmp, cudaStream_t s, bool pdl) {
    if (narr < 1 || narr > kMaxArrays) return fail(DEM_ERR_ARG, "exclusive_scan_multi_u32: %d arrays", narr);
    if (n <= 0) {
        for (int a = 0; a < narr; a++)
            if (total[a]) DEM_CUDA_TRY(cudaMemsetAsync(total[a], 0, sizeof(uint), s));
        return DEM_OK;
    }
    ScanSet set = {};
    const size_t words = scan_scratch_words(n);
    for (int a = 0; a < narr; a++) {
        set.in[a] = in[a];
        set.out[a] = out[a];
        set.total[a] = total[a];
        set.sums[a] = tmp + a * words;
    }
    return scan_set(set, narr, n, s, pdl);
}

}  // namespace dem
