// dem_common.cuh -- small vector type, error plumbing and launch helpers
// shared by the library's translation units.  Host+device.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include <nvtx3/nvToolsExt.h>
#include "dem_b200.h"

#define DEM_HD __host__ __device__ __forceinline__

namespace dem {

typedef unsigned int uint;
static constexpr uint kEmpty = 0xffffffffu;

// ---------------------------------------------------------------- 3-vectors
template <typename T> struct V3 { T x, y, z; };

template <typename T> DEM_HD V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T> DEM_HD V3<T> zero3() { return V3<T>{T(0), T(0), T(0)}; }
template <typename T> DEM_HD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> DEM_HD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> DEM_HD V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <typename T> DEM_HD V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> DEM_HD V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> DEM_HD void operator+=(V3<T>& a, V3<T> b) { a.x += b.x; a.y += b.y; a.z += b.z; }
template <typename T> DEM_HD void operator-=(V3<T>& a, V3<T> b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
template <typename T> DEM_HD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> DEM_HD V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename To, typename From> DEM_HD V3<To> cvt(V3<From> a) {
    return {(To)a.x, (To)a.y, (To)a.z};
}

DEM_HD float dsqrt(float x) { return sqrtf(x); }
DEM_HD double dsqrt(double x) { return sqrt(x); }

// 16-byte aligned 4-vector of the working precision (float4-like for FP32,
// two 16-byte words for FP64).
template <typename T> struct alignas(16) R4 { T x, y, z, w; };

// ---------------------------------------------------------------- errors
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define DEM_CUDA_TRY(call)                                                           \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) return ::dem::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)
#define DEM_LAUNCH_CHECK() DEM_CUDA_TRY(cudaGetLastError())

// NVTX range over a host scope (re-list, window, upload, adjoint phases):
// a profiler attached to the process shows where the host enqueues each
// phase; without one the calls do nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

inline unsigned grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : g);
}

// Programmatic dependent launch (sm_90+).  A kernel launched with
// programmatic stream serialization may start while its predecessor in the
// stream is still running; pdl_wait() returns once every predecessor has
// completed and its writes are visible (immediately when the kernel was
// launched normally).  pdl_trigger() lets the successor be scheduled as soon
// as every block of this kernel has started.  Before pdl_wait() a kernel may
// read only data written before the last normally launched kernel.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
cudaError_t launch_ex(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, bool pdl, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Device-wide exclusive scan of uint32 (3 launches, no host sync).
// out[i] = sum_{t<i} in[i]; if total != nullptr, *total (device) = full sum.
// out may alias in.  Scratch: tmp with scan_scratch_words(n) uint32.
size_t scan_scratch_words(long long n);
int exclusive_scan_u32(const uint* in, uint* out, long long n, uint* total, uint* tmp, cudaStream_t s,
                       bool pdl = false);
// Up to three arrays of length n in the same three launches; tmp holds
// narr * scan_scratch_words(n) uint32.  Outputs may alias their inputs.
int exclusive_scan_multi_u32(int narr, const uint* const* in, uint* const* out, uint* const* total, long long n,
                             uint* tmp, cudaStream_t s, bool pdl = false);

}  // namespace dem
