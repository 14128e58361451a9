// dem_compat.cu -- the reference-compatible entry points (the extern "C"
// wrapper set of particleSystem.cu:13-424) on sm_100a, FP64, reference data
// layout (xyz-interleaved double arrays).  Kernels follow the reference's
// decomposition -- one thread per particle for hash / neighbour rows / gather
// / wall / update, one thread per candidate pair for the force -- with the
// missing kernels and force laws written from their call contracts.
#include <cstdio>
#include <mutex>
#include <vector>
#include "dem_common.cuh"
#include "dem_compat_state.h"
#include "dem_law.cuh"

namespace dem {

enum : uint { kStatusCapacity = 1u, kStatusNonfinite = 2u };

__constant__ LawParams<double> c_pp;      // Par  (neiglist.cu:48)
__constant__ LawParams<double> c_pw;      // ParW (neiglist.cu:49)
__constant__ double c_cua = 1.0;          // neiglist.cu:27
__constant__ double c_cub = 1.55;         // neiglist.cu:28

static cudaStream_t g_stream = 0;
static std::mutex g_mu;
static std::vector<CompatDevice*> g_devs;

cudaStream_t compat_stream() { return g_stream; }

int compat_device(CompatDevice** out) {
    int dev = 0;
    DEM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    for (CompatDevice* c : g_devs)
        if (c->device == dev) { *out = c; return DEM_OK; }
    CompatDevice* c = new CompatDevice();
    c->device = dev;
    DEM_CUDA_TRY(cudaMalloc(&c->words, 16 * sizeof(uint)));
    DEM_CUDA_TRY(cudaMemsetAsync(c->words, 0, 16 * sizeof(uint), g_stream));   // ordered before the wrappers
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    DEM_CUDA_TRY(cudaMallocHost(&c->host_words, 16 * sizeof(uint)));
    g_devs.push_back(c);
    *out = c;
    return DEM_OK;
}

int compat_scratch(CompatDevice* cd, size_t words, uint** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cd->scratch_words < words) {
        if (cd->scratch) {
            DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
            DEM_CUDA_TRY(cudaFree(cd->scratch));
        }
        cd->scratch = nullptr;
        size_t w = words + words / 4 + 1024;
        DEM_CUDA_TRY(cudaMalloc(&cd->scratch, w * sizeof(uint)));
        cd->scratch_words = w;
    }
    *out = cd->scratch;
    return DEM_OK;
}

namespace {
constexpr int kBlock = 256;

// calcGridPos + calcGridAddress (neiglist.cu:54-75).  The clamp there is
// max(0, min(int, uint-1)); CUDA's min(int, unsigned int) compares as unsigned,
// so a negative coordinate maps to gridSize-1.  Reproduced as is.
__device__ __forceinline__ void ref_cell(const double3 p, const uint3 gs, const double3 cs, const double3 o,
                                         uint& gx, uint& gy, uint& gz) {
    int ix = (int)floor((p.x - o.x) / cs.x);
    int iy = (int)floor((p.y - o.y) / cs.y);
    int iz = (int)floor((p.z - o.z) / cs.z);
    gx = umin((uint)ix, gs.x - 1u);
    gy = umin((uint)iy, gs.y - 1u);
    gz = umin((uint)iz, gs.z - 1u);
}

__global__ void k_calc_hash(int n, const double3* __restrict__ pos, uint2* __restrict__ hash, uint3 gs, double3 cs,
                            double3 o) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint gx, gy, gz;
        ref_cell(pos[i], gs, cs, o, gx, gy, gz);
        hash[i] = make_uint2(gz * gs.y * gs.x + gy * gs.x + gx, (uint)i);
    }
}

__global__ void k_find_cell_start(const uint2* __restrict__ hash, uint* __restrict__ cellStart, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        uint c = hash[i].x;
        if (i == 0 || c != hash[i - 1].x) cellStart[c] = (uint)i;
    }
}

__device__ __forceinline__ void isort(uint* a, uint len) {
    for (uint s = 1; s < len; s++) {
        uint v = a[s];
        uint t = s;
        while (t > 0 && a[t - 1] > v) { a[t] = a[t - 1]; t--; }
        a[t] = v;
    }
}

// neighborarrayD (called at particleSystem.cu:85; not in the reference):
// 27-cell walk from i's cell, cell members from cellStart until the key
// changes; candidate when |x_i - x_j|^2 < cub^2.
__global__ void k_neighbor_array(int n, const double3* __restrict__ pos, const uint2* __restrict__ hash,
                                 const uint* __restrict__ cellStart, uint3 gs, double3 cs, double3 o, int maxppc,
                                 uint* __restrict__ Anei, uint* __restrict__ njgi, uint* __restrict__ njli,
                                 uint* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double3 pi = pos[i];
    uint gx, gy, gz;
    ref_cell(pi, gs, cs, o, gx, gy, gz);
    const double cub2 = c_cub * c_cub;
    uint* row = Anei + (size_t)i * maxppc;
    uint nu = 0, nl = 0;
    // pass 1: count
    for (int dz = -1; dz <= 1; dz++) {
        int z = (int)gz + dz;
        if (z < 0 || z >= (int)gs.z) continue;
        for (int dy = -1; dy <= 1; dy++) {
            int y = (int)gy + dy;
            if (y < 0 || y >= (int)gs.y) continue;
            for (int dx = -1; dx <= 1; dx++) {
                int x = (int)gx + dx;
                if (x < 0 || x >= (int)gs.x) continue;
                uint c = ((uint)z * gs.y + (uint)y) * gs.x + (uint)x;
                uint t = cellStart[c];
                if (t == kEmpty) continue;
                for (; t < (uint)n; t++) {
                    uint2 h = hash[t];
                    if (h.x != c) break;
                    if (h.y == (uint)i) continue;
                    double3 pj = pos[h.y];
                    double ddx = pj.x - pi.x, ddy = pj.y - pi.y, ddz = pj.z - pi.z;
                    double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    if (d2 < cub2) {
                        if (h.y > (uint)i) nu++; else nl++;
                    }
                }
            }
        }
    }
    uint cap = (uint)maxppc;
    uint nuw = nu < cap ? nu : cap;
    uint nlw = nl < cap - nuw ? nl : cap - nuw;
    if (nu + nl > cap) atomicOr(status, kStatusCapacity);
    // pass 2: write j>i at [0, nuw) and j<i at [nuw, nuw+nlw)
    uint wu = 0, wl = 0;
    for (int dz = -1; dz <= 1; dz++) {
        int z = (int)gz + dz;
        if (z < 0 || z >= (int)gs.z) continue;
        for (int dy = -1; dy <= 1; dy++) {
            int y = (int)gy + dy;
            if (y < 0 || y >= (int)gs.y) continue;
            for (int dx = -1; dx <= 1; dx++) {
                int x = (int)gx + dx;
                if (x < 0 || x >= (int)gs.x) continue;
                uint c = ((uint)z * gs.y + (uint)y) * gs.x + (uint)x;
                uint t = cellStart[c];
                if (t == kEmpty) continue;
                for (; t < (uint)n; t++) {
                    uint2 h = hash[t];
                    if (h.x != c) break;
                    if (h.y == (uint)i) continue;
                    double3 pj = pos[h.y];
                    double ddx = pj.x - pi.x, ddy = pj.y - pi.y, ddz = pj.z - pi.z;
                    double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                    if (d2 < cub2) {
                        if (h.y > (uint)i) { if (wu < nuw) row[wu++] = h.y; }
                        else { if (wl < nlw) row[nuw + wl++] = h.y; }
                    }
                }
            }
        }
    }
    isort(row, nuw);
    isort(row + nuw, nlw);
    njgi[i] = nuw;
    njli[i] = nlw;
}

// b[i] += a[i] (addTwoArraysD, neiglist.cu:122-130): exclusive -> inclusive scan.
__global__ void k_add_two(uint* b, const uint* a, uint n) {
    uint i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] += a[i];
}

// pairlistD (called at particleSystem.cu:172; not in the reference).
__global__ void k_pairlist(uint n, const uint* __restrict__ sjgi, const uint* __restrict__ oldsjgi,
                           const uint* __restrict__ oldLn, const uint* __restrict__ Anei, const uint* __restrict__ njgi,
                           const uint* __restrict__ njli, const double3* __restrict__ olddispt,
                           const double* __restrict__ oldfricp, int maxppc, size_t capP, uint* __restrict__ Aref,
                           uint* __restrict__ Lp, uint* __restrict__ Ln, double3* __restrict__ dispt,
                           double* __restrict__ fricp) {
    uint i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint ngi = njgi[i];
    const uint base = sjgi[i] - ngi;
    uint os = i > 0 ? oldsjgi[i - 1] : 0u, oe = oldsjgi[i];
    if ((size_t)oe > capP) oe = (uint)capP;
    if (os > oe) os = oe;
    const uint* row = Anei + (size_t)i * maxppc;
    uint* aref = Aref + (size_t)i * maxppc;
    for (uint s = 0; s < ngi; s++) {
        const uint k = base + s, j = row[s];
        if ((size_t)k >= capP) break;   // caller sized Lp/Ln below the list (maxCn < row length)
        Lp[k] = i;
        Ln[k] = j;
        aref[s] = k;
        double3 h = make_double3(0.0, 0.0, 0.0);
        double fr = 0.0;
        for (uint t = os; t < oe; t++) {
            if (oldLn[t] == j) { h = olddispt[t]; fr = oldfricp[t]; break; }
        }
        dispt[k] = h;
        fricp[k] = fr;
    }
    const uint nli = njli[i];
    for (uint s = ngi; s < ngi + nli; s++) {
        const uint j = row[s];
        uint kk = kEmpty;
        const uint* rowj = Anei + (size_t)j * maxppc;
        const uint ngj = njgi[j];
        for (uint t = 0; t < ngj; t++)
            if (rowj[t] == i) { kk = sjgi[j] - ngj + t; break; }
        aref[s] = kk;
    }
}

// calculateforcepairD (neiglist.cu:156-233) with the contact law.
__global__ void k_force_pair(uint total, const double3* __restrict__ pos, const double3* __restrict__ pdis,
                             const double3* __restrict__ angv, const double* __restrict__ rad,
                             const double* __restrict__ rmass, const uint* __restrict__ Lp, const uint* __restrict__ Ln,
                             uint* __restrict__ oldLn, double3* __restrict__ dispt, double* __restrict__ fricp,
                             double3* __restrict__ olddispt, double* __restrict__ oldfricp, double inv_dt,
                             double3* __restrict__ forcepair, double3* __restrict__ torqpairi,
                             double3* __restrict__ torqpairj, uint* __restrict__ contactpair) {
    uint k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    const uint i = Lp[k], j = Ln[k];
    const double3 xi = pos[i], xj = pos[j];
    const double ri = rad[i], rj = rad[j];
    V3<double> D = mk(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z);
    const double dist = sqrt(dot(D, D));
    const double delta = (ri + rj) - dist;
    double3 hin = dispt[k];
    V3<double> h = mk(hin.x, hin.y, hin.z);
    const double3 z3 = make_double3(0.0, 0.0, 0.0);
    if (delta > 0.0 && dist > 0.0) {
        const V3<double> n = mk(D.x / dist, D.y / dist, D.z / dist);
        const double mi = rmass[i], mj = rmass[j];
        const double rstar = ri * rj / (ri + rj), mstar = mi * mj / (mi + mj);
        const double3 ai3 = angv[i], aj3 = angv[j], di3 = pdis[i], dj3 = pdis[j];
        const V3<double> ai = mk(ai3.x, ai3.y, ai3.z), aj = mk(aj3.x, aj3.y, aj3.z);
        const V3<double> U = mk(dj3.x - di3.x, dj3.y - di3.y, dj3.z - di3.z) - cross(ri * ai + rj * aj, n);
        V3<double> Fi, Ft, Mr;
        contact_law<double>(delta, n, rstar, mstar, U, ai - aj, h, inv_dt, c_pp, Fi, Ft, Mr);
        const V3<double> nxf = cross(n, Ft);
        const V3<double> Ti = ri * nxf + Mr, Tj = rj * nxf - Mr;
        const double fr = sqrt(dot(Ft, Ft));
        forcepair[k] = make_double3(Fi.x, Fi.y, Fi.z);
        torqpairi[k] = make_double3(Ti.x, Ti.y, Ti.z);
        torqpairj[k] = make_double3(Tj.x, Tj.y, Tj.z);
        dispt[k] = make_double3(h.x, h.y, h.z);
        fricp[k] = fr;
        contactpair[k] = 1u;
        olddispt[k] = make_double3(h.x, h.y, h.z);
        oldfricp[k] = fr;
    } else {
        forcepair[k] = z3;
        torqpairi[k] = z3;
        torqpairj[k] = z3;
        dispt[k] = z3;
        fricp[k] = 0.0;
        contactpair[k] = 0u;
        olddispt[k] = z3;
        oldfricp[k] = 0.0;
    }
    oldLn[k] = j;
}

// sumallforceiD (called at particleSystem.cu:262; not in the reference).
__global__ void k_sum_force(int n, int maxppc, const uint* __restrict__ njgi, const uint* __restrict__ njli,
                            const double3* __restrict__ forcepair, const double3* __restrict__ torqpairi,
                            const double3* __restrict__ torqpairj, const uint* __restrict__ contactpair,
                            const uint* __restrict__ Aref, double3* __restrict__ forcei, double3* __restrict__ torquei,
                            uint* __restrict__ contacti) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
    uint cnt = 0;
    const uint ng = njgi[i], nt = ng + njli[i];
    const uint* row = Aref + (size_t)i * maxppc;
    for (uint s = 0; s < nt; s++) {
        const uint k = row[s];
        if (k == kEmpty) continue;
        const double3 f = forcepair[k];
        if (s < ng) {
            const double3 t = torqpairi[k];
            fx += f.x; fy += f.y; fz += f.z; tx += t.x; ty += t.y; tz += t.z;
        } else {
            const double3 t = torqpairj[k];
            fx -= f.x; fy -= f.y; fz -= f.z; tx += t.x; ty += t.y; tz += t.z;
        }
        cnt += contactpair[k];
    }
    forcei[i] = make_double3(fx, fy, fz);
    torquei[i] = make_double3(tx, ty, tz);
    contacti[i] = cnt;
}

// calculateforceiwD (neiglist.cu:238-306) with the wall law.
__global__ void k_force_wall(int n, double3 ws, const double3* __restrict__ pos, const double3* __restrict__ pdis,
                             const double3* __restrict__ angv, const double* __restrict__ rad,
                             const double* __restrict__ rmass, double inv_dt, uint total, double3* __restrict__ disptw,
                             double* __restrict__ fricpw, double3* __restrict__ forcei,
                             double3* __restrict__ torquei) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<double> F = zero3<double>(), T = zero3<double>();
    if (total != 0) {
        const double3 f = forcei[i], t = torquei[i];
        F = mk(f.x, f.y, f.z);
        T = mk(t.x, t.y, t.z);
    }
    const double m = rmass[i], r = rad[i];
    F.z += -m;
    const double3 x3 = pos[i], d3 = pdis[i], a3 = angv[i], h3 = disptw[i];
    V3<double> h = mk(h3.x, h3.y, h3.z);
    V3<double> Fw = zero3<double>(), Tw = zero3<double>();
    double fr = 0.0;
    const int hit = wall_contacts<double>(ws.x * 0.5, ws.y * 0.5, mk(x3.x, x3.y, x3.z), mk(d3.x, d3.y, d3.z),
                                          mk(a3.x, a3.y, a3.z), r, m, h, inv_dt, c_pw, Fw, Tw, &fr);
    if (hit) {
        F += Fw;
        T += Tw;
        disptw[i] = make_double3(h.x, h.y, h.z);
        fricpw[i] = fr;
    } else {
        disptw[i] = make_double3(0.0, 0.0, 0.0);
        fricpw[i] = 0.0;
    }
    forcei[i] = make_double3(F.x, F.y, F.z);
    torquei[i] = make_double3(T.x, T.y, T.z);
}

// updatepositionD (neiglist.cu:308-409), adamp = bdamp = 1.  The block
// maxima of the reference (partials reduced on the host) become one atomic
// per block into device words: iall and the bit pattern of max(0, max z)
// (non-negative doubles order like their bit patterns).
__global__ void k_update(int n, double3* __restrict__ pos, double3* __restrict__ pdis, double3* __restrict__ angv,
                         const double* __restrict__ rmass, const double* __restrict__ inert,
                         const double3* __restrict__ forcei, const double3* __restrict__ torquei,
                         double3* __restrict__ qi, double dt, uint* words) {
    __shared__ unsigned long long smz[kBlock / 32];
    __shared__ uint sall[kBlock / 32];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mz = 0.0;
    uint flag = 0;
    if (i < n) {
        const double ann = 0.5 * (c_cub - c_cua);
        double3 p = pos[i], d = pdis[i], a = angv[i], q = qi[i];
        const double3 f = forcei[i], t = torquei[i];
        const double m = rmass[i], I = inert[i];
        d.x = d.x + f.x * dt * dt / m;
        d.y = d.y + f.y * dt * dt / m;
        d.z = d.z + f.z * dt * dt / m;
        p.x += d.x; p.y += d.y; p.z += d.z;
        q.x += d.x; q.y += d.y; q.z += d.z;
        // single-precision length (cutil_math.h:1082-1093) as at neiglist.cu:359
        const double rmov = (double)sqrtf((float)(q.x * q.x + q.y * q.y + q.z * q.z));
        a.x = a.x + t.x * dt * dt / I;
        a.y = a.y + t.y * dt * dt / I;
        a.z = a.z + t.z * dt * dt / I;
        pos[i] = p; pdis[i] = d; qi[i] = q; angv[i] = a;
        mz = p.z > 0.0 ? p.z : 0.0;
        flag = rmov > ann ? 1u : 0u;
        if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) flag |= 2u;
    }
    unsigned long long mb = (unsigned long long)__double_as_longlong(mz);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, mb, o);
        mb = ob > mb ? ob : mb;
        flag |= __shfl_xor_sync(0xffffffffu, flag, o);
    }
    if (lane == 0) { smz[warp] = mb; sall[warp] = flag; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBlock / 32; w++) { mb = smz[w] > mb ? smz[w] : mb; flag |= sall[w]; }
        if (flag & 1u) atomicOr(&words[1], 1u);
        if (flag & 2u) atomicOr(&words[0], kStatusNonfinite);
        if (mb) atomicMax(reinterpret_cast<unsigned long long*>(&words[4]), mb);
    }
}

__global__ void k_count_contacts(uint n, const uint* __restrict__ contacti, uint* words) {
    __shared__ uint sw[kBlock / 32];
    uint i = blockIdx.x * blockDim.x + threadIdx.x;
    uint c = i < n ? contacti[i] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint s = 0;
        for (int w = 0; w < kBlock / 32; w++) s += sw[w];
        if (s) atomicAdd(&words[2], s);
    }
}

inline double3 d3(const double v[3]) { return make_double3(v[0], v[1], v[2]); }

int read_and_clear_status(CompatDevice* cd, uint* status_bits) {
    DEM_CUDA_TRY(cudaMemcpyAsync(cd->host_words, cd->words, sizeof(uint), cudaMemcpyDeviceToHost, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    *status_bits = cd->host_words[0];
    if (*status_bits) DEM_CUDA_TRY(cudaMemsetAsync(cd->words, 0, sizeof(uint), g_stream));
    return DEM_OK;
}
}  // namespace
}  // namespace dem

using namespace dem;

extern "C" {

int setMaterialProperties(const Matproperties* par, const Wallproperties* parw) {
    if (!par || !parw) return fail(DEM_ERR_ARG, "setMaterialProperties: null argument");
    dem_contact a{par->estarp, par->ufricp, par->vpois, par->dampnp, par->damptp, par->upp, 0.0};
    dem_contact b{parw->estarw, parw->ufricw, parw->vpoisw, parw->dampnw, parw->damptw, parw->upw, 0.0};
    LawParams<double> pa = make_law<double>(a), pb = make_law<double>(b);
    // on the wrappers' stream, after the kernels already queued there, and
    // complete before returning (a pageable upload may still be in flight
    // when a plain cudaMemcpyToSymbol returns)
    DEM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_pp, &pa, sizeof(pa), 0, cudaMemcpyHostToDevice, g_stream));
    DEM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_pw, &pb, sizeof(pb), 0, cudaMemcpyHostToDevice, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    return DEM_OK;
}

int setListCutoff(double cua, double cub) {
    if (!(cub > 0.0) || !(cua >= 0.0)) return fail(DEM_ERR_ARG, "setListCutoff: need cua >= 0, cub > 0");
    DEM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_cua, &cua, sizeof(double), 0, cudaMemcpyHostToDevice, g_stream));
    DEM_CUDA_TRY(cudaMemcpyToSymbolAsync(c_cub, &cub, sizeof(double), 0, cudaMemcpyHostToDevice, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    return DEM_OK;
}

int dem_compat_set_stream(void* s) {
    g_stream = (cudaStream_t)s;
    return DEM_OK;
}

int calcHash(double* Pos, unsigned int* particleHash, unsigned int gridSize[3], double cellSize[3],
             double worldOrigin[3], int numBodies) {
    if (numBodies <= 0) return DEM_OK;
    if (!Pos || !particleHash || !gridSize || !cellSize || !worldOrigin) return fail(DEM_ERR_ARG, "calcHash: null argument");
    k_calc_hash<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, (const double3*)Pos, (uint2*)particleHash, make_uint3(gridSize[0], gridSize[1], gridSize[2]),
        d3(cellSize), d3(worldOrigin));
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int findCellStart(unsigned int* particleHash, unsigned int* cellStart, int numBodies, unsigned int numGridCells) {
    if (!cellStart || (numBodies > 0 && !particleHash)) return fail(DEM_ERR_ARG, "findCellStart: null argument");
    DEM_CUDA_TRY(cudaMemsetAsync(cellStart, 0xff, (size_t)numGridCells * sizeof(uint), g_stream));
    if (numBodies <= 0) return DEM_OK;
    k_find_cell_start<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>((const uint2*)particleHash, cellStart,
                                                                             numBodies);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int neighborarray(double* pos, unsigned int* particleHash, unsigned int* cellStart, unsigned int gridSize[3],
                  double cellSize[3], double worldOrigin[3], int maxParticlesPerCell, int numBodies,
                  unsigned int* Anei, unsigned int* njgi, unsigned int* njli) {
    if (numBodies <= 0) return DEM_OK;
    if (!pos || !particleHash || !cellStart || !Anei || !njgi || !njli || maxParticlesPerCell <= 0)
        return fail(DEM_ERR_ARG, "neighborarray: bad argument");
    CompatDevice* cd;
    int rc = compat_device(&cd);
    if (rc) return rc;
    DEM_CUDA_TRY(cudaMemsetAsync(Anei, 0xff, (size_t)numBodies * maxParticlesPerCell * sizeof(uint), g_stream));
    k_neighbor_array<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, (const double3*)pos, (const uint2*)particleHash, cellStart,
        make_uint3(gridSize[0], gridSize[1], gridSize[2]), d3(cellSize), d3(worldOrigin), maxParticlesPerCell, Anei,
        njgi, njli, cd->words);
    DEM_LAUNCH_CHECK();
    uint st = 0;
    rc = read_and_clear_status(cd, &st);
    if (rc) return rc;
    if (st & kStatusCapacity)
        return fail(DEM_ERR_CAPACITY, "neighborarray: a particle has more than %d neighbours (rows cut)",
                    maxParticlesPerCell);
    return DEM_OK;
}

int prefixsum(unsigned int numBodies, unsigned int* njgi, unsigned int* sjgi, unsigned int* oldsjgi,
              unsigned int* totalcontacts) {
    if (!totalcontacts) return fail(DEM_ERR_ARG, "prefixsum: null totalcontacts");
    if (numBodies == 0) { *totalcontacts = 0; return DEM_OK; }
    if (!njgi || !sjgi || !oldsjgi) return fail(DEM_ERR_ARG, "prefixsum: null argument");
    CompatDevice* cd;
    int rc = compat_device(&cd);
    if (rc) return rc;
    uint* tmp;
    rc = compat_scratch(cd, scan_scratch_words(numBodies), &tmp);
    if (rc) return rc;
    DEM_CUDA_TRY(cudaMemcpyAsync(oldsjgi, sjgi, (size_t)numBodies * sizeof(uint), cudaMemcpyDeviceToDevice, g_stream));
    rc = exclusive_scan_u32(njgi, sjgi, numBodies, nullptr, tmp, g_stream);
    if (rc) return rc;
    k_add_two<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(sjgi, njgi, numBodies);
    DEM_LAUNCH_CHECK();
    DEM_CUDA_TRY(cudaMemcpyAsync(cd->host_words + 8, sjgi + numBodies - 1, sizeof(uint), cudaMemcpyDeviceToHost, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    *totalcontacts = cd->host_words[8];
    return DEM_OK;
}

int pairlist(unsigned int* sjgi, unsigned int* oldsjgi, unsigned int* oldLn, unsigned int* Anei, unsigned int* njgi,
             unsigned int* njli, double* olddispt, double* oldfricp, int maxParticlesPerCell, int maxCnPerParticle,
             unsigned int numBodies, unsigned int* Aref, unsigned int* Lp, unsigned int* Ln, double* dispt,
             double* fricp) {
    if (numBodies == 0) return DEM_OK;
    if (!sjgi || !oldsjgi || !oldLn || !Anei || !njgi || !njli || !olddispt || !oldfricp || !Aref || !Lp || !Ln ||
        !dispt || !fricp || maxParticlesPerCell <= 0 || maxCnPerParticle <= 0)
        return fail(DEM_ERR_ARG, "pairlist: bad argument");
    const size_t capN = (size_t)numBodies * maxParticlesPerCell, capP = (size_t)numBodies * maxCnPerParticle;
    DEM_CUDA_TRY(cudaMemsetAsync(Aref, 0xff, capN * sizeof(uint), g_stream));
    DEM_CUDA_TRY(cudaMemsetAsync(Lp, 0xff, capP * sizeof(uint), g_stream));
    DEM_CUDA_TRY(cudaMemsetAsync(Ln, 0xff, capP * sizeof(uint), g_stream));
    DEM_CUDA_TRY(cudaMemsetAsync(dispt, 0, capP * 3 * sizeof(double), g_stream));
    DEM_CUDA_TRY(cudaMemsetAsync(fricp, 0, capP * sizeof(double), g_stream));
    k_pairlist<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, sjgi, oldsjgi, oldLn, Anei, njgi, njli, (const double3*)olddispt, oldfricp, maxParticlesPerCell,
        capP, Aref, Lp, Ln, (double3*)dispt, fricp);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int calculateforcepair(double* pos, double* pdis, double* angv, double* rad, double* rmass, unsigned int* Lp,
                       unsigned int* Ln, unsigned int* oldLn, double* dispt, double* fricp, double* olddispt,
                       double* oldfricp, double dt, double* forcepair, double* torqpairi, double* torqpairj,
                       unsigned int* contactpair, unsigned int totalcontacts) {
    if (totalcontacts == 0) return DEM_OK;
    if (!pos || !pdis || !angv || !rad || !rmass || !Lp || !Ln || !oldLn || !dispt || !fricp || !olddispt ||
        !oldfricp || !forcepair || !torqpairi || !torqpairj || !contactpair || !(dt > 0.0))
        return fail(DEM_ERR_ARG, "calculateforcepair: bad argument");
    k_force_pair<<<grid_for(totalcontacts, kBlock), kBlock, 0, g_stream>>>(
        totalcontacts, (const double3*)pos, (const double3*)pdis, (const double3*)angv, rad, rmass, Lp, Ln, oldLn,
        (double3*)dispt, fricp, (double3*)olddispt, oldfricp, 1.0 / dt, (double3*)forcepair, (double3*)torqpairi,
        (double3*)torqpairj, contactpair);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int sumallforcei(int maxParticlesPerCell, int numBodies, unsigned int* njgi, unsigned int* njli, double* forcepair,
                 double* torqpairi, double* torqpairj, unsigned int* contactpair, unsigned int* Aref, double* forcei,
                 double* torquei, unsigned int* contacti) {
    if (numBodies <= 0) return DEM_OK;
    if (!njgi || !njli || !Aref || !forcei || !torquei || !contacti || maxParticlesPerCell <= 0)
        return fail(DEM_ERR_ARG, "sumallforcei: bad argument");
    k_sum_force<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, maxParticlesPerCell, njgi, njli, (const double3*)forcepair, (const double3*)torqpairi,
        (const double3*)torqpairj, contactpair, Aref, (double3*)forcei, (double3*)torquei, contacti);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int calculateforceiw(double worldSize[3], double* pos, double* pdis, double* angv, double* rad, double* rmass,
                     double dt, unsigned int totalcontacts, int numBodies, double* disptw, double* fricpw,
                     double* forcei, double* torquei) {
    if (numBodies <= 0) return DEM_OK;
    if (!worldSize || !pos || !pdis || !angv || !rad || !rmass || !disptw || !fricpw || !forcei || !torquei ||
        !(dt > 0.0))
        return fail(DEM_ERR_ARG, "calculateforceiw: bad argument");
    k_force_wall<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, d3(worldSize), (const double3*)pos, (const double3*)pdis, (const double3*)angv, rad, rmass,
        1.0 / dt, totalcontacts, (double3*)disptw, fricpw, (double3*)forcei, (double3*)torquei);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

int updateposition(double worldSize[3], int numBodies, double* pos, double* pdis, double* angv, double* rmass,
                   double* inert, double* forcei, double* torquei, double* qi, double dt, double cdamp,
                   unsigned int* iall, double* maxhz) {
    (void)worldSize;
    (void)cdamp;   /* read but unused by the reference too (adamp = bdamp = 1, neiglist.cu:354-355) */
    if (!iall || !maxhz) return fail(DEM_ERR_ARG, "updateposition: null iall/maxhz");
    *iall = 0;
    *maxhz = 0.0;
    if (numBodies <= 0) return DEM_OK;
    if (!pos || !pdis || !angv || !rmass || !inert || !forcei || !torquei || !qi)
        return fail(DEM_ERR_ARG, "updateposition: null argument");
    CompatDevice* cd;
    int rc = compat_device(&cd);
    if (rc) return rc;
    DEM_CUDA_TRY(cudaMemsetAsync(cd->words + 1, 0, sizeof(uint), g_stream));
    DEM_CUDA_TRY(cudaMemsetAsync(cd->words + 4, 0, 2 * sizeof(uint), g_stream));
    k_update<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(
        numBodies, (double3*)pos, (double3*)pdis, (double3*)angv, rmass, inert, (const double3*)forcei,
        (const double3*)torquei, (double3*)qi, dt, cd->words);
    DEM_LAUNCH_CHECK();
    DEM_CUDA_TRY(cudaMemcpyAsync(cd->host_words, cd->words, 8 * sizeof(uint), cudaMemcpyDeviceToHost, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    *iall = cd->host_words[1];
    unsigned long long mb;
    memcpy(&mb, cd->host_words + 4, sizeof(mb));
    double mz;
    memcpy(&mz, &mb, sizeof(mz));
    *maxhz = mz;
    if (cd->host_words[0] & kStatusNonfinite) {
        DEM_CUDA_TRY(cudaMemsetAsync(cd->words, 0, sizeof(uint), g_stream));
        return fail(DEM_ERR_NONFINITE, "updateposition: non-finite position");
    }
    return DEM_OK;
}

int outputporositycn(unsigned int numBodies, unsigned int* contacti, double maxhz, double worldSize[3],
                     unsigned int* pcntot) {
    (void)maxhz;
    (void)worldSize;
    if (!pcntot) return fail(DEM_ERR_ARG, "outputporositycn: null pcntot");
    *pcntot = 0;
    if (numBodies == 0) return DEM_OK;
    if (!contacti) return fail(DEM_ERR_ARG, "outputporositycn: null contacti");
    CompatDevice* cd;
    int rc = compat_device(&cd);
    if (rc) return rc;
    DEM_CUDA_TRY(cudaMemsetAsync(cd->words + 2, 0, sizeof(uint), g_stream));
    k_count_contacts<<<grid_for(numBodies, kBlock), kBlock, 0, g_stream>>>(numBodies, contacti, cd->words);
    DEM_LAUNCH_CHECK();
    DEM_CUDA_TRY(cudaMemcpyAsync(cd->host_words + 2, cd->words + 2, sizeof(uint), cudaMemcpyDeviceToHost, g_stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(g_stream));
    *pcntot = cd->host_words[2];
    return DEM_OK;
}

}  // extern "C"
