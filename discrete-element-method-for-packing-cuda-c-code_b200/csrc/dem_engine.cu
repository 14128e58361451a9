// dem_engine.cu -- the context API: structure-of-arrays DEM step on sm_100a.
//
// Same physics and step order as the reference's loop (dempacking.cu:535-739:
// re-list -> pair force -> gather -> wall + gravity -> integrate), laid out
// for B200:
//  * particle state as SoA planes (FP64 position / per-step displacement,
//    working-precision rotation and radius, FP64 wall history) so every
//    per-particle kernel streams fully coalesced 8/4-byte lanes;
//  * the half contact-candidate list as CSR by particle id (j ascending per
//    row) plus a reverse CSR of pair slots, replacing the fixed 30-slot Anei /
//    Aref rows (dempacking.cu:21-22) -- the gather onto particles stays
//    deterministic and atomic-free as in the reference;
//  * re-list without a general sort: cell counting (atomics) -> scan ->
//    scatter -> in-cell ranking by id, which is exactly the stable sort by
//    cell of calcHash + RadixSort (dempacking.cu:545-555) and yields cell
//    ranges directly (no cellStart memset);
//  * the FP32 (mixed) or FP64 candidate test evaluated on a cell-sorted
//    float4/double4 copy of (x, y, z, r);
//  * history carry by binary search in the previous CSR row (pairlistD's
//    contract, particleSystem.cu:143-191);
//  * the wall, gravity and integrator fused into one per-particle kernel that
//    also reduces the observables (max height, contacts) on the device;
//  * a whole re-list window (re-list + K steps) captured once as a CUDA graph;
//    no host synchronisation inside dem_step_n.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "dem_engine_internal.h"
#include "dem_compat_state.h"

namespace dem {

// Minimum resident blocks per SM requested for the per-particle kernels (caps
// their registers), and the largest grid of the grid-stride pair kernel.
#ifndef DEM_PARTICLE_MINB
#define DEM_PARTICLE_MINB 4
#endif
#ifndef DEM_PP_MINB
#define DEM_PP_MINB 3
#endif


// --------------------------------------------------------------- helpers
template <typename Real> __device__ __forceinline__ Real mul_rn(Real a, Real b);
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <typename Real> __device__ __forceinline__ Real add_rn(Real a, Real b);
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <typename Real> __device__ __forceinline__ Real sub_rn(Real a, Real b);
template <> __device__ __forceinline__ float sub_rn<float>(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ double sub_rn<double>(double a, double b) { return __dsub_rn(a, b); }
template <typename Real> __device__ __forceinline__ Real div_rn(Real a, Real b);
template <> __device__ __forceinline__ float div_rn<float>(float a, float b) { return __fdiv_rn(a, b); }
template <> __device__ __forceinline__ double div_rn<double>(double a, double b) { return __ddiv_rn(a, b); }


// Cell coordinate on one axis.  FP32: xf = (float)(x - o), floorf(xf / cs);
// FP64: floor((x - o) / cs).  Clamped to [0, g-1] (after a clamp of the
// quotient to [-1, g] so far-away positions cannot overflow the int).
template <typename Real> __device__ __forceinline__ int cell_axis(double x, double o, Real csr, int g, Real& xl) {
    xl = (Real)(x - o);
    Real v = div_rn<Real>(xl, csr);
    v = v < (Real)-1 ? (Real)-1 : (v > (Real)g ? (Real)g : v);
    int c = (int)floor(v);
    return c < 0 ? 0 : (c > g - 1 ? g - 1 : c);
}

// Candidate test, every operation rounded on its own (no FMA contraction):
// (dx*dx + dy*dy) + dz*dz < ((ri + rj) + skin)^2.
template <typename Real> __device__ __forceinline__ bool cand_test(const R4<Real>& a, const R4<Real>& b, Real skin) {
    Real dx = sub_rn<Real>(b.x, a.x), dy = sub_rn<Real>(b.y, a.y), dz = sub_rn<Real>(b.z, a.z);
    Real d2 = add_rn<Real>(mul_rn<Real>(dx, dx), mul_rn<Real>(dy, dy));
    d2 = add_rn<Real>(d2, mul_rn<Real>(dz, dz));
    Real cut = add_rn<Real>(add_rn<Real>(a.w, b.w), skin);
    return d2 < mul_rn<Real>(cut, cut);
}

__device__ __forceinline__ uint lane_id() { return threadIdx.x & 31; }

// Root of x (parent[x] <= x everywhere; a root is its own parent), halving
// the path on the way (plain stores touch only non-roots, the hooking CAS only
// roots).
__device__ __forceinline__ uint cc_find(uint* parent, uint x) {
    uint cur = __ldcg(parent + x);
    if (cur == x) return x;
    uint prev = x, next;
    while (cur > (next = __ldcg(parent + cur))) {
        parent[prev] = next;
        prev = cur;
        cur = next;
    }
    return cur;
}

// Root of x by a walk without stores, for use once all unions are made:
// other threads may meanwhile store roots into parent, which only shortens
// the walk (parent[x] < x for every non-root, so it ends).  A find with path
// halving there could overwrite a root just stored for another particle with
// a mere ancestor.
__device__ __forceinline__ uint cc_root(const uint* parent, uint x) {
    uint p;
    while ((p = __ldcg(parent + x)) != x) x = p;
    return x;
}

// Joins the components of a and b: the larger root is hooked under the
// smaller one by a compare-and-swap on the root, retried from the new roots
// when another thread hooked it first.
__device__ __forceinline__ void cc_union(uint* parent, uint a, uint b) {
    uint ra = cc_find(parent, a), rb = cc_find(parent, b);
    while (ra != rb) {
        if (ra < rb) { const uint t = ra; ra = rb; rb = t; }
        const uint old = atomicCAS(parent + ra, ra, rb);
        if (old == ra) break;
        ra = cc_find(parent, old);
        rb = cc_find(parent, rb);
    }
}


// ------------------------------------------------------------ state I/O
// Internal slot i takes the caller's particle perm[i] (identity when perm is
// null).
template <typename Real>
__global__ void k_from_aos(long long n, const double* __restrict__ pos, const double* __restrict__ pdis,
                           const double* __restrict__ angv, const double* __restrict__ rad, PRec<Real>* __restrict__ S,
                           Real* __restrict__ R, float4* __restrict__ Q, Planes3<double> W,
                           const uint* __restrict__ perm) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long u = perm ? (long long)perm[i] : i;
    const V3<double> x = mk(pos[3 * u], pos[3 * u + 1], pos[3 * u + 2]);
    const V3<double> d = pdis ? mk(pdis[3 * u], pdis[3 * u + 1], pdis[3 * u + 2]) : zero3<double>();
    const V3<Real> a = angv ? mk((Real)angv[3 * u], (Real)angv[3 * u + 1], (Real)angv[3 * u + 2]) : zero3<Real>();
    const Real r = (Real)rad[u];
    st_rec(S + i, x, d, a, r);
    R[i] = r;
    Q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    W.x[i] = 0.0; W.y[i] = 0.0; W.z[i] = 0.0;
}

// Particles nact .. n-1 (not yet poured in) report their injection state.
// Internal slot i goes to the caller's particle perm[i] (identity when perm is
// null).
template <typename Real>
__global__ void k_to_aos(long long n, long long nact, const PRec<Real>* __restrict__ S,
                         const PRec<Real>* __restrict__ pour, double* __restrict__ pos, double* __restrict__ pdis,
                         double* __restrict__ angv, const uint* __restrict__ perm) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3<double> x, d;
    V3<Real> a;
    Real r;
    ld_rec<false>((i < nact ? S : pour) + i, x, d, a, r);
    const long long u = perm ? (long long)perm[i] : i;
    if (pos) { pos[3 * u] = x.x; pos[3 * u + 1] = x.y; pos[3 * u + 2] = x.z; }
    if (pdis) { pdis[3 * u] = d.x; pdis[3 * u + 1] = d.y; pdis[3 * u + 2] = d.z; }
    if (angv) { angv[3 * u] = (double)a.x; angv[3 * u + 1] = (double)a.y; angv[3 * u + 2] = (double)a.z; }
}

// Poured packing: particles nold .. nnew-1 join the system with their
// injection records (dempacking.cu:459-460), zero displacement since the list
// and no wall contact; their rows of the current (previous) list are empty,
// so the coming re-list carries no history into them.
template <typename Real>
__global__ void k_pour_activate(long long nold, long long nnew, const PRec<Real>* __restrict__ pour,
                                PRec<Real>* __restrict__ S, float4* __restrict__ Q, Planes3<double> W,
                                uint* __restrict__ off) {
    const long long i = nold + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnew) return;
    S[i] = pour[i];
    Q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    W.x[i] = 0.0; W.y[i] = 0.0; W.z[i] = 0.0;
    off[i + 1] = off[nold];
}

// --------------------------------------------------------------- re-list
// Scatter each particle (id, cell, list coordinates x,y,z,r in the list
// precision) into its cell's range at its arrival slot, unordered inside the
// cell, and record each particle's slot (tpos); the count array returns to
// zero for the next re-list.  Reads are coalesced by id.  The walk and the
// fill work on this order directly: a row's candidate set does not depend on
// the order inside a cell, and every row is sorted by j before use.
template <typename Real>
__global__ void k_scatter(long long n, const uint* __restrict__ key, const uint* __restrict__ arrival,
                          const uint* __restrict__ cstart, uint* __restrict__ count, const PRec<Real>* __restrict__ S,
                          const Real* __restrict__ R, GridC g, uint* __restrict__ sidu, uint* __restrict__ skeyu,
                          R4<Real>* __restrict__ sposu, uint* __restrict__ tpos) {
    pdl_wait();
    pdl_trigger();
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint c = key[i];
    const V3<double> p = ld_pos<false>(S + i);
    R4<Real> v;
    v.x = (Real)(p.x - g.ox);
    v.y = (Real)(p.y - g.oy);
    v.z = (Real)(p.z - g.oz);
    v.w = R[i];
    const uint slot = cstart[c] + arrival[i];
    count[c] = 0u;
    sidu[slot] = (uint)i;
    skeyu[slot] = c;
    sposu[slot] = v;
    tpos[i] = slot;
}

// Row candidates kept per particle by the candidate pass; longer rows are
// filtered again by the fill.
constexpr uint kScr = 8;

// ------------------------------------------------------------- outer list
// The re-list searches candidates in an outer list: per particle every other
// particle within r_i + r_j + oskin (both directions; oskin = skin + ext,
// ext = min(skin, r_max / 10)) at the outer build, found by the cell walk on
// a grid of cells >= 2 r_max + oskin.  The list is kept while no particle is
// farther than odelta = 0.4 ext from its position at the build: a pair within
// r_i + r_j + skin now was within r_i + r_j + skin + 2 odelta < r_i + r_j +
// oskin then (with room for the rounding of the FP32 tests), so filtering the
// outer rows with the exact candidate test gives exactly the pairs the cell
// walk would give.  In a window graph the build is the body of a conditional
// node that the check kernel switches on; an eager re-list always builds.

// A particle's list coordinates (as k_scatter writes them): position relative
// to the grid origin and radius, in the list precision.
template <typename Real>
__device__ __forceinline__ R4<Real> rec_r4(const PRec<Real>* __restrict__ S, const Real* __restrict__ R, uint i,
                                           const GridC& g) {
    const V3<double> p = ld_pos<false>(S + i);
    R4<Real> v;
    v.x = (Real)(p.x - g.ox);
    v.y = (Real)(p.y - g.oy);
    v.z = (Real)(p.z - g.oz);
    v.w = R[i];
    return v;
}

// The re-list's first pass over the particles' positions: switches the
// outer build on (cond: a graph's conditional node) when the outer list is
// invalid (oflag) or a particle moved more than odelta since the build, and
// keeps each particle's cell on the configured grid (dem_download_cells)
// with its wall candidacy in the top bit: within r + skin/2 of a wall (a
// particle moves less than skin/2 per window, which the step checks, so no
// other particle can touch a wall before the next re-list -- the pair list's
// guarantee).  Cell keys stay below 2^31 (the grid is checked).
constexpr uint kNearWall = 0x80000000u;
template <typename Real>
__global__ void k_outer_check(long long n, const PRec<Real>* __restrict__ S, const Real* __restrict__ R, GridC g,
                              double hx, double hy, double half_skin, uint* __restrict__ ikey, Planes3<double> xo,
                              double odelta2, const uint* __restrict__ oflag, uint* __restrict__ wcount, int cond,
                              cudaGraphConditionalHandle h) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *wcount = 0u;   // the candidate pass counts the wall candidates
    bool need = i == 0 && *oflag != 0u;
    if (i < n) {
        const V3<double> p = ld_pos<false>(S + i);
        const double dx = p.x - xo.x[i], dy = p.y - xo.y[i], dz = p.z - xo.z[i];
        need = need || !(dx * dx + dy * dy + dz * dz <= odelta2);
        const double mg = (double)R[i] + half_skin;
        const bool near = (p.z < mg) || (p.x + hx < mg) || (hx - p.x < mg) || (p.y + hy < mg) || (hy - p.y < mg);
        const Real csr = (Real)g.cs;
        Real xl;
        const int cx = cell_axis<Real>(p.x, g.ox, csr, g.gx, xl);
        const int cy = cell_axis<Real>(p.y, g.oy, csr, g.gy, xl);
        const int cz = cell_axis<Real>(p.z, g.oz, csr, g.gz, xl);
        ikey[i] = (((uint)cz * (uint)g.gy + (uint)cy) * (uint)g.gx + (uint)cx) | (near ? kNearWall : 0u);
    }
    if (cond && __any_sync(0xffffffffu, need) && lane_id() == 0) cudaGraphSetConditional(h, 1u);
}

// Cell key of each particle on the outer grid (calcHashD's role,
// neiglist.cu:77-97), and its slot among the cell's members (the counting
// sort of k_scatter).
template <typename Real>
__global__ void k_cell_hash(long long n, const PRec<Real>* __restrict__ S, GridC g, uint* __restrict__ key,
                            uint* __restrict__ count, uint* __restrict__ arrival) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3<double> p = ld_pos<false>(S + i);
    const Real csr = (Real)g.cs;
    Real xl;
    const int cx = cell_axis<Real>(p.x, g.ox, csr, g.gx, xl);
    const int cy = cell_axis<Real>(p.y, g.oy, csr, g.gy, xl);
    const int cz = cell_axis<Real>(p.z, g.oz, csr, g.gz, xl);
    const uint c = ((uint)cz * (uint)g.gy + (uint)cy) * (uint)g.gx + (uint)cx;
    key[i] = c;
    arrival[i] = atomicAdd(&count[c], 1u);
}

// The outer walk from sorted slot t: every candidate within r_i + r_j + oskin
// in the 27 cells (both directions); FILL writes them at out (capacity cap).
template <typename Real, bool FILL>
__device__ __forceinline__ uint walk27_all(long long t, const R4<Real>& me, uint c, const GridC& g,
                                           const uint* __restrict__ cstart, const uint* __restrict__ sid2,
                                           const R4<Real>* __restrict__ spos, Real oskin, uint* __restrict__ out,
                                           uint outcap) {
    const int cx = (int)(c % (uint)g.gx);
    const int cy = (int)((c / (uint)g.gx) % (uint)g.gy);
    const int cz = (int)(c / ((uint)g.gx * (uint)g.gy));
    const int x0 = cx > 0 ? cx - 1 : 0, x1 = cx < g.gx - 1 ? cx + 1 : g.gx - 1;
    uint nall = 0;
    for (int r = 0; r < 9; r++) {
        const int z = cz - 1 + r / 3, y = cy - 1 + r % 3;
        if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
        const uint rowc = ((uint)z * (uint)g.gy + (uint)y) * (uint)g.gx;
        const uint u0 = cstart[rowc + x0], u1 = cstart[rowc + x1 + 1];
        for (uint u = u0; u < u1; u++) {
            if ((long long)u == t) continue;
            if (cand_test<Real>(me, spos[u], oskin)) {
                if (FILL && nall < outcap) out[nall] = sid2[u];
                nall++;
            }
        }
    }
    return nall;
}

// Outer build, count pass: each particle's outer row length.
template <typename Real>
__global__ void k_outer_count(long long n, const uint* __restrict__ sid2, const R4<Real>* __restrict__ spos,
                              const uint* __restrict__ skey, const uint* __restrict__ cstart, GridC g, Real oskin,
                              uint* __restrict__ ocnt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    ocnt[sid2[t]] = walk27_all<Real, false>(t, spos[t], skey[t], g, cstart, sid2, spos, oskin, nullptr, 0);
}

// Outer build, fill pass: the rows, each particle's position at the build,
// and the list marked valid (or, beyond the capacity, the capacity status and
// the list left invalid).
template <typename Real>
__global__ void k_outer_fill(long long n, const uint* __restrict__ sid2, const R4<Real>* __restrict__ spos,
                             const uint* __restrict__ skey, const uint* __restrict__ cstart, GridC g, Real oskin,
                             const uint* __restrict__ coff, uint* __restrict__ cln, long long ccap,
                             const PRec<Real>* __restrict__ S, Planes3<double> xo, uint* __restrict__ oflag,
                             EngineWords* words) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool over = (long long)coff[n] > ccap;
    if (t == 0) {
        *oflag = over ? 1u : 0u;
        if (over) atomicOr(&words->status, kStCapacity);
    }
    if (t >= n || over) return;
    const uint i = sid2[t];
    const uint b = coff[i];
    walk27_all<Real, true>(t, spos[t], skey[t], g, cstart, sid2, spos, oskin, cln + b, coff[i + 1] - b);
    const V3<double> p = ld_pos<false>(S + i);
    xo.x[i] = p.x; xo.y[i] = p.y; xo.z[i] = p.z;
}

// The re-list's candidate pass on the outer list, per particle i (id order):
// a wall candidacy (found by k_outer_check) takes a slot, and the outer row
// is filtered with the exact candidate test on the list coordinates: the
// counts of the row (j > i) and of the reverse row (j < i), the first kScr
// row candidates, and the bound flag (any candidate or a wall candidacy).  A
// bound particle starts the re-list's components (cluster batches) as a
// singleton; free particles take no part in them.
#define DEM_FILTER_PARAMS                                                                                      \
    long long n, const PRec<Real>* __restrict__ S, const Real* __restrict__ R, GridC g, Real skin,                   \
        const uint* __restrict__ coff, const uint* __restrict__ cln, long long ccap, uint* __restrict__ wslot,     \
        uint* __restrict__ wlist, uint* __restrict__ wcount, uint* __restrict__ cc_parent,                         \
        uint* __restrict__ cc_zero, uint* __restrict__ cc_base, long long np, const uint* __restrict__ ikey,        \
        uint* __restrict__ njli, uint* __restrict__ bflag, uint* __restrict__ scr
#define DEM_FILTER_ARGS \
    n, S, R, g, skin, coff, cln, ccap, wslot, wlist, wcount, cc_parent, cc_zero, cc_base, np, ikey, njli, bflag, scr
// The candidate pass for kFilterItems consecutive particles i0, i0+1, ...
// of one thread: their cell words (wall-candidacy bit) and outer-row bounds
// are loaded together first, so that the thread waits on one chain of loads
// rather than one per particle; only particles with outer candidates load
// positions.  Outputs per particle: row and reverse-row counts, bound flag.
template <int K> struct FilterCounts { uint up[K], dn[K], bd[K]; };
template <typename Real, int K>
__device__ __forceinline__ FilterCounts<K> filter_items(long long i0, DEM_FILTER_PARAMS) {
    FilterCounts<K> o;
    uint key[K], cb[K + 1];
    const bool whole = i0 + K <= n;
    if (whole && K == 4) {   // i0 is a multiple of 4: aligned 16-byte loads
        const uint4 kq = *reinterpret_cast<const uint4*>(ikey + i0);
        const uint4 cq = *reinterpret_cast<const uint4*>(coff + i0);
        key[0] = kq.x; key[1] = kq.y; key[2] = kq.z; key[3] = kq.w;
        cb[0] = cq.x; cb[1] = cq.y; cb[2] = cq.z; cb[3] = cq.w;
        cb[K] = coff[i0 + K];
    } else {
#pragma unroll
        for (int k = 0; k <= K; k++) {   // coff has n + 1 entries
            if (k < K) key[k] = i0 + k < n ? ikey[i0 + k] : 0u;
            cb[k] = i0 + k <= n ? coff[i0 + k] : 0u;
        }
    }
    const bool list_ok = (long long)coff[n] <= ccap;
    uint nwall = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const long long ii = i0 + k;
        uint nup = 0, nall = 0;
        if (ii < n && list_ok && cb[k + 1] > cb[k]) {   // positions only where there are candidates
            const uint i = (uint)ii;
            const V3<double> p = ld_pos<false>(S + i);
            R4<Real> me;
            me.x = (Real)(p.x - g.ox);
            me.y = (Real)(p.y - g.oy);
            me.z = (Real)(p.z - g.oz);
            me.w = R[i];
            uint* out = scr + (size_t)i * kScr;
            for (uint q = cb[k]; q < cb[k + 1]; q++) {
                const uint j = cln[q];
                if (cand_test<Real>(me, rec_r4<Real>(S, R, j, g), skin)) {
                    nall++;
                    if (j > i) {
                        if (nup < kScr) out[nup] = j;
                        nup++;
                    }
                }
            }
        }
        const bool near = ii < n && (key[k] & kNearWall) != 0u;
        nwall += near ? 1u : 0u;
        o.up[k] = nup;
        o.dn[k] = nall - nup;
        o.bd[k] = (ii < n && (nall > 0 || near)) ? 1u : 0u;
    }
    // wall slots: one atomic per warp for all its wall candidates (slots only
    // name them; their order does not matter)
    const uint lane = lane_id();
    uint incw = nwall;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint t = __shfl_up_sync(0xffffffffu, incw, d);
        if ((int)lane >= d) incw += t;
    }
    const uint wtot = __shfl_sync(0xffffffffu, incw, 31);
    uint wbase = 0;
    if (lane == 31 && wtot) wbase = atomicAdd(wcount, wtot);
    uint ws = __shfl_sync(0xffffffffu, wbase, 31) + incw - nwall;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const long long ii = i0 + k;
        if (ii >= n) continue;
        const uint i = (uint)ii;
        njli[i] = o.dn[k];
        uint slot = kEmpty;
        if (key[k] & kNearWall) {
            slot = ws++;
            wlist[slot] = i;
        }
        wslot[i] = slot;
        bflag[i] = o.bd[k];
        if (cc_parent && o.bd[k]) {   // the coming re-list's components start as singletons
            cc_parent[i] = i;
            cc_zero[i] = 0u; cc_zero[np + i] = 0u; cc_zero[2 * np + i] = 0u;
            cc_base[i] = kEmpty;
        }
    }
    return o;
}

// The candidate pass fused with the exclusive scans of its three counts
// (row offsets off, reverse-row offsets roff, bound positions bpos; totals
// at [n]) by a single-pass scan with decoupled look-back (Merrill & Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016): tiles
// of kFilterTile particles (kFilterItems consecutive ones per thread) take
// tickets in the order they start, publish
// their totals, and add up the published words of the tiles before them, so
// no tile waits on one that has not started.  The tile also writes the bound
// list (ascending id) and the free list.  Look-back words (lb): [0] the tile
// ticket, then per tile and count a 64-bit word, the value in the low 32 bits
// and the kind above (1: the tile's own total, 2: the total through the
// tile); the fill clears them for the next re-list.
constexpr int kFilterThreads = 512, kFilterItems = 4, kFilterTile = kFilterThreads * kFilterItems;
constexpr int kCcThreads = 256;   // the component pass: one bound-list entry per thread and tile
constexpr unsigned long long kLbAgg = 1ull << 32, kLbIncl = 2ull << 32;
constexpr int kLbSpin = 1 << 16;   // a look-back word not published after this many polls: kStBarrier
// which bounded wait gave up (EngineWords::pad[0], reported by dem_get_scalars)
enum : uint { kWaitFilterLb = 1u, kWaitFilterTicket = 2u, kWaitCcLb = 4u, kWaitCcRoot = 8u, kWaitBatchTable = 16u };
__device__ __forceinline__ void wait_gave_up(EngineWords* w, uint site) {
    atomicOr(&w->status, kStBarrier);
    atomicOr(&w->pad[0], site);
}
// [0, 2 + 6 T) the candidate pass's words (T: its tiles of np particles),
// then the component pass's: 2 + 2 Tc (Tc: its tiles of np entries)
inline size_t lb_cc(long long np) { return 2 + 6 * (size_t)grid_for(np, kFilterTile); }
inline size_t lb_words(long long np) { return lb_cc(np) + 2 + 2 * (size_t)grid_for(np, kCcThreads); }

__device__ __forceinline__ void lb_store(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long lb_load(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
template <typename Real>
__global__ void __launch_bounds__(kFilterThreads) k_filter_scan(DEM_FILTER_PARAMS, EngineWords* words, uint* lb,
                                                                uint* __restrict__ off, uint* __restrict__ roff,
                                                                uint* __restrict__ bpos, uint* __restrict__ blist,
                                                                uint* __restrict__ flist, uint* __restrict__ ccw,
                                                                uint* __restrict__ bw, long long nbb) {
    constexpr int W = kFilterThreads / 32;
    __shared__ uint s_tile;
    __shared__ uint s_w[3][W];
    __shared__ uint s_red[3][W];
    __shared__ uint s_agg[3], s_pre[3];
    __shared__ int s_near[3];
    pdl_trigger();
    if (threadIdx.x == 0) s_tile = atomicAdd(lb, 1u);
    __syncthreads();
    const uint tile = s_tile;
    if (tile >= gridDim.x) {   // a ticket left over (the words were not cleared): nothing out of range
        if (threadIdx.x == 0) wait_gave_up(words, kWaitFilterTicket);
        return;
    }
    // the thread's kFilterItems consecutive particles
    const long long i0 = (long long)tile * kFilterTile + (long long)threadIdx.x * kFilterItems;
    if (ccw) {   // the component pass's words and batch windows start empty
        const long long nthr = (long long)gridDim.x * kFilterThreads;
        const long long t0 = (long long)tile * kFilterThreads + threadIdx.x;
        if (t0 < 4) ccw[t0] = 0u;
        for (long long k = t0; k < 3 * nbb; k += nthr) bw[k] = k < nbb ? 0xffffffffu : 0u;
    }
    const FilterCounts<kFilterItems> fc = filter_items<Real, kFilterItems>(i0, DEM_FILTER_ARGS);
    const uint *up = fc.up, *dn = fc.dn, *bd = fc.bd;
    uint v[3] = {0u, 0u, 0u}, mrow = 0;
#pragma unroll
    for (int k = 0; k < kFilterItems; k++) {
        v[0] += up[k]; v[1] += dn[k]; v[2] += bd[k];
        mrow = max(mrow, up[k] + dn[k]);
    }
    mrow = __reduce_max_sync(0xffffffffu, mrow);
    const uint lane = lane_id(), warp = threadIdx.x >> 5;
    if (lane == 0 && mrow) atomicMax(&words->max_row, mrow);
    uint inc[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        inc[a] = v[a];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint t = __shfl_up_sync(0xffffffffu, inc[a], d);
            if ((int)lane >= d) inc[a] += t;
        }
        if (lane == 31) s_w[a][warp] = inc[a];
    }
    __syncthreads();
    if (warp == 0) {   // warp totals -> warp offsets; the tile's totals
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const uint w = (int)lane < W ? s_w[a][lane] : 0u;
            uint wi = w;
#pragma unroll
            for (int d = 1; d < W; d <<= 1) {
                const uint t = __shfl_up_sync(0xffffffffu, wi, d);
                if ((int)lane >= d) wi += t;
            }
            if ((int)lane < W) s_w[a][lane] = wi - w;
            if ((int)lane == W - 1) s_agg[a] = wi;
        }
    }
    __syncthreads();
    // publish the tile's totals; the prefix: the whole block looks back over
    // kFilterThreads earlier tiles per round (thread k: tile - 1 - k), adding
    // every word up to the nearest inclusive one
    unsigned long long* st = reinterpret_cast<unsigned long long*>(lb + 2);
    const uint me = threadIdx.x;
    uint pre = 0;   // threads 0..2: the prefix of count `me`
    if (tile == 0) {
        if (me < 3) lb_store(st + me, kLbIncl | s_agg[me]);
    } else {
        if (me < 3) lb_store(st + 3 * (size_t)tile + me, kLbAgg | s_agg[me]);
        bool done[3] = {false, false, false};
        for (long long base = (long long)tile - 1; !(done[0] && done[1] && done[2]); base -= kFilterThreads) {
            const long long t = base - (long long)me;
            unsigned long long w[3] = {kLbIncl, kLbIncl, kLbIncl};   // before tile 0: zero
            if (t >= 0) {
                const unsigned long long* q = st + 3 * t;
                for (int spin = 0;; spin++) {
                    w[0] = lb_load(q); w[1] = lb_load(q + 1); w[2] = lb_load(q + 2);
                    if ((w[0] >> 32) && (w[1] >> 32) && (w[2] >> 32)) break;
                    if (spin >= kLbSpin) {   // never published: record it, count the tile as zero
                        wait_gave_up(words, kWaitFilterLb);
                        w[0] = w[1] = w[2] = kLbIncl;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            if (me < 3) s_near[me] = kFilterThreads;
            __syncthreads();
#pragma unroll
            for (int a = 0; a < 3; a++) {   // the nearest inclusive word of each count
                const uint m = __ballot_sync(0xffffffffu, (w[a] >> 32) == 2ull);
                if (!done[a] && lane == 0 && m) atomicMin(&s_near[a], (int)(warp * 32 + __ffs(m) - 1));
            }
            __syncthreads();
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const uint x = (!done[a] && (int)me <= s_near[a]) ? (uint)w[a] : 0u;
                const uint sx = __reduce_add_sync(0xffffffffu, x);
                if (lane == 0) s_red[a][warp] = sx;
            }
            __syncthreads();
            const bool dme = me == 0 ? done[0] : (me == 1 ? done[1] : done[2]);
            if (me < 3 && !dme)
                for (int k = 0; k < W; k++) pre += s_red[me][k];
#pragma unroll
            for (int a = 0; a < 3; a++) done[a] = done[a] || s_near[a] < kFilterThreads;
            __syncthreads();   // s_near and s_red are written again next round
        }
        if (me < 3) lb_store(st + 3 * (size_t)tile + me, kLbIncl | (pre + s_agg[me]));
    }
    if (me < 3) {
        s_pre[me] = pre;
        if (tile == gridDim.x - 1) {   // the totals
            uint* tot = me == 0 ? off : (me == 1 ? roff : bpos);
            tot[n] = pre + s_agg[me];
        }
    }
    __syncthreads();
    uint e0 = s_pre[0] + s_w[0][warp] + inc[0] - v[0];
    uint e1 = s_pre[1] + s_w[1][warp] + inc[1] - v[1];
    uint e2 = s_pre[2] + s_w[2][warp] + inc[2] - v[2];
#pragma unroll
    for (int k = 0; k < kFilterItems; k++) {
        const long long ii = i0 + k;
        if (ii < n) {
            const uint i = (uint)ii;
            off[i] = e0;
            roff[i] = e1;
            bpos[i] = e2;
            if (bd[k]) blist[e2] = i;
            else flist[i - e2] = i;
        }
        e0 += up[k]; e1 += dn[k]; e2 += bd[k];
    }
}

__device__ __forceinline__ void isort_u32(uint* a, uint len) {
    for (uint s = 1; s < len; s++) {
        uint v = a[s];
        uint u = s;
        while (u > 0 && a[u - 1] > v) { a[u] = a[u - 1]; u--; }
        a[u] = v;
    }
}

// Fill the CSR row of i (j>i ascending), carry the FP64 tangential history
// from the previous list, record the reverse slots.  Every particle with a
// row is bound, so the pass strides over the bound list only.
#define DEM_FILL_PARAMS                                                                                               \
    long long n, const PRec<Real>* __restrict__ S, const Real* __restrict__ R, GridC g, Real skin,                    \
    const uint* __restrict__ coff, const uint* __restrict__ cln, const uint* __restrict__ off,                        \
    const uint* __restrict__ roff, uint* __restrict__ njli, uint* __restrict__ ln, uint* __restrict__ lp,             \
    Planes3<double> H, const uint* __restrict__ ooff, const uint* __restrict__ oln, Planes3<double> OH,               \
    uint* __restrict__ rk, R4<Real>* __restrict__ pf, long long cap, EngineWords* words,                              \
    uint* __restrict__ carry, const uint* __restrict__ scr, uint* cc_parent
#define DEM_FILL_ARGS                                                                                                 \
    n, S, R, g, skin, coff, cln, off, roff, njli, ln, lp, H, ooff, oln, OH, rk, pf, cap, words, carry, scr, cc_parent
template <typename Real> __device__ __forceinline__ void fill_item(uint i, DEM_FILL_PARAMS) {
    const uint b = off[i], e = off[i + 1];
    if (e == b) return;
    if (e - b <= kScr) {
        for (uint k = 0; k < e - b; k++) ln[b + k] = scr[(size_t)i * kScr + k];
    } else {   // a long row: filter the particle's outer row again
        const R4<Real> me = rec_r4<Real>(S, R, i, g);
        uint w = 0;
        for (uint k = coff[i], k1 = coff[i + 1]; k < k1 && w < e - b; k++) {
            const uint j = cln[k];
            if (j > i && cand_test<Real>(me, rec_r4<Real>(S, R, j, g), skin)) ln[b + w++] = j;
        }
    }
    isort_u32(ln + b, e - b);
    const bool old_ok = (long long)ooff[n] <= cap;   // an overflowed old list carries nothing
    const uint ob = old_ok ? ooff[i] : 0u, oe = old_ok ? ooff[i + 1] : 0u;
    for (uint k = b; k < e; k++) {
        const uint j = ln[k];
        lp[k] = i;
        // binary search j in the previous row of i (ascending)
        uint lo = ob, hi = oe;
        while (lo < hi) {
            uint mid = (lo + hi) >> 1;
            if (oln[mid] < j) lo = mid + 1; else hi = mid;
        }
        if (lo < oe && oln[lo] == j) {
            H.x[k] = OH.x[lo]; H.y[k] = OH.y[lo]; H.z[k] = OH.z[lo];
            if (carry) carry[k] = lo;
        } else {
            H.x[k] = 0.0; H.y[k] = 0.0; H.z[k] = 0.0;
            if (carry) carry[k] = kEmpty;
        }
        R4<Real> z4;
        z4.x = z4.y = z4.z = z4.w = (Real)0;
        pf[k] = z4;
        const uint left = atomicSub(&njli[j], 1u);
        if (left == 0u) {   // counts of the two walks disagree: cannot happen with the symmetric test
            atomicOr(&words->status, kStCapacity);
            continue;
        }
        rk[roff[j] + left - 1u] = k;
        if (cc_parent) cc_union(cc_parent, i, j);   // the window's components (cluster batches)
    }
}

// The fill over the bound list (grid-stride); it also clears the candidate
// pass's look-back words (lbw of them) for the next re-list.
template <typename Real>
__global__ void k_nbr_fill(DEM_FILL_PARAMS, const uint* __restrict__ bpos, const uint* __restrict__ blist,
                           const uint* __restrict__ cc_skip, uint* __restrict__ lb, long long lbw) {
    pdl_wait();
    pdl_trigger();
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x, nthr = (long long)gridDim.x * blockDim.x;
    for (long long k = tid; k < lbw; k += nthr) lb[k] = 0u;
    if ((long long)off[n] > cap) {
        if (tid == 0) atomicOr(&words->status, kStCapacity);
        return;
    }
    if (cc_parent && *cc_skip) cc_parent = nullptr;   // a dense bed: no component pass this re-list
    const long long nb = bpos[n];
    for (long long t = tid; t < nb; t += nthr) fill_item<Real>(blist[t], DEM_FILL_ARGS);
}

// Sort each reverse row (pair indices ascending: a deterministic order for
// the gather) and record each pair's reverse slot ru[k]; every particle with
// a reverse row is bound (the pass strides over the bound list).  With
// cluster batches (parent != nullptr): every bound particle also takes its
// component's root (all unions were made by the fill) and adds itself and
// its row's pairs to the root's counts.
__global__ void k_rev_sort(long long n, const uint* __restrict__ roff, uint* __restrict__ rk, uint* __restrict__ ru,
                           const uint* __restrict__ off, long long cap, uint* parent, const uint* __restrict__ bpos,
                           const uint* __restrict__ blist, uint* __restrict__ csize, uint* __restrict__ cpairs,
                           const uint* __restrict__ cc_skip, uint* __restrict__ ccw) {
    pdl_wait();
    pdl_trigger();
    if ((long long)off[n] > cap) return;
    if (parent && *cc_skip) parent = nullptr;
    const long long nb = bpos[n];
    uint mx = 0;   // the largest running component count: the largest component
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nb;
         t += (long long)gridDim.x * blockDim.x) {
        const uint i = blist[t];
        const uint b = roff[i], e = roff[i + 1];
        isort_u32(rk + b, e - b);
        for (uint u = b; u < e; u++) ru[rk[u]] = u;
        if (parent) {
            const uint r = cc_root(parent, i);
            parent[i] = r;
            mx = max(mx, atomicAdd(csize + r, 1u) + 1u);
            atomicAdd(cpairs + r, off[i + 1] - off[i]);
        }
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane_id() == 0 && mx) atomicMax(ccw + 2, mx);
}

// ------------------------------------------------------- cluster batches
// The window's interaction graph is the pair list: two spheres without a
// listed pair cannot touch before the next re-list (the skin guard checks
// it).  Its connected components are therefore independent for the whole
// window.  The re-list finds them with a lock-free union-find over the pairs
// (hooking the larger root under the smaller, the scheme of ECL-CC,
// Jaiganesh & Burtscher 2018), groups the bound particles by component into
// slots (components in root order; members of a component in any order:
// every particle's sums keep their list order, so the states do not depend
// on it), and cuts the slots into batches of whole components, one per
// resident block of k_batch where they fit (the batch window, cc_target),
// that one block steps through the window in shared memory.  A batch above
// the block's capacity (a bed of touching spheres is one component) sends
// the whole window to the grid-barrier window kernel instead.

// The batch window: the bound particles spread over the batch kernel's
// resident blocks G, at least kBatchMin, at most P minus the largest component
// (so that a window's components and the tail of its last one fit a block).
__device__ __forceinline__ uint cc_target(uint nb, uint G, uint P, uint maxc) {
    uint t = (nb + G - 1) / G;
    const uint hi = P > maxc ? P - maxc : 0u;
    t = min(t, hi);
    return max(t, kBatchMin);
}

// First slot of batch b (the first component whose first slot is b * target
// or later; all bound particles when none is), and the batch's particles and
// pairs against the block's capacity (P, Q).  bw: [0, nbb) first slots,
// [nbb, 2 nbb) particles, [2 nbb, 3 nbb) pairs, per batch window.
__device__ __forceinline__ void cc_batch_entry(uint b, uint nb, uint tgt, long long nbmax, long long nbb, uint P,
                                               uint Q, const uint* bw, uint* __restrict__ batch, uint* ccw) {
    uint s0 = __ldcg(bw + b);
    long long k = b;
    // a window with no first slot lies inside a component that started
    // earlier (longer than a block if the search runs out: its batch's count
    // is over P already)
    while (s0 == 0xffffffffu && k < nbmax && k - b <= (long long)(P / tgt) + 1) s0 = __ldcg(bw + (++k));
    if (s0 == 0xffffffffu || s0 > nb) s0 = nb;
    batch[b] = s0;
    if (__ldcg(bw + nbb + b) > P || __ldcg(bw + 2 * nbb + b) > Q) atomicOr(ccw + 1, 1u);
}

// The component pass in one launch, after the reverse rows (which leave
// every bound particle's root in parent[], the components' particle and pair
// counts at their roots, and the largest component in ccw[2]).  Tiles of
// kCcThreads bound-list entries, taken by ticket: each root's first slot
// is the exclusive scan, in root order, of the component sizes (decoupled
// look-back over the tiles before, as in the candidate pass); each member
// then takes a slot in its component's range (a root precedes its members,
// so its tile took its ticket earlier; the member waits, bounded, for the
// root's first slot), and each root adds its component to the batch window
// its first slot falls in.  The block that finishes last writes the batch
// table.  ccw: [0] unused, [1] not batchable, [2] largest component, [3]
// the batch window.  lbc: [0] tile ticket, [1] finished blocks, then one
// 64-bit look-back word per tile (cleared by the next re-list's fill).
__global__ void __launch_bounds__(kCcThreads)
    k_cc_pass(long long n, long long cap, long long nbmax, long long nbb, uint G, uint P, uint Q,
              const uint* __restrict__ off, const uint* __restrict__ bpos, const uint* __restrict__ blist,
              const uint* __restrict__ parent, const uint* __restrict__ size, const uint* __restrict__ pairs,
              uint* base, uint* __restrict__ fill, uint* __restrict__ order, uint* bw, uint* __restrict__ batch,
              uint* ccw, uint* __restrict__ cc_skip, uint* lbc, EngineWords* words) {
    constexpr int W = kCcThreads / 32;
    __shared__ uint s_tile, s_last, s_agg, s_pre;
    __shared__ uint s_w[W], s_red[W];
    __shared__ int s_near;
    pdl_wait();
    pdl_trigger();
    const uint nb = bpos[n];
    const uint skip = *cc_skip;
    const uint maxc = ccw[2];
    const bool over = (long long)off[n] > cap;
    const uint tgt = cc_target(nb, G, P, maxc);
    // skip: no components this re-list (the grid-barrier window kernel has
    // the window); every block still counts itself finished, and the last
    // one moves the skip count (cc_skip is read by every block first)
    const bool run = !(skip || over);
    if (!run && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(ccw + 1, 1u);
    if (run && blockIdx.x == 0 && threadIdx.x == 0) ccw[3] = tgt;
    const uint ntile = !run ? 0u : (nb == 0 ? 1u : (nb + kCcThreads - 1) / kCcThreads);
    unsigned long long* st = reinterpret_cast<unsigned long long*>(lbc + 2);
    const uint me = threadIdx.x, lane = lane_id(), warp = me >> 5;
    for (;;) {
        if (me == 0) s_tile = atomicAdd(lbc, 1u);
        __syncthreads();
        const uint tile = s_tile;
        if (tile >= ntile) break;
        const uint t = tile * kCcThreads + me;
        uint i = 0, r = kEmpty, sz = 0;
        if (t < nb) {
            i = blist[t];
            r = parent[i];
            if (r >= (uint)n || parent[r] != r) {   // not a root: the window goes to the grid-barrier kernel
                atomicOr(ccw + 1, 1u);
                r = kEmpty;
            } else if (r == i) {
                sz = size[i];
            }
        }
        // exclusive scan of the roots' sizes within the tile
        uint inc = sz;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint x = __shfl_up_sync(0xffffffffu, inc, d);
            if ((int)lane >= d) inc += x;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint w = (int)lane < W ? s_w[lane] : 0u;
            uint wi = w;
#pragma unroll
            for (int d = 1; d < W; d <<= 1) {
                const uint x = __shfl_up_sync(0xffffffffu, wi, d);
                if ((int)lane >= d) wi += x;
            }
            if ((int)lane < W) s_w[lane] = wi - w;
            if ((int)lane == W - 1) s_agg = wi;
        }
        __syncthreads();
        // the tiles before: published totals up to the nearest inclusive one
        uint pre = 0;
        if (tile == 0) {
            if (me == 0) lb_store(st, kLbIncl | s_agg);
        } else {
            if (me == 0) lb_store(st + tile, kLbAgg | s_agg);
            bool done = false;
            for (long long b0 = (long long)tile - 1; !done; b0 -= kCcThreads) {
                const long long tt = b0 - (long long)me;
                unsigned long long w = kLbIncl;
                if (tt >= 0) {
                    for (int spin = 0;; spin++) {
                        w = lb_load(st + tt);
                        if (w >> 32) break;
                        if (spin >= kLbSpin) {
                            wait_gave_up(words, kWaitCcLb);
                            atomicOr(ccw + 1, 1u);
                            w = kLbIncl;
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                if (me == 0) s_near = kCcThreads;
                __syncthreads();
                const uint m = __ballot_sync(0xffffffffu, (w >> 32) == 2ull);
                if (lane == 0 && m) atomicMin(&s_near, (int)(warp * 32 + __ffs(m) - 1));
                __syncthreads();
                const uint x = __reduce_add_sync(0xffffffffu, (int)me <= s_near ? (uint)w : 0u);
                if (lane == 0) s_red[warp] = x;
                __syncthreads();
                if (me == 0)
                    for (int k = 0; k < W; k++) pre += s_red[k];
                done = s_near < kCcThreads;
                __syncthreads();
            }
            if (me == 0) lb_store(st + tile, kLbIncl | (pre + s_agg));
        }
        if (me == 0) s_pre = pre;
        __syncthreads();
        if (r != kEmpty && r == i) {   // the root's first slot
            const uint b = s_pre + s_w[warp] + inc - sz;
            asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(base + i), "r"(b) : "memory");
        }
        __syncthreads();
        if (r != kEmpty) {
            uint b;
            for (int spin = 0;; spin++) {   // the root's tile started before this one
                asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(b) : "l"(base + r) : "memory");
                if (b != kEmpty) break;
                if (spin >= kLbSpin) {
                    wait_gave_up(words, kWaitCcRoot);
                    atomicOr(ccw + 1, 1u);
                    break;
                }
                __nanosleep(32);
            }
            if (b != kEmpty) {
                const uint s = b + atomicAdd(fill + r, 1u);
                if (s >= nb) atomicOr(ccw + 1, 1u);
                else order[s] = i;
                if (r == i) {
                    const uint bt = b / tgt;
                    if ((long long)bt >= nbb) {
                        atomicOr(ccw + 1, 1u);
                    } else {
                        atomicMin(bw + bt, b);
                        atomicAdd(bw + nbb + bt, size[i]);
                        atomicAdd(bw + 2 * nbb + bt, pairs[i]);
                    }
                }
            }
        }
        __syncthreads();   // s_tile, s_w, s_pre are written again by the next tile
    }
    // the block that finishes last: the batch table (and the dense-bed skip);
    // its reads are of words changed by atomics only (bw, ccw), and one fence
    // after the block barrier orders the block's updates before its count
    __syncthreads();
    if (me == 0) {
        __threadfence();
        s_last = atomicAdd(lbc + 1, 1u) == gridDim.x - 1 ? 1u : 0u;
        if (s_last) __threadfence();
    }
    __syncthreads();
    if (!s_last) return;
    if (me == 0) {
        if (skip) *cc_skip = skip - 1u;
        else if (maxc > P) *cc_skip = kDenseSkip;   // a component larger than a block (a dense bed)
    }
    if (!run || __ldcg(ccw + 1)) return;
    const uint nbatch = (nb + tgt - 1) / tgt;
    const uint bmax = (long long)nbatch < nbmax ? nbatch : (uint)nbmax;
    for (uint b = me; b <= bmax; b += blockDim.x) cc_batch_entry(b, nb, tgt, nbmax, nbb, P, Q, bw, batch, ccw);
}

// ------------------------------------------------------------ pair force
// Contact of one listed pair (lo, hi) = (Lp, Ln), the body of
// calculateforcepairD (neiglist.cu:156-233) with the law of dem_law.cuh.
// Geometry from FP64 positions; in the mixed form the overlap is
// (s^2 - d^2)/(s + d) with the numerator formed in FP64 (no cancellation)
// and rounded once, the distance, the division and the rest of the law in
// FP32 except the FP64 history update.  Returns 1 when touching; Fi is the force
// on lo, Ti/Tj the torques on lo/hi; h is the pair's history (in/out).
template <typename Real>
__device__ __forceinline__ int pair_eval(V3<double> xi, V3<double> xj, V3<double> di, V3<double> dj, V3<Real> ai,
                                         V3<Real> aj, Real ri, Real rj, V3<double>& h, const LawParams<Real>& pp,
                                         Real inv_dt, Real density, V3<Real>& Fi, V3<Real>& Ti, V3<Real>& Tj) {
    const V3<double> Dv = xj - xi;
    const double d2 = dot(Dv, Dv);
    const double s = (double)ri + (double)rj;
    Real delta;
    V3<Real> nn;
    if constexpr (sizeof(Real) == 4) {
        // the overlap's numerator s^2 - d^2 in FP64 (no cancellation), the
        // rest in FP32: delta = (s^2 - d^2) / (s + d), n = D / d
        const float d2f = (float)d2;
        const float dist = sqrtf(d2f);
        delta = (float)(s * s - d2) / ((float)s + dist);
        if (!(delta > 0.f && d2f > 0.f)) {
            h = zero3<double>();
            return 0;
        }
        const float inv = 1.f / dist;
        nn = mk((float)Dv.x * inv, (float)Dv.y * inv, (float)Dv.z * inv);
    } else {
        const double dist = sqrt(d2);
        delta = (Real)(s - dist);
        if (!(delta > (Real)0 && dist > 0.0)) {
            h = zero3<double>();
            return 0;
        }
        const double inv = 1.0 / dist;
        nn = cvt<Real>(Dv * inv);
    }
    const Real rstar = ri * rj / (ri + rj);
    const Real mi = density * (Real)8 * ri * ri * ri, mj = density * (Real)8 * rj * rj * rj;
    const Real mstar = mi * mj / (mi + mj);
    const V3<Real> U = cvt<Real>(dj - di) - cross(ri * ai + rj * aj, nn);
    V3<Real> Ft, Mr;
    contact_law<Real>(delta, nn, rstar, mstar, U, ai - aj, h, inv_dt, pp, Fi, Ft, Mr);
    const V3<Real> nxf = cross(nn, Ft);
    Ti = ri * nxf + Mr;
    Tj = rj * nxf - Mr;
    return 1;
}

// Arguments of the PCCP step kernels (pair items, bound particles, free
// particles) and of the window kernel that runs all of a window's steps.
template <typename Real> struct StepArgs {
    long long n, cap;
    const uint *off, *lp, *ln, *ru, *roff, *rk, *wlist, *wcount, *wslot, *bpos, *blist, *flist;
    PRec<Real>* S;                // particle records (in place)
    Planes3<double> W, H;         // wall history, pair history (in place)
    const Real* R;
    float4* Q;                    // displacement since the list (xyz), wall flag (w)
    R4<Real> *pf, *pti, *rfj, *rtj, *wf;
    LawParams<Real> pp, pw;
    ParticleCommon pc;
    Real dtr, inv_dt, density;
    int split;                    // window kernels: bound items per thread of the bound blocks (0: all blocks)
    // cluster batches: when batch != 0 the window's bound particles are
    // stepped by k_batch unless ccw[1] (a component or batch too large) is
    // set, in which case the grid-barrier window kernel steps the window
    int batch;
    const uint* ccw;
    EngineWords* words;
    double *dbgF, *dbgT;
    uint* dbgC;
    // adjoint tape of the window kernel (tx == nullptr: none): per step, the
    // state before the step of every bound particle (tx, td, ta: 3 planes of
    // tnp), its wall history (twh), its total force and torque (tF, tT: xyz
    // per particle), and every listed pair's history before the step (th: 3
    // planes of cap), and its pair-contact count (tc: per particle); the
    // window's first step is tape step tstep0.
    double *tx, *td, *twh, *tF, *tT, *th;
    uint* tc;
    Real* ta;
    long long tnp;
    int tstep0;
};

// Loads of data that other blocks of the same launch write (the window
// kernel): L2-coherent (.cg), never through the non-coherent or L1 paths.
template <bool COH, typename T> __device__ __forceinline__ T ldx(const T* p) {
    if constexpr (COH) return __ldcg(p);
    else return *p;
}
template <bool COH> __device__ __forceinline__ R4<float> ld4(const R4<float>* p) {
    float4 v = COH ? __ldcg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
    return R4<float>{v.x, v.y, v.z, v.w};
}
template <bool COH> __device__ __forceinline__ R4<double> ld4(const R4<double>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 u = COH ? __ldcg(q) : q[0], v = COH ? __ldcg(q + 1) : q[1];
    return R4<double>{u.x, u.y, v.x, v.y};
}
template <bool COH, typename T> __device__ __forceinline__ V3<T> ld3p(Planes3<T> p, uint i) {
    return mk(ldx<COH>(p.x + i), ldx<COH>(p.y + i), ldx<COH>(p.z + i));
}

// Wall item c of particle i (calforceiw's role, neiglist.cu:287-301): history
// W in place (zero when not touching), wall force and torque in wf[2c],
// wf[2c+1].
template <typename Real, bool COH>
__device__ __forceinline__ void wall_item(const StepArgs<Real>& a, long long c, uint i, long long ts = -1) {
    V3<double> x, d;
    V3<Real> av;
    Real r;
    ld_rec<COH>(a.S + i, x, d, av, r);
    const Real m = a.density * (Real)8 * r * r * r;
    V3<double> h = ld3p<COH>(a.W, i);
    if (ts >= 0) {
        double* t = a.twh + 3 * a.tnp * ts;
        t[i] = h.x; t[a.tnp + i] = h.y; t[2 * a.tnp + i] = h.z;
    }
    V3<Real> Fw = zero3<Real>(), Tw = zero3<Real>();
    const int hit = wall_contacts<Real>(a.pc.hx, a.pc.hy, x, cvt<Real>(d), av, r, m, h, a.inv_dt, a.pw, Fw, Tw,
                                        (Real*)nullptr);
    a.W.x[i] = h.x; a.W.y[i] = h.y; a.W.z[i] = h.z;
    R4<Real> a4, b4;
    a4.x = Fw.x; a4.y = Fw.y; a4.z = Fw.z; a4.w = hit ? (Real)1 : (Real)0;
    b4.x = Tw.x; b4.y = Tw.y; b4.z = Tw.z; b4.w = (Real)0;
    a.wf[2 * c] = a4;
    a.wf[2 * c + 1] = b4;
}

// Pair item k = (lo i, hi j) (calculateforcepairD's role, neiglist.cu:156-233):
// history H[k] in place; force/torque on lo in pf[k]/pti[k] (row slot k),
// force/torque on hi in rfj[u]/rtj[u] at the pair's reverse-row slot
// u = ru[k], so the gather reads both of a sphere's row ranges directly.
// .w = 1 marks a contact.
template <typename Real, bool COH>
__device__ __forceinline__ void pair_item(const StepArgs<Real>& a, long long k, uint i, uint j, uint rslot,
                                          long long ts = -1) {
    V3<double> h = mk(ldx<COH>(a.H.x + k), ldx<COH>(a.H.y + k), ldx<COH>(a.H.z + k));
    if (ts >= 0) {
        double* t = a.th + 3 * a.cap * ts;
        t[k] = h.x; t[a.cap + k] = h.y; t[2 * a.cap + k] = h.z;
    }
    V3<double> xi, di, xj, dj;
    V3<Real> ai, aj;
    Real ri, rj;
    ld_rec<COH>(a.S + i, xi, di, ai, ri);
    ld_rec<COH>(a.S + j, xj, dj, aj, rj);
    V3<Real> Fi, Ti, Tj;
    const int c = pair_eval<Real>(xi, xj, di, dj, ai, aj, ri, rj, h, a.pp, a.inv_dt, a.density, Fi, Ti, Tj);
    a.H.x[k] = h.x; a.H.y[k] = h.y; a.H.z[k] = h.z;
    R4<Real> fo, fr;
    if (c) {
        fo.x = Fi.x; fo.y = Fi.y; fo.z = Fi.z; fo.w = (Real)1;
        fr.x = -Fi.x; fr.y = -Fi.y; fr.z = -Fi.z; fr.w = (Real)1;
        R4<Real> a4, b4;
        a4.x = Ti.x; a4.y = Ti.y; a4.z = Ti.z; a4.w = (Real)0;
        b4.x = Tj.x; b4.y = Tj.y; b4.z = Tj.z; b4.w = (Real)0;
        a.pti[k] = a4;
        a.rtj[rslot] = b4;
    } else {
        fo.x = fo.y = fo.z = fo.w = (Real)0;
        fr = fo;
    }
    a.pf[k] = fo;
    a.rfj[rslot] = fr;
}

// Indices of item u: items [0, nw) are the window's wall candidates, items
// [nw, nw + P) the listed pairs.
template <typename Real>
__device__ __forceinline__ void item_indices(const StepArgs<Real>& a, long long u, uint nw, long long items, uint& i,
                                             uint& j, uint& rslot) {
    if (u < (long long)nw) {
        i = a.wlist[u];
    } else if (u < items) {
        const long long k = u - nw;
        i = a.lp[k]; j = a.ln[k]; rslot = a.ru[k];
    }
}

// PCCP pair kernel: wall candidates and listed pairs as one item space on a
// one-wave grid (grid-stride), so every thread takes at most one item per
// pass.
template <typename Real>
__global__ void __launch_bounds__(256) k_pair(StepArgs<Real> a) {
    pdl_trigger();
    const long long stride = (long long)gridDim.x * blockDim.x;
    // list-time data (written by the re-list): safe before pdl_wait
    const uint nw = *a.wcount;
    const uint total = a.off[a.n];
    const long long items = (long long)nw + ((long long)total <= a.cap ? (long long)total : 0ll);
    long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    uint i = 0, j = 0, rslot = 0;
    item_indices(a, u, nw, items, i, j, rslot);
    pdl_wait();
    for (; u < items; u += stride) {
        if (u < (long long)nw) wall_item<Real, false>(a, u, i);
        else pair_item<Real, false>(a, u - nw, i, j, rslot);
        item_indices(a, u + stride, nw, items, i, j, rslot);
    }
}

// --------------------------------------------------- particle update
// Per-step observables are written as one partial per block (no same-address
// atomics in the hot kernels) and reduced on the host when asked for.

// One step of the integrator for one particle, in registers (updatepositionD,
// neiglist.cu:356-360: symplectic Euler in displacement form), then the
// per-step checks.  Every operation is an explicitly rounded intrinsic, so
// the per-step kernels and the free-particle window kernel give bit-identical
// states.  FP64 form: the reference's F dt dt / m term by term; mixed form:
// one reciprocal dt^2/m (FP64) and dt^2/I (FP32) per particle, fused
// multiply-adds into the FP64 displacement and the FP32 rotation.
// The mixed integrator's per-particle factors dt^2/m (FP64) and dt^2/I
// (FP32): constant through a window, so window-long loops compute them once.
__device__ __forceinline__ double mixed_km(double dt, float m) { return __ddiv_rn(__dmul_rn(dt, dt), (double)m); }
__device__ __forceinline__ float mixed_ki(float dtr, float I) { return __fdiv_rn(__fmul_rn(dtr, dtr), I); }

// Mixed step with the factors given (the same operations as integrate<float>).
// FIN = false leaves out the non-finite check, which a caller then makes
// once on the final state (a non-finite position or displacement stays
// non-finite through later steps of the same particle).
template <bool FIN = true>
__device__ __forceinline__ void integrate_k(V3<float> F, V3<float> T, double km, float kI, float half_skin2,
                                            V3<double>& x, V3<double>& d, V3<float>& a, float4& q, uint& flags,
                                            double& mz) {
    d.x = __fma_rn((double)F.x, km, d.x);
    d.y = __fma_rn((double)F.y, km, d.y);
    d.z = __fma_rn((double)F.z, km, d.z);
    a.x = __fmaf_rn(T.x, kI, a.x);
    a.y = __fmaf_rn(T.y, kI, a.y);
    a.z = __fmaf_rn(T.z, kI, a.z);
    x.x = __dadd_rn(x.x, d.x); x.y = __dadd_rn(x.y, d.y); x.z = __dadd_rn(x.z, d.z);
    q.x = __fadd_rn(q.x, __double2float_rn(d.x));
    q.y = __fadd_rn(q.y, __double2float_rn(d.y));
    q.z = __fadd_rn(q.z, __double2float_rn(d.z));
    const float q2 = __fadd_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.y, q.y)), __fmul_rn(q.z, q.z));
    if (q2 > half_skin2) flags |= kStSkin;
    if (FIN && (!isfinite(x.x + x.y + x.z) || !isfinite(d.x + d.y + d.z))) flags |= kStNonfinite;
    mz = x.z > 0.0 ? x.z : 0.0;
}

template <typename Real>
__device__ __forceinline__ void integrate(V3<Real> F, V3<Real> T, Real m, Real I, double dt, Real dtr,
                                          float half_skin2, V3<double>& x, V3<double>& d, V3<Real>& a, float4& q,
                                          uint& flags, double& mz) {
    if constexpr (sizeof(Real) == 8) {
        d.x = __dadd_rn(d.x, __ddiv_rn(__dmul_rn(__dmul_rn(F.x, dt), dt), m));
        d.y = __dadd_rn(d.y, __ddiv_rn(__dmul_rn(__dmul_rn(F.y, dt), dt), m));
        d.z = __dadd_rn(d.z, __ddiv_rn(__dmul_rn(__dmul_rn(F.z, dt), dt), m));
        a.x = __dadd_rn(a.x, __ddiv_rn(__dmul_rn(__dmul_rn(T.x, dtr), dtr), I));
        a.y = __dadd_rn(a.y, __ddiv_rn(__dmul_rn(__dmul_rn(T.y, dtr), dtr), I));
        a.z = __dadd_rn(a.z, __ddiv_rn(__dmul_rn(__dmul_rn(T.z, dtr), dtr), I));
    } else {
        const double km = mixed_km(dt, (float)m);
        const float kI = mixed_ki((float)dtr, (float)I);
        d.x = __fma_rn((double)F.x, km, d.x);
        d.y = __fma_rn((double)F.y, km, d.y);
        d.z = __fma_rn((double)F.z, km, d.z);
        a.x = __fmaf_rn(T.x, kI, a.x);
        a.y = __fmaf_rn(T.y, kI, a.y);
        a.z = __fmaf_rn(T.z, kI, a.z);
    }
    x.x = __dadd_rn(x.x, d.x); x.y = __dadd_rn(x.y, d.y); x.z = __dadd_rn(x.z, d.z);
    q.x = __fadd_rn(q.x, __double2float_rn(d.x));
    q.y = __fadd_rn(q.y, __double2float_rn(d.y));
    q.z = __fadd_rn(q.z, __double2float_rn(d.z));
    const float q2 = __fadd_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.y, q.y)), __fmul_rn(q.z, q.z));
    if (q2 > half_skin2) flags |= kStSkin;
    if (!isfinite(x.x + x.y + x.z) || !isfinite(d.x + d.y + d.z)) flags |= kStNonfinite;
    mz = x.z > 0.0 ? x.z : 0.0;
}

template <typename Real> __device__ __forceinline__ Real sphere_mass(Real density, Real r) {
    return density * (Real)8 * r * r * r;
}

// Gravity + walls (calculateforceiwD, neiglist.cu:238-306) + integrator
// (updatepositionD, neiglist.cu:308-409) for particle i whose pair sums are
// in F/T; writes the new state to the output planes.
template <typename Real, bool WALLS>
__device__ __forceinline__ void particle_finish(long long i, V3<Real> F, V3<Real> T, Real r, V3<double> x,
                                                V3<double> d, V3<Real> a, float4 q, PRec<Real>* So,
                                                float4* __restrict__ Q,
                                                Planes3<double> W, const LawParams<Real>& pw, const ParticleCommon& pc,
                                                Real dtr, Real inv_dt, Real density, double& mz, uint& flags,
                                                uint cnt, double* dbgF, double* dbgT, uint* dbgC) {
    const Real m = sphere_mass(density, r);
    const Real I = (Real)0.4 * m * (r * r);
    if (pc.first) { q.x = 0.f; q.y = 0.f; q.z = 0.f; }   // displacement since the list (dempacking.cu:541)
    uint wflag = __float_as_uint(q.w);
    if (WALLS) {   // walls evaluated here (PP step); the PCCP step adds gathered wall forces before
        F.z += -m;
        const double rd = (double)r;
        const bool touch = (x.z < rd) || (x.x + pc.hx < rd) || (pc.hx - x.x < rd) || (x.y + pc.hy < rd) ||
                           (pc.hy - x.y < rd);
        if (touch || wflag) {
            V3<double> h = wflag ? mk(W.x[i], W.y[i], W.z[i]) : zero3<double>();
            const int hit = wall_contacts<Real>(pc.hx, pc.hy, x, cvt<Real>(d), a, r, m, h, inv_dt, pw, F, T,
                                                (Real*)nullptr);
            if (hit || wflag) { W.x[i] = h.x; W.y[i] = h.y; W.z[i] = h.z; }
            wflag = hit ? 1u : 0u;
        }
    }
    if (dbgF) {   // total force/torque of this step (pairs + gravity + walls), on request
        dbgF[3 * i] = F.x; dbgF[3 * i + 1] = F.y; dbgF[3 * i + 2] = F.z;
        dbgT[3 * i] = T.x; dbgT[3 * i + 1] = T.y; dbgT[3 * i + 2] = T.z;
        dbgC[i] = cnt;
    }
    integrate<Real>(F, T, m, I, pc.dt, dtr, pc.half_skin2, x, d, a, q, flags, mz);
    q.w = __uint_as_float(wflag);
    st_rec(So + i, x, d, a, r);
    Q[i] = q;
}

// Per-step observables: on the observed step (the last of a window, or of an
// eager call) one partial per block -- max height, contact count -- with no
// same-address atomics; on every step the status flags (skin, non-finite),
// OR-ed into the status word by one lane per warp that saw any.
__device__ __forceinline__ void block_observables(double mz, uint cnt, uint flags, int observe, StepPartials part,
                                                  EngineWords* words) {
    if (!observe) {
        flags = __reduce_or_sync(0xffffffffu, flags);
        if (flags && lane_id() == 0) atomicOr(&words->status, flags);
        return;
    }
    __shared__ unsigned long long s_mz[32];   // one entry per warp, blocks of up to 1024 threads
    __shared__ uint s_cnt[32], s_fl[32];
    unsigned long long mb = (unsigned long long)__double_as_longlong(mz);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, mb, o);
        mb = ob > mb ? ob : mb;
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    flags = __reduce_or_sync(0xffffffffu, flags);
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0) { s_mz[warp] = mb; s_cnt[warp] = cnt; s_fl[warp] = flags; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int w = 1; w < nw; w++) { mb = s_mz[w] > mb ? s_mz[w] : mb; cnt += s_cnt[w]; flags |= s_fl[w]; }
        part.maxhz_bits[blockIdx.x] = mb;
        part.contacts[blockIdx.x] = cnt;
        if (flags) atomicOr(&words->status, flags);
    }
}

// Clears the partials [from, to) of an observed step that this kernel does
// not write (they may hold another launch shape's partials).
__device__ __forceinline__ void clear_partials(StepPartials part, size_t from, size_t to) {
    if (threadIdx.x == 0)
        for (size_t b = from + blockIdx.x; b < to; b += gridDim.x) {
            part.maxhz_bits[b] = 0ull;
            part.contacts[b] = 0u;
        }
}

// Bound particle i (a listed pair or a wall candidacy this window): the PCCP
// gather (sumallforceiD's role) through the CSR row and the reverse row of
// the sphere, both read as contiguous ranges, gravity, the gathered wall
// force, then particle_finish.  State is updated in place.
template <typename Real, bool COH>
__device__ __forceinline__ void bound_item(const StepArgs<Real>& a, const ParticleCommon& pc, uint i, Real r, uint ws,
                                           uint total, uint o0, uint o1, uint r0, uint r1, double& mz, uint& cnt,
                                           uint& flags, long long ts = -1) {
    const uint cnt0 = cnt;
    V3<double> x, d;
    V3<Real> av;
    Real rr;
    ld_rec<COH>(a.S + i, x, d, av, rr);
    const float4 q = ldx<COH>(a.Q + i);
    if (ts >= 0) {   // state before the step
        const long long np = a.tnp, o = 3 * np * ts;
        a.tx[o + i] = x.x; a.tx[o + np + i] = x.y; a.tx[o + 2 * np + i] = x.z;
        a.td[o + i] = d.x; a.td[o + np + i] = d.y; a.td[o + 2 * np + i] = d.z;
        a.ta[o + i] = av.x; a.ta[o + np + i] = av.y; a.ta[o + 2 * np + i] = av.z;
    }
    V3<Real> F = zero3<Real>(), T = zero3<Real>();
    if ((long long)total <= a.cap) {
        for (uint k = o0; k < o1; k++) {
            const R4<Real> f = ld4<COH>(a.pf + k);
            if (f.w != (Real)0) {
                const R4<Real> tq = ld4<COH>(a.pti + k);
                F.x += f.x; F.y += f.y; F.z += f.z;
                T.x += tq.x; T.y += tq.y; T.z += tq.z;
                cnt++;
            }
        }
        for (uint u = r0; u < r1; u++) {
            const R4<Real> f = ld4<COH>(a.rfj + u);
            if (f.w != (Real)0) {
                const R4<Real> tq = ld4<COH>(a.rtj + u);
                F.x += f.x; F.y += f.y; F.z += f.z;
                T.x += tq.x; T.y += tq.y; T.z += tq.z;
                cnt++;
            }
        }
    }
    F.z += -sphere_mass(a.density, r);   // gravity, then the walls (calculateforceiwD's order)
    if (ws != kEmpty) {
        const R4<Real> fw = ld4<COH>(a.wf + 2 * ws), tw = ld4<COH>(a.wf + 2 * ws + 1);
        F.x += fw.x; F.y += fw.y; F.z += fw.z;
        T.x += tw.x; T.y += tw.y; T.z += tw.z;
    }
    if (ts >= 0) {   // total force and torque of the step, and its pair contacts
        double* f = a.tF + 3 * a.tnp * ts;
        double* t = a.tT + 3 * a.tnp * ts;
        f[3 * i] = F.x; f[3 * i + 1] = F.y; f[3 * i + 2] = F.z;
        t[3 * i] = T.x; t[3 * i + 1] = T.y; t[3 * i + 2] = T.z;
        a.tc[a.tnp * ts + i] = cnt - cnt0;
    }
    particle_finish<Real, false>(i, F, T, r, x, d, av, q, a.S, a.Q, a.W, a.pw, pc, a.dtr, a.inv_dt, a.density, mz,
                                 flags, cnt, a.dbgF, a.dbgT, a.dbgC);
}

// PCCP particle kernel: one thread per bound particle (blist[t], t < nB =
// bpos[n]).
template <typename Real>
__global__ void __launch_bounds__(256, DEM_PARTICLE_MINB) k_particle(StepArgs<Real> a, StepPartials part,
                                                                     size_t clr1) {
    pdl_trigger();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double mz = 0.0;
    uint cnt = 0, flags = 0;
    // list-time data and the radius: safe before pdl_wait
    const bool live = t < (long long)a.bpos[a.n];
    uint i = 0, ws = kEmpty, total = 0, o0 = 0, o1 = 0, r0 = 0, r1 = 0;
    Real r = (Real)0;
    if (live) {
        i = a.blist[t];
        r = a.R[i];
        ws = a.wslot[i];
        total = a.off[a.n];
        o0 = a.off[i]; o1 = a.off[i + 1]; r0 = a.roff[i]; r1 = a.roff[i + 1];
    }
    pdl_wait();
    if (live) bound_item<Real, false>(a, a.pc, i, r, ws, total, o0, o1, r0, r1, mz, cnt, flags);
    block_observables(mz, cnt, flags, a.pc.observe, part, a.words);
    if (a.pc.observe) clear_partials(part, gridDim.x, clr1);
}

// Free particle i (no listed pair and no wall candidacy in this window): until
// the next re-list it moves under gravity alone, independent of every other
// particle (the skin check guards that).  Steps slot0 .. slot0+nsteps-1 of the
// window run in registers: the state is read once and written once, with the
// per-step arithmetic of particle_finish.  mz_obs receives the height after
// step observe_slot (if in range).
template <typename Real>
__device__ __forceinline__ void free_item(const StepArgs<Real>& a, const PRec<Real>* Sin, PRec<Real>* Sout, uint i,
                                          int slot0, int nsteps, int observe_slot, bool rec, double& mz_obs,
                                          uint& flags) {
    V3<double> x, d;
    V3<Real> av;
    Real r;
    ld_rec<false>(Sin + i, x, d, av, r);
    float4 q = a.Q[i];
    const Real m = sphere_mass(a.density, r);
    const Real I = (Real)0.4 * m * (r * r);
    const double km = mixed_km(a.pc.dt, (float)m);
    const float kI = mixed_ki((float)a.dtr, (float)I);
    const Real gz = (Real)0 + -sphere_mass(a.density, r);   // the force of every step: gravity
    for (int s = slot0; s < slot0 + nsteps; s++) {
        if (s == 0) { q.x = 0.f; q.y = 0.f; q.z = 0.f; }
        V3<Real> F = zero3<Real>(), T = zero3<Real>();
        F.z = gz;
        if (rec) {
            a.dbgF[3 * i] = F.x; a.dbgF[3 * i + 1] = F.y; a.dbgF[3 * i + 2] = F.z;
            a.dbgT[3 * i] = T.x; a.dbgT[3 * i + 1] = T.y; a.dbgT[3 * i + 2] = T.z;
            a.dbgC[i] = 0;
        }
        double mz;
        if constexpr (sizeof(Real) == 4)   // the factors computed once (the same values integrate computes)
            integrate_k<false>(F, T, km, kI, a.pc.half_skin2, x, d, av, q, flags, mz);
        else
            integrate<Real>(F, T, m, I, a.pc.dt, a.dtr, a.pc.half_skin2, x, d, av, q, flags, mz);
        if (s == observe_slot) mz_obs = mz;
    }
    if constexpr (sizeof(Real) == 4)
        if (!isfinite(x.x + x.y + x.z) || !isfinite(d.x + d.y + d.z)) flags |= kStNonfinite;
    st_rec(Sout + i, x, d, av, r);
    a.Q[i] = q;
}

// Free particles (flist[t], t < n - nB), slots slot0 .. slot0+nsteps-1.
template <typename Real>
__global__ void __launch_bounds__(256) k_free_run(StepArgs<Real> a, int slot0, int nsteps, int observe_slot,
                                                  StepPartials part, size_t clr0, size_t clr1) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double mz_obs = 0.0;
    uint flags = 0;
    if (t < a.n - (long long)a.bpos[a.n])
        free_item<Real>(a, a.S, a.S, a.flist[t], slot0, nsteps, observe_slot, a.dbgF != nullptr && nsteps == 1, mz_obs,
                        flags);
    const int observe = observe_slot >= slot0 && observe_slot < slot0 + nsteps;
    block_observables(mz_obs, 0u, flags, observe, part, a.words);
    if (observe) clear_partials(part, clr0, clr1);
}

// Grid-wide barrier of the window kernel (all blocks co-resident: cooperative
// launch).  bar[0] is the launch's arrival counter and bar[kBarGiveUp] its
// give-up word, both zeroed before every launch.  The wait is bounded: a
// block that waits longer than kBarrierNs of %globaltimer AND kBarrierMinPolls
// polls (or kBarrierMaxPolls polls in any case) records kStBarrier in the
// status word and raises the launch's give-up word, after which the launch's
// remaining barriers do not wait, so it always ends.  The timer is restarted
// if it steps backwards, and the poll floor keeps a forward step of the timer
// (the driver recalibrates %globaltimer) from ending a healthy wait.  A later
// launch starts with its own give-up word clear.
constexpr unsigned long long kBarrierNs = 1000000000ull;   // 1 s
constexpr uint kBarrierMinPolls = 200000u;                 // >= ~0.1 s of polling
constexpr uint kBarrierMaxPolls = 20000000u;               // a few seconds at most
constexpr int kBarGiveUp = 32;                             // bar[32]: own 128-byte line
constexpr int kBarWords = 64;                              // words zeroed per launch

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint ld_acquire(const uint* p) {
    uint v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(uint* p, uint v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Barrier number `k` (0, 1, ...) among the first `nblk` blocks of a
// window-kernel launch (the blocks that hold bound work): every one adds 1 to
// the arrival counter with release semantics and waits, with acquire loads,
// until it reaches (k+1) x nblk (bounded as above).
__device__ __forceinline__ void grid_arrive(uint* bar) {
    __syncthreads();
    if (threadIdx.x == 0) red_release_add(bar, 1u);
}
__device__ __forceinline__ void grid_wait(uint* bar, uint k, uint nblk, EngineWords* words) {
    if (threadIdx.x == 0) {
        const uint target = (k + 1u) * nblk;
        if (!ld_acquire(bar + kBarGiveUp)) {
            unsigned long long t0 = global_ns();
            uint polls = 0;
            while (ld_acquire(bar) < target) {
                __nanosleep(20);
                ++polls;
                const unsigned long long now = global_ns();
                if (now < t0) t0 = now;   // the timer stepped back: restart the clock
                if ((now - t0 > kBarrierNs && polls > kBarrierMinPolls) || polls > kBarrierMaxPolls) {
                    atomicOr(&words->status, kStBarrier);
                    atomicExch(bar + kBarGiveUp, 1u);
                    break;
                }
            }
        }
    }
    __syncthreads();
}
__device__ __forceinline__ void grid_barrier(uint* bar, uint k, uint nblk, EngineWords* words) {
    grid_arrive(bar);
    grid_wait(bar, k, nblk, words);
}

// Check of the bounded wait: the launch's one block arrives once and waits
// for barrier 1, which needs a second arrival that never comes; the wait must
// give up, record kStBarrier and raise the give-up word.  `spent` receives
// the nanoseconds waited.
__global__ void k_barrier_check(uint* bar, EngineWords* words, unsigned long long* spent) {
    const unsigned long long t0 = global_ns();
    grid_arrive(bar);                    // the counter reaches 1
    grid_wait(bar, 1, gridDim.x, words);  // waits for 2 (one block): gives up
    if (threadIdx.x == 0) *spent = global_ns() - t0;
}

// The whole window's steps in one cooperative launch (after the re-list).
// The launch's blocks are split by the window's work: the first `nbb` blocks
// (bound_blocks) hold the bound work and step it together -- per step, phase
// 1 = wall + pair items, barrier among them, phase 2 = bound particles,
// barrier -- while the other blocks run every free particle through all K
// steps in registers, without any barrier (a free particle meets nothing
// before the next re-list, so its steps need no other particle).  When the
// bound work needs every block (a dense bed), the free particles are dealt
// over the steps instead: 1/K of them in each phase 2.  Items and particles
// keep their thread for the whole window; data written by other blocks is
// read with L2-coherent loads.  The arithmetic is that of the per-step
// kernels (same device functions), so the states are bit-identical whatever
// the split.  Observables of the window's last step go to `part` (one
// partial per block; the slot's remaining partials are cleared).
constexpr int kWinThreads = 512;

// Blocks of a window launch of `grid` blocks that take the bound work:
// `split` bound items (or bound particles, whichever are more) per thread,
// ceil(max(items, nb) / (kWinThreads * split)) blocks; all of them when split
// <= 0 or when every particle is bound; none when there is no bound work.
__device__ __forceinline__ uint bound_blocks(long long items, long long nb, long long nf, uint grid, int split) {
    if (split <= 0 || nf == 0) return grid;
    const long long need = items > nb ? items : nb;
    const long long per = (long long)kWinThreads * split;
    const long long b = (need + per - 1) / per;
    return (uint)(b < (long long)grid ? b : (long long)grid);
}

// Free particles flist[fid], flist[fid + stride], ... through all K steps
// (the free-only blocks of a split window launch).
template <typename Real>
__device__ __forceinline__ void free_sweep(const StepArgs<Real>& a, const PRec<Real>* Sin, PRec<Real>* Sout,
                                           long long fid, long long stride, long long nf, int K, double& mz,
                                           uint& flags) {
    for (long long t = fid; t < nf; t += stride) {
        double mzi = 0.0;
        free_item<Real>(a, Sin, Sout, a.flist[t], 0, K, K - 1, false, mzi, flags);
        mz = fmax(mz, mzi);
    }
}

template <typename Real, int MINB>
__global__ void __launch_bounds__(kWinThreads, MINB) k_window(StepArgs<Real> a, int K, StepPartials part, size_t npart,
                                                           uint* bar) {
    if (a.batch && !a.ccw[1]) return;   // the cluster batches (k_batch) step this window
    uint nbar = 0;
    const uint nw = *a.wcount;
    const uint total = a.off[a.n];
    const long long items = (long long)nw + ((long long)total <= a.cap ? (long long)total : 0ll);
    // a batched window's free particles are k_free_run's (beside this kernel)
    const long long nb = a.bpos[a.n], nf = a.batch ? 0 : a.n - nb;
    const uint nbb = bound_blocks(items, nb, nf, gridDim.x, a.split);
    const long long warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double mz = 0.0;
    uint cnt = 0, flags = 0;
    if (blockIdx.x >= nbb) {   // free-only block
        const uint nfb = gridDim.x - nbb;
        free_sweep<Real>(a, a.S, a.S, (warp * nfb + (blockIdx.x - nbb)) * 32 + lane, (long long)nfb * kWinThreads, nf,
                         K, mz, flags);
        block_observables(mz, cnt, flags, 1, part, a.words);
        clear_partials(part, gridDim.x, npart);
        return;
    }
    const bool deal_free = nbb == gridDim.x;   // no free-only blocks: free particles go with the steps
    const long long nthr = (long long)nbb * blockDim.x;
    // work index: warps dealt round-robin over the bound blocks (SMs), lanes
    // contiguous, so every phase spreads over all of them
    const long long tid = (warp * nbb + blockIdx.x) * 32 + lane;
    // this thread's first item and first bound particle: indices kept in
    // registers for the whole window (further ones are reloaded per step)
    uint i0 = 0, j0 = 0, s0 = 0;
    item_indices(a, tid, nw, items, i0, j0, s0);
    uint b0 = 0, ws0 = kEmpty, o00 = 0, o10 = 0, r00 = 0, r10 = 0;
    Real rb0 = (Real)0;
    if (tid < nb) {
        b0 = a.blist[tid];
        rb0 = a.R[b0];
        ws0 = a.wslot[b0];
        o00 = a.off[b0]; o10 = a.off[b0 + 1]; r00 = a.roff[b0]; r10 = a.roff[b0 + 1];
    }
    ParticleCommon pc = a.pc;
    for (int s = 0; s < K; s++) {
        const long long ts = a.tx ? (long long)a.tstep0 + s : -1ll;
        // phase 1: wall and pair items
        for (long long u = tid; u < items; u += nthr) {
            uint i = i0, j = j0, rslot = s0;
            if (u != tid) item_indices(a, u, nw, items, i, j, rslot);
            if (u < (long long)nw) wall_item<Real, true>(a, u, i, ts);
            else pair_item<Real, true>(a, u - nw, i, j, rslot, ts);
        }
        grid_barrier(bar, nbar++, nbb, a.words);
        // phase 2: bound particles; with no free-only blocks, this step's
        // share of the free particles (each run through all K steps) from the
        // other end of the work range
        pc.first = s == 0 ? 1 : 0;
        for (long long t = tid; t < nb; t += nthr) {
            double mzi = 0.0;
            uint ci = 0;
            if (t == tid) {
                bound_item<Real, true>(a, pc, b0, rb0, ws0, total, o00, o10, r00, r10, mzi, ci, flags, ts);
            } else {
                const uint i = a.blist[t];
                bound_item<Real, true>(a, pc, i, a.R[i], a.wslot[i], total, a.off[i], a.off[i + 1], a.roff[i],
                                       a.roff[i + 1], mzi, ci, flags, ts);
            }
            if (s == K - 1) { mz = fmax(mz, mzi); cnt += ci; }
        }
        if (deal_free) {
            const long long f0 = nf * s / K, f1 = nf * (s + 1) / K;
            for (long long t = f0 + (nthr - 1 - tid); t < f1; t += nthr) {
                double mzi = 0.0;
                free_item<Real>(a, a.S, a.S, a.flist[t], 0, K, K - 1, false, mzi, flags);
                mz = fmax(mz, mzi);
            }
        }
        if (s < K - 1) grid_barrier(bar, nbar++, nbb, a.words);
    }
    block_observables(mz, cnt, flags, 1, part, a.words);
    clear_partials(part, gridDim.x, npart);
}

// One block steps whole batches of small components through all K steps of
// the window in shared memory: per step, the batch's pair items (pair_eval)
// and wall items (wall_contacts), a block barrier, the batch's particles
// (gather in list order: own row, then reverse row; gravity, walls,
// integrate), a block barrier.  The operations and their order are those of
// pair_item / wall_item / bound_item, so the states are those of the
// grid-barrier window kernel and of the per-step kernels, bit for bit.  The
// free particles run concurrently in k_free_run.  Observables of the window's
// last step go to `part` (one partial per block; [gridDim.x, clr1) cleared).
template <typename Real> struct BatchSmem {
    V3<double>* x; V3<double>* d; V3<Real>* a; Real* r; float4* q; V3<double>* wh;
    double* km; float* ki;       // the mixed integrator's factors dt^2/m, dt^2/I
    uint *gid, *ws, *pb, *pl, *rb, *rl, *wl, *wli;   // wl: wall-candidate flags then slots; wli: their list
    R4<Real>* wf; R4<Real>* wt;
    uint *plo, *phi, *pk, *prv;
    V3<double>* ph;
    R4<Real> *fo, *ti, *tj;
    uint* scan;
};
// The block's shared-memory layout: byte offsets fixed at compile time (each
// array 16-byte aligned), so every array is the base plus a constant.
template <typename Real> struct BatchOff {
    static constexpr uint P = BatchCap<Real>::P, Q = BatchCap<Real>::Q;
    static constexpr size_t al(size_t b) { return (b + 15) & ~size_t(15); }
    static constexpr size_t x = 0;
    static constexpr size_t d = x + al(P * sizeof(V3<double>));
    static constexpr size_t wh = d + al(P * sizeof(V3<double>));
    static constexpr size_t q = wh + al(P * sizeof(V3<double>));
    static constexpr size_t wf = q + al(P * sizeof(float4));
    static constexpr size_t wt = wf + al(P * sizeof(R4<Real>));
    static constexpr size_t a = wt + al(P * sizeof(R4<Real>));
    static constexpr size_t r = a + al(P * sizeof(V3<Real>));
    static constexpr size_t km = r + al(P * sizeof(Real));
    static constexpr size_t ki = km + al(P * sizeof(double));
    static constexpr size_t gid = ki + al(P * sizeof(float));
    static constexpr size_t ws = gid + al(P * 4);
    static constexpr size_t pb = ws + al(P * 4);
    static constexpr size_t pl = pb + al(P * 4);
    static constexpr size_t rb = pl + al(P * 4);
    static constexpr size_t rl = rb + al(P * 4);
    static constexpr size_t wl = rl + al(P * 4);
    static constexpr size_t wli = wl + al(P * 4);
    static constexpr size_t ph = wli + al(P * 4);
    static constexpr size_t fo = ph + al(Q * sizeof(V3<double>));
    static constexpr size_t ti = fo + al(Q * sizeof(R4<Real>));
    static constexpr size_t tj = ti + al(Q * sizeof(R4<Real>));
    static constexpr size_t plo = tj + al(Q * sizeof(R4<Real>));
    static constexpr size_t phi = plo + al(Q * 4);
    static constexpr size_t pk = phi + al(Q * 4);
    static constexpr size_t prv = pk + al(Q * 4);
    static constexpr size_t scan = prv + al(Q * 4);
    static constexpr size_t end = scan + al(34 * 4);
};
template <typename Real> __host__ __device__ inline size_t batch_smem_layout(unsigned char* base, BatchSmem<Real>* L) {
    using O = BatchOff<Real>;
    if (L) {
        L->x = (V3<double>*)(base + O::x); L->d = (V3<double>*)(base + O::d); L->wh = (V3<double>*)(base + O::wh);
        L->q = (float4*)(base + O::q); L->wf = (R4<Real>*)(base + O::wf); L->wt = (R4<Real>*)(base + O::wt);
        L->a = (V3<Real>*)(base + O::a); L->r = (Real*)(base + O::r); L->km = (double*)(base + O::km);
        L->ki = (float*)(base + O::ki); L->gid = (uint*)(base + O::gid); L->ws = (uint*)(base + O::ws);
        L->pb = (uint*)(base + O::pb); L->pl = (uint*)(base + O::pl); L->rb = (uint*)(base + O::rb);
        L->rl = (uint*)(base + O::rl); L->wl = (uint*)(base + O::wl); L->wli = (uint*)(base + O::wli);
        L->ph = (V3<double>*)(base + O::ph); L->fo = (R4<Real>*)(base + O::fo); L->ti = (R4<Real>*)(base + O::ti);
        L->tj = (R4<Real>*)(base + O::tj); L->plo = (uint*)(base + O::plo); L->phi = (uint*)(base + O::phi);
        L->pk = (uint*)(base + O::pk); L->prv = (uint*)(base + O::prv); L->scan = (uint*)(base + O::scan);
    }
    return O::end;
}

// k_batch's register cap: the mixed kernel at 80 (40 bytes of spills) leaves
// room on its SM for two blocks of k_free_run (256 x 48 registers), which
// then runs beside the batches instead of after them; FP64 keeps 128.
template <typename Real> struct BatchRegs { static constexpr int value = sizeof(Real) == 4 ? 80 : 128; };

template <typename Real>
__global__ void __maxnreg__(BatchRegs<Real>::value) k_batch(StepArgs<Real> a, int K, const uint* __restrict__ corder,
                                                         const uint* __restrict__ cbatch, uint* cloc,
                                                         StepPartials part, size_t clr1) {
    if (a.ccw[1]) return;   // a component or a batch too large: the grid-barrier window kernel has the window
    extern __shared__ __align__(16) unsigned char smem[];
    BatchSmem<Real> L;
    batch_smem_layout<Real>(smem, &L);
    const long long nb = a.bpos[a.n];
    const uint tgt = a.ccw[3];
    if (tgt == 0u) {   // no batch table (cannot happen while ccw[1] is clear): reported, nothing stepped
        if (threadIdx.x == 0) wait_gave_up(a.words, kWaitBatchTable);
        return;
    }
    const uint nbatch = (uint)((nb + tgt - 1) / tgt);
    double mz = 0.0;
    uint cnt = 0, flags = 0;
    ParticleCommon pc = a.pc;
    constexpr uint P = BatchCap<Real>::P, Q = BatchCap<Real>::Q;
    for (uint bi = blockIdx.x; bi < nbatch; bi += gridDim.x) {
        const uint s0 = cbatch[bi], s1 = cbatch[bi + 1];
        // a batch that is not whole components (a re-list that cut it wrongly)
        // is skipped and reported (capacity status), never stepped; every
        // test below ends in a block-wide vote, so all threads skip together
        if (s1 < s0 || s1 > (uint)nb || s1 - s0 > P) {
            if (threadIdx.x == 0) atomicOr(&a.words->status, kStCapacity);
            continue;
        }
        const uint m = s1 - s0;
        uint bad = 0;
        // the batch's particles into shared memory
        for (uint p = threadIdx.x; p < m; p += blockDim.x) {
            const uint i = corder[s0 + p];
            if (i >= (uint)a.n) { bad = 1u; continue; }
            cloc[i] = p;
            L.gid[p] = i;
            V3<double> x, d;
            V3<Real> av;
            Real r;
            ld_rec<false>(a.S + i, x, d, av, r);
            L.x[p] = x; L.d[p] = d; L.a[p] = av; L.r[p] = r;
            L.q[p] = a.Q[i];
            L.wh[p] = mk(a.W.x[i], a.W.y[i], a.W.z[i]);
            L.ws[p] = a.wslot[i];
            L.wl[p] = a.wslot[i] != kEmpty ? 1u : 0u;
            L.pl[p] = a.off[i + 1] - a.off[i];
            L.rl[p] = a.roff[i + 1] - a.roff[i];
            const Real mass = sphere_mass(a.density, r);
            L.km[p] = mixed_km(a.pc.dt, (float)mass);
            L.ki[p] = mixed_ki((float)a.dtr, (float)((Real)0.4 * mass * (r * r)));
        }
        if (__syncthreads_or(bad)) {
            if (threadIdx.x == 0) atomicOr(&a.words->status, kStCapacity);
            continue;
        }
        const uint npairs = block_exscan(L.pl, L.pb, m, L.scan);
        const uint nrev = block_exscan(L.rl, L.rb, m, L.scan);
        if (npairs > Q || nrev != npairs) {   // not whole components: skipped, reported
            if (threadIdx.x == 0) atomicOr(&a.words->status, kStCapacity);
            continue;
        }
        const uint nwall = block_exscan(L.wl, L.wl, m, L.scan);   // the batch's wall candidates, listed
        for (uint p = threadIdx.x; p < m; p += blockDim.x)
            if (L.ws[p] != kEmpty) L.wli[L.wl[p]] = p;
        // the batch's pairs: own rows in list order, reverse rows as pair
        // slots; each partner must be a particle of this batch (and each
        // particle once in it)
        for (uint p = threadIdx.x; p < m; p += blockDim.x) {
            const uint i = L.gid[p], o0 = a.off[i], b0 = L.pb[p];
            if (__ldcg(cloc + i) != p) bad = 1u;
            for (uint e = 0; e < L.pl[p]; e++) {
                const uint k = o0 + e;
                const uint j = a.ln[k];
                const uint hi = j < (uint)a.n ? __ldcg(cloc + j) : 0xffffffffu;
                if (hi >= m || L.gid[hi] != j) { bad = 1u; break; }
                L.plo[b0 + e] = p;
                L.phi[b0 + e] = hi;
                L.pk[b0 + e] = k;
                L.ph[b0 + e] = mk(a.H.x[k], a.H.y[k], a.H.z[k]);
            }
            const uint r0 = a.roff[i], rb = L.rb[p];
            for (uint u = 0; u < L.rl[p] && !bad; u++) {
                const uint k = a.rk[r0 + u];
                const uint lo = a.lp[k];
                const uint q = lo < (uint)a.n ? __ldcg(cloc + lo) : 0xffffffffu;
                if (q >= m || L.gid[q] != lo) { bad = 1u; break; }
                const uint slot = L.pb[q] + (k - a.off[lo]);
                if (slot >= npairs) { bad = 1u; break; }
                L.prv[rb + u] = slot;
            }
        }
        if (__syncthreads_or(bad)) {
            if (threadIdx.x == 0) atomicOr(&a.words->status, kStCapacity);
            continue;
        }
        for (int st = 0; st < K; st++) {
            const long long ts = a.tx ? (long long)a.tstep0 + st : -1ll;
            // pair items and wall items (pair_item, wall_item), one item per thread
            for (uint u = threadIdx.x; u < npairs + nwall; u += blockDim.x) {
                if (u < npairs) {
                    const uint e = u;
                    const uint lo = L.plo[e], hi = L.phi[e];
                    V3<double> h = L.ph[e];
                    if (ts >= 0) {
                        double* t = a.th + 3 * a.cap * ts;
                        const uint k = L.pk[e];
                        t[k] = h.x; t[a.cap + k] = h.y; t[2 * a.cap + k] = h.z;
                    }
                    V3<Real> Fi, Ti, Tj;
                    const int c = pair_eval<Real>(L.x[lo], L.x[hi], L.d[lo], L.d[hi], L.a[lo], L.a[hi], L.r[lo],
                                                  L.r[hi], h, a.pp, a.inv_dt, a.density, Fi, Ti, Tj);
                    L.ph[e] = h;
                    R4<Real> fo;
                    if (c) {
                        fo.x = Fi.x; fo.y = Fi.y; fo.z = Fi.z; fo.w = (Real)1;
                        R4<Real> t4;
                        t4.x = Ti.x; t4.y = Ti.y; t4.z = Ti.z; t4.w = (Real)0;
                        L.ti[e] = t4;
                        t4.x = Tj.x; t4.y = Tj.y; t4.z = Tj.z;
                        L.tj[e] = t4;
                    } else {
                        fo.x = fo.y = fo.z = fo.w = (Real)0;
                    }
                    L.fo[e] = fo;
                } else {
                    const uint p = L.wli[u - npairs];
                    const Real r = L.r[p];
                    const Real mass = a.density * (Real)8 * r * r * r;
                    V3<double> h = L.wh[p];
                    if (ts >= 0) {
                        double* t = a.twh + 3 * a.tnp * ts;
                        const uint i = L.gid[p];
                        t[i] = h.x; t[a.tnp + i] = h.y; t[2 * a.tnp + i] = h.z;
                    }
                    V3<Real> Fw = zero3<Real>(), Tw = zero3<Real>();
                    const int hit = wall_contacts<Real>(a.pc.hx, a.pc.hy, L.x[p], cvt<Real>(L.d[p]), L.a[p], r, mass,
                                                        h, a.inv_dt, a.pw, Fw, Tw, (Real*)nullptr);
                    L.wh[p] = h;
                    R4<Real> a4, b4;
                    a4.x = Fw.x; a4.y = Fw.y; a4.z = Fw.z; a4.w = hit ? (Real)1 : (Real)0;
                    b4.x = Tw.x; b4.y = Tw.y; b4.z = Tw.z; b4.w = (Real)0;
                    L.wf[p] = a4;
                    L.wt[p] = b4;
                }
            }
            __syncthreads();
            // particles (bound_item, particle_finish)
            pc.first = st == 0 ? 1 : 0;
            for (uint p = threadIdx.x; p < m; p += blockDim.x) {
                V3<double> x = L.x[p], d = L.d[p];
                V3<Real> av = L.a[p];
                const Real r = L.r[p];
                float4 q = L.q[p];
                const uint i = L.gid[p];
                if (ts >= 0) {
                    const long long np = a.tnp, o = 3 * np * ts;
                    a.tx[o + i] = x.x; a.tx[o + np + i] = x.y; a.tx[o + 2 * np + i] = x.z;
                    a.td[o + i] = d.x; a.td[o + np + i] = d.y; a.td[o + 2 * np + i] = d.z;
                    a.ta[o + i] = av.x; a.ta[o + np + i] = av.y; a.ta[o + 2 * np + i] = av.z;
                }
                V3<Real> F = zero3<Real>(), T = zero3<Real>();
                uint ci = 0;
                for (uint e = L.pb[p], e1 = L.pb[p] + L.pl[p]; e < e1; e++) {
                    const R4<Real> f = L.fo[e];
                    if (f.w != (Real)0) {
                        const R4<Real> tq = L.ti[e];
                        F.x += f.x; F.y += f.y; F.z += f.z;
                        T.x += tq.x; T.y += tq.y; T.z += tq.z;
                        ci++;
                    }
                }
                for (uint v = L.rb[p], v1 = L.rb[p] + L.rl[p]; v < v1; v++) {
                    const uint e = L.prv[v];
                    const R4<Real> f = L.fo[e];
                    if (f.w != (Real)0) {
                        const R4<Real> tq = L.tj[e];
                        F.x += -f.x; F.y += -f.y; F.z += -f.z;
                        T.x += tq.x; T.y += tq.y; T.z += tq.z;
                        ci++;
                    }
                }
                F.z += -sphere_mass(a.density, r);
                if (L.ws[p] != kEmpty) {
                    const R4<Real> fw = L.wf[p], tw = L.wt[p];
                    F.x += fw.x; F.y += fw.y; F.z += fw.z;
                    T.x += tw.x; T.y += tw.y; T.z += tw.z;
                }
                if (ts >= 0) {
                    double* f = a.tF + 3 * a.tnp * ts;
                    double* t = a.tT + 3 * a.tnp * ts;
                    f[3 * i] = F.x; f[3 * i + 1] = F.y; f[3 * i + 2] = F.z;
                    t[3 * i] = T.x; t[3 * i + 1] = T.y; t[3 * i + 2] = T.z;
                    a.tc[a.tnp * ts + i] = ci;
                }
                const Real mass = sphere_mass(a.density, r);
                const Real I = (Real)0.4 * mass * (r * r);
                if (pc.first) { q.x = 0.f; q.y = 0.f; q.z = 0.f; }
                const uint wflag = __float_as_uint(q.w);
                double mzi;
                if constexpr (sizeof(Real) == 4)
                    integrate_k(F, T, L.km[p], L.ki[p], pc.half_skin2, x, d, av, q, flags, mzi);
                else
                    integrate<Real>(F, T, mass, I, pc.dt, a.dtr, pc.half_skin2, x, d, av, q, flags, mzi);
                q.w = __uint_as_float(wflag);
                L.x[p] = x; L.d[p] = d; L.a[p] = av; L.q[p] = q;
                if (st == K - 1) { mz = fmax(mz, mzi); cnt += ci; }
            }
            __syncthreads();
        }
        // back to global memory
        for (uint p = threadIdx.x; p < m; p += blockDim.x) {
            const uint i = L.gid[p];
            st_rec(a.S + i, L.x[p], L.d[p], L.a[p], L.r[p]);
            a.Q[i] = L.q[p];
            const V3<double> h = L.wh[p];
            a.W.x[i] = h.x; a.W.y[i] = h.y; a.W.z[i] = h.z;
        }
        for (uint e = threadIdx.x; e < npairs; e += blockDim.x) {
            const uint k = L.pk[e];
            const V3<double> h = L.ph[e];
            a.H.x[k] = h.x; a.H.y[k] = h.y; a.H.z[k] = h.z;
        }
        __syncthreads();   // the shared arrays are refilled by the next batch
    }
    block_observables(mz, cnt, flags, 1, part, a.words);
    clear_partials(part, gridDim.x, clr1);
}

// PP (particle-parallel, the paper's Figure 1(b)): each particle evaluates all
// of its pairs itself -- its own row (it is lo) and its reverse row (it is hi)
// -- and its walls, then integrates.  Each pair is evaluated by both of its
// particles with the same arguments in the same order, so the two results are
// bit-identical; only lo writes the pair's new history.  State and history
// are read from the "in" buffers and written to the "out" buffers (ping-pong).
template <typename Real, bool COH>
__device__ __forceinline__ void pp_item(long long i, Real r, uint total, uint o0, uint o1, uint r0, uint r1,
                                        const uint* __restrict__ rk, const uint* __restrict__ lp,
                                        const uint* __restrict__ ln, long long cap, const PRec<Real>* Si, PRec<Real>* So,
                                        float4* Q, Planes3<double> W, Planes3<double> Hi, Planes3<double> Ho,
                                        const LawParams<Real>& pp, const LawParams<Real>& pw, const ParticleCommon& pc,
                                        Real dtr, Real inv_dt, Real density, double& mz, uint& cnt, uint& flags,
                                        double* dbgF, double* dbgT, uint* dbgC) {
    V3<double> x, d;
    V3<Real> a;
    Real rr;
    ld_rec<COH>(Si + i, x, d, a, rr);
    const float4 q = ldx<COH>(Q + i);
    V3<Real> F = zero3<Real>(), T = zero3<Real>();
    if ((long long)total <= cap) {
        for (uint k = o0; k < o1; k++) {
            const uint j = ln[k];
            V3<double> h = mk(ldx<COH>(Hi.x + k), ldx<COH>(Hi.y + k), ldx<COH>(Hi.z + k));
            V3<double> xj, dj;
            V3<Real> aj;
            Real rj;
            ld_rec<COH>(Si + j, xj, dj, aj, rj);
            V3<Real> Fl, Tl, Th;
            const int c = pair_eval<Real>(x, xj, d, dj, a, aj, r, rj, h, pp, inv_dt, density, Fl, Tl, Th);
            Ho.x[k] = h.x; Ho.y[k] = h.y; Ho.z[k] = h.z;
            if (c) { F += Fl; T += Tl; cnt++; }
        }
        for (uint u = r0; u < r1; u++) {
            const uint k = rk[u];
            if (k >= total) continue;
            const uint j = lp[k];
            V3<double> h = mk(ldx<COH>(Hi.x + k), ldx<COH>(Hi.y + k), ldx<COH>(Hi.z + k));
            V3<double> xj, dj;
            V3<Real> aj;
            Real rj;
            ld_rec<COH>(Si + j, xj, dj, aj, rj);
            V3<Real> Fl, Tl, Th;
            const int c = pair_eval<Real>(xj, x, dj, d, aj, a, rj, r, h, pp, inv_dt, density, Fl, Tl, Th);
            if (c) { F -= Fl; T += Th; cnt++; }
        }
    }
    particle_finish<Real, true>(i, F, T, r, x, d, a, q, So, Q, W, pw, pc, dtr, inv_dt, density, mz, flags, cnt, dbgF,
                                dbgT, dbgC);
}

template <typename Real>
__global__ void __launch_bounds__(256, DEM_PP_MINB) k_step_pp(
    long long n, const uint* __restrict__ off, const uint* __restrict__ roff, const uint* __restrict__ rk,
    const uint* __restrict__ lp, const uint* __restrict__ ln, long long cap, const PRec<Real>* __restrict__ Si,
    PRec<Real>* __restrict__ So, const Real* __restrict__ R, float4* __restrict__ Q, Planes3<double> W, Planes3<double> Hi, Planes3<double> Ho, LawParams<Real> pp,
    LawParams<Real> pw, ParticleCommon pc, Real dtr, Real inv_dt, Real density, StepPartials part,
    EngineWords* words, double* dbgF, double* dbgT, uint* dbgC, size_t clr0, size_t clr1) {
    pdl_trigger();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double mz = 0.0;
    uint cnt = 0, flags = 0;
    // list-time data and the radius: safe before pdl_wait
    Real r = (Real)0;
    uint total = 0, o0 = 0, o1 = 0, r0 = 0, r1 = 0;
    if (i < n) {
        r = R[i];
        total = off[n];
        o0 = off[i]; o1 = off[i + 1]; r0 = roff[i]; r1 = roff[i + 1];
    }
    pdl_wait();
    if (i < n)
        pp_item<Real, false>(i, r, total, o0, o1, r0, r1, rk, lp, ln, cap, Si, So, Q, W, Hi, Ho, pp, pw, pc, dtr, inv_dt,
                             density, mz, cnt, flags, dbgF, dbgT, dbgC);
    block_observables(mz, cnt, flags, pc.observe, part, words);
    if (pc.observe) clear_partials(part, clr0, clr1);
}

// PP window kernel (one cooperative launch per window, as k_window, with the
// same split of its blocks): per step, every bound particle runs pp_item from
// the "in" buffers into the "out" buffers, one barrier among the bound blocks
// per step, then the buffers swap; the free particles run all K steps in
// registers (read from the window's first state buffer, written to its last),
// in the free-only blocks or, with none, 1/K of them per step.  Same device
// functions as the per-step PP kernel, so the states are bit-identical.
template <typename Real>
__global__ void __launch_bounds__(kWinThreads, 1) k_window_pp(StepArgs<Real> a, PRec<Real>* S0, PRec<Real>* S1,
                                                              Planes3<double> H0, Planes3<double> H1, int K,
                                                              StepPartials part, size_t npart, uint* bar) {
    uint nbar = 0;
    const uint total = a.off[a.n];
    const long long nb = a.bpos[a.n], nf = a.n - nb;
    const uint nbb = bound_blocks(nb, nb, nf, gridDim.x, a.split);
    const long long warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    PRec<Real>* Sf = (K & 1) ? S1 : S0;   // the free particles' final buffer
    double mz = 0.0;
    uint cnt = 0, flags = 0;
    if (blockIdx.x >= nbb) {   // free-only block
        const uint nfb = gridDim.x - nbb;
        free_sweep<Real>(a, S0, Sf, (warp * nfb + (blockIdx.x - nbb)) * 32 + lane, (long long)nfb * kWinThreads, nf, K,
                         mz, flags);
        block_observables(mz, cnt, flags, 1, part, a.words);
        clear_partials(part, gridDim.x, npart);
        return;
    }
    const bool deal_free = nbb == gridDim.x;
    const long long nthr = (long long)nbb * blockDim.x;
    const long long tid = (warp * nbb + blockIdx.x) * 32 + lane;
    // this thread's first bound particle: list data kept in registers
    uint b0 = 0, o00 = 0, o10 = 0, r00 = 0, r10 = 0;
    Real rb0 = (Real)0;
    if (tid < nb) {
        b0 = a.blist[tid];
        rb0 = a.R[b0];
        o00 = a.off[b0]; o10 = a.off[b0 + 1]; r00 = a.roff[b0]; r10 = a.roff[b0 + 1];
    }
    ParticleCommon pc = a.pc;
    for (int s = 0; s < K; s++) {
        PRec<Real>* Si = (s & 1) ? S1 : S0;
        PRec<Real>* So = (s & 1) ? S0 : S1;
        const Planes3<double> Hi = (s & 1) ? H1 : H0, Ho = (s & 1) ? H0 : H1;
        pc.first = s == 0 ? 1 : 0;
        for (long long t = tid; t < nb; t += nthr) {
            double mzi = 0.0;
            uint ci = 0;
            if (t == tid) {
                pp_item<Real, true>(b0, rb0, total, o00, o10, r00, r10, a.rk, a.lp, a.ln, a.cap, Si, So, a.Q, a.W, Hi,
                                    Ho, a.pp, a.pw, pc, a.dtr, a.inv_dt, a.density, mzi, ci, flags, nullptr, nullptr,
                                    nullptr);
            } else {
                const uint i = a.blist[t];
                pp_item<Real, true>(i, a.R[i], total, a.off[i], a.off[i + 1], a.roff[i], a.roff[i + 1], a.rk, a.lp,
                                    a.ln, a.cap, Si, So, a.Q, a.W, Hi, Ho, a.pp, a.pw, pc, a.dtr, a.inv_dt, a.density,
                                    mzi, ci, flags, nullptr, nullptr, nullptr);
            }
            if (s == K - 1) { mz = fmax(mz, mzi); cnt += ci; }
        }
        if (deal_free) {
            const long long f0 = nf * s / K, f1 = nf * (s + 1) / K;
            for (long long t = f0 + (nthr - 1 - tid); t < f1; t += nthr) {
                double mzi = 0.0;
                free_item<Real>(a, S0, Sf, a.flist[t], 0, K, K - 1, false, mzi, flags);
                mz = fmax(mz, mzi);
            }
        }
        if (s < K - 1) grid_barrier(bar, nbar++, nbb, a.words);
    }
    block_observables(mz, cnt, flags, 1, part, a.words);
    clear_partials(part, gridDim.x, npart);
}

// out[0]: the largest positive radius (its bits), out[2]: nonzero when a
// radius is not positive (or not a number).
__global__ void k_rmax(long long n, const double* __restrict__ rad, unsigned long long* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double r = i < n ? rad[i] : 0.0;
    if (__any_sync(0xffffffffu, i < n && !(r > 0.0)) && lane_id() == 0) atomicOr(out + 2, 1ull);
    unsigned long long b = (unsigned long long)__double_as_longlong(r > 0.0 ? r : 0.0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
        b = ob > b ? ob : b;
    }
    if (lane_id() == 0 && b) atomicMax(out, b);
}

// Sum of r^3 over the radii, one block in a fixed order (no atomics: the
// same bits on every run); launch with 1024 threads.
__global__ void __launch_bounds__(1024) k_vol(long long n, const double* __restrict__ rad, double* out) {
    __shared__ double sw[32];
    double v = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const double r = rad[i];
        v += r * r * r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane_id() == 0) sw[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sw[w];
        *out = t;
    }
}

__global__ void k_pairs_out(const uint* __restrict__ off, long long n, long long cap, const uint* __restrict__ lp,
                            const uint* __restrict__ ln, Planes3<double> H, uint* __restrict__ olp, uint* __restrict__ oln,
                            double* __restrict__ oh) {
    const uint total = off[n];
    if ((long long)total > cap) return;
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)total) return;
    olp[k] = lp[k];
    oln[k] = ln[k];
    oh[3 * k] = H.x[k]; oh[3 * k + 1] = H.y[k]; oh[3 * k + 2] = H.z[k];
}

}  // namespace dem

using namespace dem;

// ===================================================================== ctx

namespace {

void free_graphs(dem_ctx* c) {
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int h = 0; h < 2; h++)
                for (int t = 0; t < 2; t++)
                    if (c->gexec[a][b][h][t]) {
                        cudaGraphExecDestroy(c->gexec[a][b][h][t]);
                        c->gexec[a][b][h][t] = nullptr;
                    }
    adjoint_drop_graphs(c);
}

void free_cells(dem_ctx* c) {
    if (c->ccount) cudaFree(c->ccount);
    if (c->cstart) cudaFree(c->cstart);
    c->ccount = c->cstart = nullptr;
}

ParticleCommon particle_common(const dem_ctx* c, int slot) {
    ParticleCommon pc;
    pc.dt = c->cfg.dt;
    pc.hx = c->cfg.world[0] * 0.5;
    pc.hy = c->cfg.world[1] * 0.5;
    const float hs = (float)(0.5 * c->cfg.skin);
    pc.half_skin2 = hs * hs;
    pc.first = slot == 0 ? 1 : 0;
    pc.observe = slot == c->observe_slot ? 1 : 0;
    return pc;
}

// Per slot: fpart partials of the particle kernels (the bound-particle, batch
// and window kernels: fpart is at least each one's grid), then nblk of the
// free-particle kernel.  A kernel that writes a region clears the rest of it
// (or, when it steps every particle, the rest of the slot).
StepPartials partials(const dem_ctx* c, int slot) {
    return StepPartials{c->part_mz + (size_t)slot * c->npart, c->part_cnt + (size_t)slot * c->npart};
}
StepPartials free_partials(const dem_ctx* c, int slot) {
    return StepPartials{c->part_mz + (size_t)slot * c->npart + c->fpart,
                        c->part_cnt + (size_t)slot * c->npart + c->fpart};
}

// List build from the current state, carrying history from list buffer src
// (phase c->hph) into buffer 1-src (phase 0).
// The outer build on stream st (plain launches: in a graph it is the body of
// a conditional node): cells of the outer grid, their scan, the counting
// scatter, the row lengths, their scan, the rows.
template <typename Real> int outer_build(dem_ctx* c, const PRec<Real>* S, cudaStream_t st) {
    const long long n = c->n;
    const int B = 256;
    const GridC og = c->ogrid;
    k_cell_hash<Real><<<grid_for(n, B), B, 0, st>>>(n, S, og, c->key, c->ccount, c->arrival);
    DEM_LAUNCH_CHECK();
    int rc = exclusive_scan_u32(c->ccount, c->cstart, c->oncells, c->cstart + c->oncells, c->scan_tmp, st, false);
    if (rc) return rc;
    k_scatter<Real><<<grid_for(n, B), B, 0, st>>>(n, (const uint*)c->key, (const uint*)c->arrival,
                                                  (const uint*)c->cstart, c->ccount, S, (const Real*)c->rad, og,
                                                  c->sid, c->skeyu, (R4<Real>*)c->sposu, c->tpos);
    DEM_LAUNCH_CHECK();
    const Real oskin = (Real)c->oskin;
    k_outer_count<Real><<<grid_for(n, B), B, 0, st>>>(n, (const uint*)c->sid, (const R4<Real>*)c->sposu,
                                                      (const uint*)c->skeyu, (const uint*)c->cstart, og, oskin,
                                                      c->ocnt);
    DEM_LAUNCH_CHECK();
    if ((rc = exclusive_scan_u32(c->ocnt, c->coff, n, c->coff + n, c->scan_tmp, st, false))) return rc;
    k_outer_fill<Real><<<grid_for(n, B), B, 0, st>>>(n, (const uint*)c->sid, (const R4<Real>*)c->sposu,
                                                     (const uint*)c->skeyu, (const uint*)c->cstart, og, oskin,
                                                     (const uint*)c->coff, c->cln, c->ccap, S,
                                                     planes<double>(c->xo, c->npad), c->oflag, c->words);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

// In a capture: k_outer_check, then a conditional node whose body (captured
// on the context's build stream) is the outer build; the capture goes on
// after the node.
template <typename Real>
int launch_outer_check(dem_ctx* c, const PRec<Real>* S, cudaStream_t s, int cond, cudaGraphConditionalHandle h) {
    k_outer_check<Real><<<grid_for(c->n, 256), 256, 0, s>>>(
        c->n, S, (const Real*)c->rad, c->grid, c->cfg.world[0] * 0.5, c->cfg.world[1] * 0.5, 0.5 * c->cfg.skin,
        c->ikey, planes<double>(c->xo, c->npad), c->odelta2, (const uint*)c->oflag, c->wcount, cond, h);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

template <typename Real> int outer_build_conditional(dem_ctx* c, const PRec<Real>* S) {
    cudaStream_t s = c->stream;
    cudaStreamCaptureStatus st;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    DEM_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &nd));
    cudaGraphConditionalHandle h;
    DEM_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
    const int crc = launch_outer_check<Real>(c, S, s, 1, h);
    if (crc) return crc;
    DEM_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    DEM_CUDA_TRY(cudaGraphAddNode(&node, cg, deps, nd, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    DEM_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    DEM_CUDA_TRY(cudaStreamBeginCaptureToGraph(c->cstream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int rc = outer_build<Real>(c, S, c->cstream);
    cudaGraph_t got = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->cstream, &got);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (outer build)", __FILE__, __LINE__);
    return DEM_OK;
}

template <typename Real> int launch_free(dem_ctx* c, int lst, int slot0, int nsteps, cudaStream_t s, int batch = 0);

template <typename Real> int launch_relist(dem_ctx* c, int src) {
    const long long n = c->n;
    const int dst = 1 - src;
    const int B = 256;
    cudaStream_t s = c->stream;
    const PRec<Real>* S = (const PRec<Real>*)c->rec[c->sbuf];
    GridC g = c->grid;
    const bool cc = c->batching && c->mode == DEM_FORCE_PCCP && c->cc_parent;
    // every launch after the first is programmatic: each kernel waits for its
    // predecessor before it touches memory, so only the launch latency overlaps
    const bool pdl = c->pdl && !c->profiling;
    // the outer list: rebuilt when needed (a graph's conditional node, switched
    // by k_outer_check), always in an eager re-list
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    DEM_CUDA_TRY(cudaStreamIsCapturing(s, &cst));
    int rc;
    if (cst == cudaStreamCaptureStatusActive && c->outer_cond) {
        rc = outer_build_conditional<Real>(c, S);
    } else {
        rc = launch_outer_check<Real>(c, S, s, 0, cudaGraphConditionalHandle{});
        if (!rc) rc = outer_build<Real>(c, S, s);
    }
    if (rc) return rc;
    const Real skin = (Real)c->cfg.skin;
    // candidates, their counts' scans, bound and free lists: one pass
    k_filter_scan<Real><<<grid_for(n, kFilterTile), kFilterThreads, 0, s>>>(
        n, S, (const Real*)c->rad, g, skin, (const uint*)c->coff, (const uint*)c->cln, c->ccap, c->wslot, c->wlist,
        c->wcount, cc ? c->cc_parent : nullptr, c->cc_size, c->cc_base, c->npad, (const uint*)c->ikey, c->njli,
        c->bflag, c->scr,
        c->words, c->lb, c->off[dst], c->roff, c->bpos, c->blist, c->flist, cc ? c->cc_words : nullptr, c->cc_bw,
        (long long)c->nbatch_max + 2);
    DEM_LAUNCH_CHECK();
    // a batched window follows: its free particles need nothing of the
    // re-list after the free list, and the passes after the candidate pass
    // touch bound particles only, so they step the whole window from here,
    // beside the rest of the re-list (joined at the window's end); the fork
    // comes after the candidate pass (free_fork 1) or after the fill (2)
    auto fork_free = [&]() -> int {
        DEM_CUDA_TRY(cudaEventRecord(c->evfork, s));
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream2, c->evfork, 0));
        const int frc = launch_free<Real>(c, dst, 0, c->cfg.relist_interval, c->stream2, 1);
        if (frc) return frc;
        DEM_CUDA_TRY(cudaEventRecord(c->evjoin, c->stream2));
        return DEM_OK;
    };
    if (c->free_early && c->free_fork == 1 && (rc = fork_free())) return rc;
    const unsigned BG = c->bound_grid;
    DEM_CUDA_TRY(launch_ex(
        k_nbr_fill<Real>, BG, B, s, pdl, n, S, (const Real*)c->rad, g, skin, (const uint*)c->coff,
        (const uint*)c->cln, (const uint*)c->off[dst], (const uint*)c->roff,
        c->njli, c->ln[dst], c->lp, planes<double>(c->hist[dst][0], c->cap), (const uint*)c->off[src],
        (const uint*)c->ln[src], planes<double>(c->hist[src][c->hph], c->cap), c->rk, (R4<Real>*)c->pf, c->cap,
        c->words, c->carry, (const uint*)c->scr, cc ? c->cc_parent : nullptr, (const uint*)c->bpos,
        (const uint*)c->blist, (const uint*)c->cc_skip, c->lb, (long long)lb_words(c->npad)));
    if (c->free_early && c->free_fork == 2 && (rc = fork_free())) return rc;
    DEM_CUDA_TRY(launch_ex(k_rev_sort, BG, B, s, pdl, n, (const uint*)c->roff, c->rk, c->ru,
                           (const uint*)c->off[dst], c->cap, cc ? c->cc_parent : nullptr, (const uint*)c->bpos,
                           (const uint*)c->blist, c->cc_size, c->cc_pairs, (const uint*)c->cc_skip, c->cc_words));
    if (cc) {   // the window's components and batches (cluster-batched window path)
        const uint* off = c->off[dst];
        const long long nbb = c->nbatch_max + 2;
        DEM_CUDA_TRY(launch_ex(k_cc_pass, BG, kCcThreads, s, pdl, n, c->cap, c->nbatch_max, nbb, c->batch_grid,
                               BatchCap<Real>::P, BatchCap<Real>::Q, off, (const uint*)c->bpos,
                               (const uint*)c->blist, (const uint*)c->cc_parent, (const uint*)c->cc_size,
                               (const uint*)c->cc_pairs, c->cc_base, c->cc_fill, c->cc_order, c->cc_bw, c->cc_batch,
                               c->cc_words, c->cc_skip, c->lb + lb_cc(c->npad), c->words));
    }
    return DEM_OK;
}

// Step kernels after the first of a window may launch programmatically
// (overlapping their predecessor's tail); never while profiling or recording,
// where events or tape kernels sit between them.
bool step_pdl(const dem_ctx* c, int slot, bool first_of_step) {
    return c->pdl && !c->profiling && !c->record && (slot > 0 || !first_of_step);
}

template <typename Real> StepArgs<Real> step_args(const dem_ctx* c, int lst, int slot) {
    const long long np = c->npad;
    StepArgs<Real> a;
    a.n = c->n;
    a.cap = c->cap;
    a.off = c->off[lst]; a.lp = c->lp; a.ln = c->ln[lst]; a.ru = c->ru; a.roff = c->roff; a.rk = c->rk;
    a.wlist = c->wlist; a.wcount = c->wcount; a.wslot = c->wslot;
    a.bpos = c->bpos; a.blist = c->blist; a.flist = c->flist;
    a.S = (PRec<Real>*)c->rec[0];
    a.W = planes<double>(c->wh, np);
    a.H = planes<double>(c->hist[lst][0], c->cap);
    a.R = (const Real*)c->rad;
    a.Q = c->q;
    a.pf = (R4<Real>*)c->pf; a.pti = (R4<Real>*)c->pti; a.rfj = (R4<Real>*)c->rfj; a.rtj = (R4<Real>*)c->rtj;
    a.wf = (R4<Real>*)c->wf;
    a.pp = make_law<Real>(c->mat.pp);
    a.pw = make_law<Real>(c->mat.pw);
    a.pc = particle_common(c, slot);
    a.dtr = (Real)c->cfg.dt;
    a.inv_dt = (Real)(1.0 / c->cfg.dt);
    a.density = (Real)c->cfg.density;
    a.split = c->win_split;
    a.batch = 0;
    a.ccw = c->cc_words;
    a.words = c->words;
    a.dbgF = c->record ? c->dbgF : nullptr;
    a.dbgT = c->record ? c->dbgT : nullptr;
    a.dbgC = c->record ? c->dbgC : nullptr;
    a.tx = a.td = a.twh = a.tF = a.tT = a.th = nullptr;
    a.tc = nullptr;
    a.ta = nullptr;
    a.tnp = np;
    a.tstep0 = 0;
    return a;
}

template <typename Real> int launch_pair(dem_ctx* c, int lst, int slot) {
    DEM_CUDA_TRY(launch_ex(k_pair<Real>, c->pair_grid, 256, c->stream, step_pdl(c, slot, true),
                           step_args<Real>(c, lst, slot)));
    return DEM_OK;
}

template <typename Real> int launch_particle(dem_ctx* c, int lst, int slot) {
    DEM_CUDA_TRY(launch_ex(k_particle<Real>, grid_for(c->n, 256), 256, c->stream, step_pdl(c, slot, false),
                           step_args<Real>(c, lst, slot), partials(c, slot), (size_t)c->fpart));
    return DEM_OK;
}

// Free particles, window slots slot0 .. slot0+nsteps-1, on stream s.
template <typename Real> int launch_free(dem_ctx* c, int lst, int slot0, int nsteps, cudaStream_t s, int batch) {
    const int obs = c->observe_slot;
    const int os = (obs >= slot0 && obs < slot0 + nsteps) ? obs : slot0;
    StepArgs<Real> a = step_args<Real>(c, lst, slot0);
    a.batch = batch;
    if (nsteps != 1) a.dbgF = a.dbgT = nullptr, a.dbgC = nullptr;
    const unsigned g = grid_for(c->n, 256);
    k_free_run<Real><<<g, 256, 0, s>>>(a, slot0, nsteps, obs, free_partials(c, os), (size_t)g, (size_t)c->nblk);
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

// The window kernel's instance: one block per SM (up to 128 registers), or
// two (64 registers, with spills).
template <typename Real> auto window_fn(int minb) { return minb == 2 ? k_window<Real, 2> : k_window<Real, 1>; }

// The window kernel: all K steps of the window in one cooperative launch.
template <typename Real> int launch_window(dem_ctx* c, int lst, const WindowTape* tape, int batch = 0) {
    const int K = c->cfg.relist_interval;
    DEM_CUDA_TRY(cudaMemsetAsync(c->bar, 0, kBarWords * sizeof(uint), c->stream));   // counter, give-up word
    StepArgs<Real> a = step_args<Real>(c, lst, 0);
    a.batch = batch;
    a.dbgF = a.dbgT = nullptr;
    a.dbgC = nullptr;
    if (tape) {
        a.tx = tape->tx; a.td = tape->td; a.twh = tape->twh; a.tF = tape->tF; a.tT = tape->tT; a.th = tape->th;
        a.tc = tape->tc;
        a.ta = (Real*)tape->ta;
        a.tstep0 = tape->step0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->win_grid);
    cfg.blockDim = dim3(kWinThreads);
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    // a batched window's kernel leaves the free particles' partials to k_free_run
    DEM_CUDA_TRY(cudaLaunchKernelEx(&cfg, window_fn<Real>(c->win_minb), a, K, partials(c, K - 1),
                                    batch ? (size_t)c->fpart : c->npart, c->bar));
    return DEM_OK;
}

// PP window kernel: state buffer sb and history phase hp at the window start.
template <typename Real> int launch_window_pp(dem_ctx* c, int lst, int sb, int hp) {
    const int K = c->cfg.relist_interval;
    DEM_CUDA_TRY(cudaMemsetAsync(c->bar, 0, kBarWords * sizeof(uint), c->stream));   // counter, give-up word
    StepArgs<Real> a = step_args<Real>(c, lst, 0);
    a.dbgF = a.dbgT = nullptr;
    a.dbgC = nullptr;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->win_grid);
    cfg.blockDim = dim3(kWinThreads);
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    DEM_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_window_pp<Real>, a, (PRec<Real>*)c->rec[sb], (PRec<Real>*)c->rec[1 - sb],
                                    planes<double>(c->hist[lst][hp], c->cap),
                                    planes<double>(c->hist[lst][1 - hp], c->cap), K, partials(c, K - 1), c->npart,
                                    c->bar));
    return DEM_OK;
}

// The cluster-batched window: the grid-barrier window kernel (it steps the
// window only when a component or batch is too large for a block), then the
// free particles (forked stream) beside the batches, joined.
template <typename Real> int launch_batched_window(dem_ctx* c, int lst, const WindowTape* tape) {
    const int K = c->cfg.relist_interval;
    int rc = launch_window<Real>(c, lst, tape, 1);
    if (rc) return rc;
    if (!c->free_early) DEM_CUDA_TRY(cudaEventRecord(c->evfork, c->stream));
    StepArgs<Real> a = step_args<Real>(c, lst, 0);
    a.batch = 1;
    a.dbgF = a.dbgT = nullptr;
    a.dbgC = nullptr;
    if (tape) {
        a.tx = tape->tx; a.td = tape->td; a.twh = tape->twh; a.tF = tape->tF; a.tT = tape->tT; a.th = tape->th;
        a.tc = tape->tc;
        a.ta = (Real*)tape->ta;
        a.tstep0 = tape->step0;
    }
    // the batches first and at the higher priority: their blocks (one per SM)
    // take their SMs before the free particles' blocks fill the room beside them
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c->batch_grid);
        cfg.blockDim = dim3(kBatchThreads);
        cfg.dynamicSmemBytes = c->batch_smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributePriority;
        at[0].val.priority = c->prio_hi;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        DEM_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch<Real>, a, K, (const uint*)c->cc_order,
                                        (const uint*)c->cc_batch, c->cc_loc, partials(c, K - 1), (size_t)c->fpart));
    }
    if (!c->free_early) {   // else forked by the re-list, right after the candidate pass
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream2, c->evfork, 0));
        rc = launch_free<Real>(c, lst, 0, K, c->stream2, 1);
        if (rc) return rc;
        DEM_CUDA_TRY(cudaEventRecord(c->evjoin, c->stream2));
    }
    DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->evjoin, 0));
    return DEM_OK;
}


// PP step: reads state buffer sbuf and history phase hph, writes the others.
template <typename Real> int launch_pp(dem_ctx* c, int lst, int slot, int sb, int hp) {
    const long long n = c->n, np = c->npad;
    LawParams<Real> pp = make_law<Real>(c->mat.pp), pw = make_law<Real>(c->mat.pw);
    const double dt = c->cfg.dt;
    DEM_CUDA_TRY(launch_ex(
        k_step_pp<Real>, grid_for(n, 256), 256, c->stream, step_pdl(c, slot, true), n, (const uint*)c->off[lst],
        (const uint*)c->roff, (const uint*)c->rk, (const uint*)c->lp, (const uint*)c->ln[lst], c->cap,
        (const PRec<Real>*)c->rec[sb], (PRec<Real>*)c->rec[1 - sb], (const Real*)c->rad, c->q,
        planes<double>(c->wh, np), planes<double>(c->hist[lst][hp], c->cap),
        planes<double>(c->hist[lst][1 - hp], c->cap), pp, pw, particle_common(c, slot), (Real)dt, (Real)(1.0 / dt),
        (Real)c->cfg.density, partials(c, slot), c->words, c->record ? c->dbgF : nullptr,
        c->record ? c->dbgT : nullptr, c->record ? c->dbgC : nullptr, (size_t)grid_for(n, 256), c->npart));
    return DEM_OK;
}

}  // namespace

namespace dem {
bool use_batches(const dem_ctx* c) { return c->batching && c->mode == DEM_FORCE_PCCP && c->cc_parent != nullptr; }

int window_kernel(dem_ctx* c, int lst, const WindowTape* tape) {
    NvtxRange r("dem window kernel");
    if (use_batches(c))
        return c->prec == DEM_PREC_MIXED ? launch_batched_window<float>(c, lst, tape)
                                         : launch_batched_window<double>(c, lst, tape);
    return c->prec == DEM_PREC_MIXED ? launch_window<float>(c, lst, tape) : launch_window<double>(c, lst, tape);
}

int relist(dem_ctx* c, int src) {
    NvtxRange r("dem re-list");
    return c->prec == DEM_PREC_MIXED ? launch_relist<float>(c, src) : launch_relist<double>(c, src);
}

// One DEM step on list buffer lst (window slot `slot`): PCCP = pair kernel +
// particle kernel; PP = one kernel.  Advances the ping-pong indices.
int step_kernels(dem_ctx* c, int lst, int slot, double* ms_pair, double* ms_part) {
    int rc;
    const bool mixed = c->prec == DEM_PREC_MIXED;
    if (c->profiling) DEM_CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
    const bool wt = c->wtiming_capture;
    if (c->mode == DEM_FORCE_PP) {
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[2 + 2 * slot], c->stream, cudaEventRecordExternal));
        rc = mixed ? launch_pp<float>(c, lst, slot, c->sbuf, c->hph) : launch_pp<double>(c, lst, slot, c->sbuf, c->hph);
        if (rc) return rc;
        if (c->profiling) DEM_CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
        c->sbuf ^= 1;
        c->hph ^= 1;
    } else {
        rc = mixed ? launch_pair<float>(c, lst, slot) : launch_pair<double>(c, lst, slot);
        if (rc) return rc;
        if (c->profiling) DEM_CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[2 + 2 * slot], c->stream, cudaEventRecordExternal));
        rc = mixed ? launch_particle<float>(c, lst, slot) : launch_particle<double>(c, lst, slot);
        if (rc) return rc;
        if (!c->free_in_window) {   // eager step: the free particles' one step, same stream
            rc = mixed ? launch_free<float>(c, lst, slot, 1, c->stream) : launch_free<double>(c, lst, slot, 1, c->stream);
            if (rc) return rc;
        }
    }
    if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[3 + 2 * slot], c->stream, cudaEventRecordExternal));
    if (c->profiling) {
        DEM_CUDA_TRY(cudaEventRecord(c->ev[2], c->stream));
        float a = 0.f, b = 0.f;
        DEM_CUDA_TRY(cudaEventSynchronize(c->ev[2]));
        DEM_CUDA_TRY(cudaEventElapsedTime(&a, c->ev[0], c->ev[1]));
        DEM_CUDA_TRY(cudaEventElapsedTime(&b, c->ev[1], c->ev[2]));
        if (c->mode == DEM_FORCE_PP) { *ms_pair = 0.0; *ms_part = a; }
        else { *ms_pair = a; *ms_part = b; }
    }
    return DEM_OK;
}

}  // namespace dem

namespace {
// Enqueue one full window (re-list from list `src`, then K steps).
int enqueue_window(dem_ctx* c, int src) {
    const int K = c->cfg.relist_interval;
    const bool wt = c->wtiming_capture;
    if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[0], c->stream, cudaEventRecordExternal));
    // a batched window: the free particles start inside the re-list
    c->free_early = c->free_fork > 0 && c->mode == DEM_FORCE_PCCP && !c->record && c->win_kernel && use_batches(c);
    c->observe_slot = K - 1;
    int rc = relist(c, src);
    if (rc) { c->free_early = false; return rc; }
    if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[1], c->stream, cudaEventRecordExternal));
    c->hph = 0;
    const int lst = 1 - src;
    const bool mixed = c->prec == DEM_PREC_MIXED;
    if (c->mode == DEM_FORCE_PCCP && !c->record && c->win_kernel) {
        // every step of the window in one cooperative launch, or the cluster
        // batches beside the free particles
        rc = window_kernel(c, lst, nullptr);
        c->free_early = false;
        if (rc) return rc;
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[2], c->stream, cudaEventRecordExternal));
        c->wtiming_path = 1;
        return DEM_OK;
    }
    c->free_early = false;
    if (c->mode == DEM_FORCE_PP && !c->record && c->win_kernel) {
        // PP: every step of the window in one cooperative launch
        rc = mixed ? launch_window_pp<float>(c, lst, c->sbuf, c->hph)
                   : launch_window_pp<double>(c, lst, c->sbuf, c->hph);
        if (rc) return rc;
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[2], c->stream, cudaEventRecordExternal));
        c->wtiming_path = 1;
        return DEM_OK;
    }
    // per-step kernels.  PCCP: the free particles' whole window is one kernel
    // on a forked branch, concurrent with the bound chain (pair + particle per
    // step); the two touch disjoint particles and join before the next
    // re-list.  While forces are recorded every step, the free particles step
    // with the bound ones instead.
    const bool fork = c->mode == DEM_FORCE_PCCP && !c->record;
    if (fork) {
        DEM_CUDA_TRY(cudaEventRecord(c->evfork, c->stream));
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream2, c->evfork, 0));
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[2 + 2 * K], c->stream2, cudaEventRecordExternal));
        rc = mixed ? launch_free<float>(c, lst, 0, K, c->stream2) : launch_free<double>(c, lst, 0, K, c->stream2);
        if (rc) return rc;
        if (wt) DEM_CUDA_TRY(cudaEventRecordWithFlags(c->wev[3 + 2 * K], c->stream2, cudaEventRecordExternal));
        DEM_CUDA_TRY(cudaEventRecord(c->evjoin, c->stream2));
        c->free_in_window = true;
    }
    double a, b;
    for (int s = 0; s < K; s++) {
        rc = step_kernels(c, lst, s, &a, &b);
        if (rc) { c->free_in_window = false; return rc; }
    }
    c->free_in_window = false;
    if (fork) DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->evjoin, 0));
    c->wtiming_path = fork ? 2 : 0;
    return DEM_OK;
}

// Capture (once) and launch the window graph for the current buffers.
int launch_window_graph(dem_ctx* c) {
    NvtxRange r("dem window graph");
    const int src = c->cur, sb = c->sbuf, hp = c->hph;
    const int tm = c->wtiming ? 1 : 0;
    cudaGraphExec_t& ge = c->gexec[src][sb][hp][tm];
    if (!ge) {
        cudaGraph_t g = nullptr;
        DEM_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->wtiming_capture = tm != 0;
        int rc = enqueue_window(c, src);
        c->wtiming_capture = false;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        // capture only records: restore the indices, the launch below advances them
        c->sbuf = sb;
        c->hph = hp;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
    DEM_CUDA_TRY(cudaGraphLaunch(ge, c->stream));
    if (tm) c->wtiming_ran = true;
    const int K = c->cfg.relist_interval;
    c->hph = 0;
    if (c->mode == DEM_FORCE_PP) {
        c->sbuf = (sb + K) & 1;
        c->hph = K & 1;
    }
    return DEM_OK;
}

// Poured packing: is a layer due before the step with index s (0-based; the
// reference's it = s + 1 and time = dt*it, dempacking.cu:375-381)?  The
// threshold is the reference's (float)N*tnewpar/float(nplayer).
bool pour_due(const dem_ctx* c, long long s) {
    if (!c->pouring || c->n >= c->ntot) return false;
    const double time = c->cfg.dt * (double)(s + 1);
    return time > (double)(float)c->n * c->pour_tnewpar / (double)(float)c->pour_nplayer;
}

// The next layer joins (dempacking.cu:459-461): nplayer more particles (the
// rest at the end), and the step re-lists.
int pour_insert(dem_ctx* c) {
    const long long nold = c->n, nnew = std::min(nold + c->pour_nplayer, c->ntot);
    const unsigned g = grid_for(nnew - nold, 256);
    const Planes3<double> W = planes<double>(c->wh, c->npad);
    if (c->prec == DEM_PREC_MIXED)
        k_pour_activate<float><<<g, 256, 0, c->stream>>>(nold, nnew, (const PRec<float>*)c->pour_rec,
                                                         (PRec<float>*)c->rec[c->sbuf], c->q, W, c->off[c->cur]);
    else
        k_pour_activate<double><<<g, 256, 0, c->stream>>>(nold, nnew, (const PRec<double>*)c->pour_rec,
                                                          (PRec<double>*)c->rec[c->sbuf], c->q, W, c->off[c->cur]);
    DEM_LAUNCH_CHECK();
    c->n = nnew;
    c->vol = 4.0 / 3.0 * M_PI * c->r3sum[nnew];
    c->in_window = 0;   // this step re-lists (m_hiall = 1)
    free_graphs(c);     // the particle count is part of every captured launch
    // the new particles have no outer rows yet
    DEM_CUDA_TRY(cudaMemsetAsync(c->oflag, 0x01, sizeof(uint), c->stream));
    return DEM_OK;
}

size_t real_size(int prec) { return prec == DEM_PREC_MIXED ? sizeof(float) : sizeof(double); }

}  // namespace

namespace dem {
int host_perm(dem_ctx* c) {
    if (!c->hperm_stale) return DEM_OK;
    const long long n = c->ntot;
    c->hperm.resize(n);
    DEM_CUDA_TRY(cudaMemcpyAsync(c->hperm.data(), c->perm, n * sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->hperm_stale = false;
    return DEM_OK;
}
}  // namespace dem

extern "C" {

int dem_create(const dem_config* cfg, dem_ctx** out) {
    if (!cfg || !out) return fail(DEM_ERR_ARG, "dem_create: null argument");
    *out = nullptr;
    if (cfg->n <= 0 || cfg->n > 0x7fffffffLL) return fail(DEM_ERR_ARG, "dem_create: n out of range (%lld)", cfg->n);
    if (cfg->precision != DEM_PREC_FP64 && cfg->precision != DEM_PREC_MIXED)
        return fail(DEM_ERR_ARG, "dem_create: unknown precision %d", cfg->precision);
    if (cfg->force_mode != DEM_FORCE_PCCP && cfg->force_mode != DEM_FORCE_PP)
        return fail(DEM_ERR_ARG, "dem_create: unknown force mode %d", cfg->force_mode);
    if (cfg->relist_interval <= 0 || cfg->relist_interval > 100000)
        return fail(DEM_ERR_ARG, "dem_create: relist_interval must be in [1, 100000]");
    if (!(cfg->dt > 0.0) || !(cfg->skin > 0.0) || !(cfg->density > 0.0))
        return fail(DEM_ERR_ARG, "dem_create: dt, skin and density must be > 0");
    for (int a = 0; a < 3; a++)
        if (!(cfg->world[a] > 0.0)) return fail(DEM_ERR_ARG, "dem_create: world sizes must be > 0");
    dem_ctx* c = new dem_ctx();
    c->cfg = *cfg;
    c->prec = cfg->precision;
    c->mode = cfg->force_mode;
    c->n = cfg->n;
    c->ntot = cfg->n;
    c->npad = (cfg->n + 63) / 64 * 64;
    c->cap = cfg->pair_capacity > 0 ? cfg->pair_capacity : 8 * cfg->n;
    if (c->cap > 0x7fffffffLL) c->cap = 0x7fffffffLL;
    int rc = DEM_OK;
    auto bail = [&](int code) { dem_destroy(c); return code; };
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__));
    // The context's stream first: every initialising memset below is queued on
    // it and complete before dem_create returns.  (A plain cudaMemset would go
    // to the legacy stream, which the context's non-blocking streams do not
    // wait for: on a GPU busy with other streams' kernels it could land after
    // the context's first upload or state load.)
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__));
    c->stream = c->own_stream;
    const cudaStream_t s0 = c->own_stream;
    const long long n = c->n, np = c->npad, cap = c->cap;
    const size_t rs = real_size(c->prec);
    const int nstate = c->mode == DEM_FORCE_PP ? 2 : 1;
    const size_t recb = c->prec == DEM_PREC_MIXED ? sizeof(PRec<float>) : sizeof(PRec<double>);
    for (int b = 0; b < nstate; b++) {
        e = cudaMalloc(&c->rec[b], np * recb);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->rec[b], 0, np * recb, s0);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc (state)", __FILE__, __LINE__));
    }
    for (int l = 0; l < 2; l++)
        for (int h = 0; h < nstate; h++)
            if ((rc = dalloc(&c->hist[l][h], 3 * cap))) return bail(rc);
    if ((rc = dalloc(&c->wh, 3 * np)) || (rc = dalloc(&c->q, np)) || (rc = dalloc(&c->staging, 10 * np)) ||
        (rc = dalloc(&c->key, np)) || (rc = dalloc(&c->sid, np)) ||
        (rc = dalloc(&c->skeyu, np)) || (rc = dalloc(&c->njgi, np)) ||
        (rc = dalloc(&c->njli, np)) || (rc = dalloc(&c->off[0], np + 1)) || (rc = dalloc(&c->off[1], np + 1)) ||
        (rc = dalloc(&c->roff, np + 1)) || (rc = dalloc(&c->ln[0], cap)) || (rc = dalloc(&c->ln[1], cap)) ||
        (rc = dalloc(&c->lp, cap)) || (rc = dalloc(&c->rk, cap)) || (rc = dalloc(&c->ru, cap)) || (rc = dalloc(&c->words, 1)) ||
        (rc = dalloc(&c->rmax_bits, 3)) || (rc = dalloc(&c->wslot, np)) || (rc = dalloc(&c->wlist, np)) ||
        (rc = dalloc(&c->wcount, 1)) || (rc = dalloc(&c->arrival, np)) || (rc = dalloc(&c->scr, np * kScr)) ||
        (rc = dalloc(&c->bflag, np)) || (rc = dalloc(&c->bpos, np + 1)) || (rc = dalloc(&c->blist, np)) ||
        (rc = dalloc(&c->flist, np)) || (rc = dalloc(&c->bar, kBarWords)) || (rc = dalloc(&c->tpos, np)))
        return bail(rc);
    // the outer candidate list (rows in both directions; its skin is set
    // with the grid, from r_max): four times the pair capacity
    c->ccap = std::min<long long>(4 * cap, 0x7fffffffLL);
    if ((rc = dalloc(&c->coff, np + 1)) || (rc = dalloc(&c->cln, c->ccap)) || (rc = dalloc(&c->ocnt, np)) ||
        (rc = dalloc(&c->xo, 3 * np)) || (rc = dalloc(&c->oflag, 2)) || (rc = dalloc(&c->ikey, np)) ||
        (rc = dalloc(&c->lb, lb_words(np))))
        return bail(rc);
    e = cudaMemsetAsync(c->oflag, 0x01, sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->lb, 0, lb_words(np) * sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->coff, 0, (np + 1) * sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(e, "outer list set-up", __FILE__, __LINE__));
    e = cudaMalloc(&c->wf, 2 * np * 4 * rs);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc (wall forces)", __FILE__, __LINE__));
    e = cudaMalloc(&c->rad, np * rs);
    if (e == cudaSuccess) e = cudaMalloc(&c->sposu, np * 4 * rs);
    if (e == cudaSuccess) e = cudaMalloc(&c->pf, cap * 4 * rs);
    if (e == cudaSuccess && c->mode == DEM_FORCE_PCCP) e = cudaMalloc(&c->pti, cap * 4 * rs);
    if (e == cudaSuccess && c->mode == DEM_FORCE_PCCP) e = cudaMalloc(&c->rfj, cap * 4 * rs);
    if (e == cudaSuccess && c->mode == DEM_FORCE_PCCP) e = cudaMalloc(&c->rtj, cap * 4 * rs);
    if (e == cudaSuccess) e = cudaMallocHost(&c->host_pinned, 4096);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc (engine buffers)", __FILE__, __LINE__));
    c->nblk = grid_for(n, 256);
    {   // one resident wave of the pair kernel (grid-stride over its items)
        int nsm = 0, per = 0;
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
        if (e == cudaSuccess)
            e = c->prec == DEM_PREC_MIXED ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair<float>, 256, 0)
                                          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair<double>, 256, 0);
        if (e != cudaSuccess) return bail(cuda_fail(e, "pair kernel occupancy", __FILE__, __LINE__));
        c->pair_grid = (unsigned)std::max(1, nsm * std::max(per, 1));
        int wper = 0;   // the window kernel: every block co-resident (cooperative launch)
        const bool mx = c->prec == DEM_PREC_MIXED;
        if (c->mode == DEM_FORCE_PP)
            e = mx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wper, k_window_pp<float>, kWinThreads, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wper, k_window_pp<double>, kWinThreads, 0);
        else {
            // window-kernel blocks per SM: two in the mixed form (64 registers;
            // the settled 500,000-sphere bed 7.5 % faster), one in FP64 (its
            // spills at 64 made it 5 % slower); DEM_B200_WINDOW_MINB=1|2 overrides
            const char* wm = getenv("DEM_B200_WINDOW_MINB");
            c->win_minb = (wm && (wm[0] == '1' || wm[0] == '2')) ? wm[0] - '0' : (mx ? 2 : 1);
            e = mx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wper, window_fn<float>(c->win_minb), kWinThreads, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wper, window_fn<double>(c->win_minb), kWinThreads,
                                                                   0);
        }
        if (e != cudaSuccess) return bail(cuda_fail(e, "window kernel occupancy", __FILE__, __LINE__));
        int coop = 0;
        e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaDeviceGetAttribute", __FILE__, __LINE__));
        c->win_grid = (unsigned)std::max(1, nsm * wper);
        const char* wk = getenv("DEM_B200_WINDOW");   // "0": per-step kernels for whole windows too
        c->win_kernel = coop && wper > 0 && !(wk && wk[0] == '0');
        // the re-list passes over the bound particles (fill, reverse rows,
        // components) stride over a grid of 4 blocks per SM: one pass covers
        // 150K bound particles, the ~10 % bound of a 500K free-flight bed
        c->bound_grid = (unsigned)std::max(1, 4 * nsm);
        // "0": the outer build in every re-list, no conditional node (a profiler
        // does not see the kernel nodes of a graph that has conditional nodes)
        const char* oc = getenv("DEM_B200_OUTER_COND");
        c->outer_cond = !(oc && oc[0] == '0');
        const char* pdl = getenv("DEM_B200_PDL");   // "0": plain launches everywhere
        c->pdl = !(pdl && pdl[0] == '0');
        // where a batched window's free particles start: "0" in the window,
        // "1" (default) after the re-list's candidate pass, "2" after its fill
        const char* ff = getenv("DEM_B200_FREE_FORK");
        c->free_fork = (ff && (ff[0] == '0' || ff[0] == '2')) ? ff[0] - '0' : 1;
        const char* ro = getenv("DEM_B200_REORDER");   // "0": keep the caller's particle order
        c->reorder = !(ro && ro[0] == '0');
        const char* sp = getenv("DEM_B200_SPLIT");   // window kernels' bound items per thread (0: no split)
        if (sp && sp[0]) c->win_split = atoi(sp);
        const char* bt = getenv("DEM_B200_BATCH");   // "0": no cluster batches (grid-barrier window kernel)
        c->batching = c->mode == DEM_FORCE_PCCP && c->win_kernel && !(bt && bt[0] == '0');
        if (c->batching) {
            const bool mx = c->prec == DEM_PREC_MIXED;
            c->batch_smem = mx ? batch_smem_layout<float>(nullptr, nullptr) : batch_smem_layout<double>(nullptr, nullptr);
            e = mx ? cudaFuncSetAttribute(k_batch<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->batch_smem)
                   : cudaFuncSetAttribute(k_batch<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)c->batch_smem);
            int bper = 0;
            if (e == cudaSuccess)
                e = mx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bper, k_batch<float>, kBatchThreads, c->batch_smem)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bper, k_batch<double>, kBatchThreads,
                                                                       c->batch_smem);
            if (e != cudaSuccess) return bail(cuda_fail(e, "batch kernel set-up", __FILE__, __LINE__));
            c->batching = bper > 0;
            c->batch_grid = (unsigned)std::max<long long>(1, std::min<long long>((long long)nsm * bper, grid_for(n, 256)));
            c->nbatch_max = (np + kBatchMin - 1) / kBatchMin + 1;
        }
    }
    // partials per slot: the particle kernels' (at least as many as the
    // window kernel has blocks), then the free kernel's
    c->fpart = std::max<size_t>((size_t)c->nblk, c->win_grid);
    c->npart = c->fpart + c->nblk;
    if ((rc = dalloc(&c->part_mz, (size_t)cfg->relist_interval * c->npart)) ||
        (rc = dalloc(&c->part_cnt, (size_t)cfg->relist_interval * c->npart)))
        return bail(rc);
    e = cudaMemsetAsync(c->part_mz, 0, (size_t)cfg->relist_interval * c->npart * sizeof(unsigned long long), s0);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(c->part_cnt, 0, (size_t)cfg->relist_interval * c->npart * sizeof(uint), s0);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset (partials)", __FILE__, __LINE__));
    if (c->batching) {
        if ((rc = dalloc(&c->cc_parent, np)) || (rc = dalloc(&c->cc_size, 3 * np)) || (rc = dalloc(&c->cc_base, np)) ||
            (rc = dalloc(&c->cc_order, np)) || (rc = dalloc(&c->cc_batch, c->nbatch_max + 2)) ||
            (rc = dalloc(&c->cc_loc, np)) || (rc = dalloc(&c->cc_words, 4)) || (rc = dalloc(&c->cc_skip, 2)) ||
            (rc = dalloc(&c->cc_bw, 3 * (c->nbatch_max + 2))))
            return bail(rc);
        c->cc_pairs = c->cc_size + np;
        c->cc_fill = c->cc_size + 2 * np;
        e = cudaMemsetAsync(c->cc_words, 0, 4 * sizeof(uint), s0);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->cc_skip, 0, 2 * sizeof(uint), s0);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset (batch words)", __FILE__, __LINE__));
    }
    c->scan_words = 3 * scan_scratch_words(std::max<long long>(np + 1, 1));
    if ((rc = dalloc(&c->scan_tmp, c->scan_words))) return bail(rc);
    e = cudaMemsetAsync(c->words, 0, sizeof(EngineWords), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->bar, 0, kBarWords * sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->off[0], 0, (np + 1) * sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->off[1], 0, (np + 1) * sizeof(uint), s0);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->roff, 0, (np + 1) * sizeof(uint), s0);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMemset (engine init)", __FILE__, __LINE__));
    for (int k = 0; k < 4; k++) {
        e = cudaEventCreate(&c->ev[k]);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaEventCreate", __FILE__, __LINE__));
    }
    e = cudaEventCreateWithFlags(&c->ext_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->h2d_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_rad, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        int lo = 0, hi = 0;
        e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
        c->prio_hi = hi;
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evfork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evjoin, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__));
    e = cudaStreamSynchronize(s0);   // the initialisation above is done
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamSynchronize", __FILE__, __LINE__));
    *out = c;
    return DEM_OK;
}

int dem_destroy(dem_ctx* c) {
    if (!c) return DEM_OK;
    cudaStreamSynchronize(c->stream);
    dem_adjoint_release(c);
    free_graphs(c);
    free_cells(c);
    void* ptrs[] = {c->rec[0], c->rec[1], c->rad, c->q, c->wh,
                    c->staging, c->key, c->sid, c->skeyu, c->sposu, c->njgi, c->njli, c->coff, c->cln, c->ocnt,
                    c->xo, c->oflag, c->ikey, c->lb,
                    c->off[0], c->off[1], c->roff, c->ln[0], c->ln[1], c->lp, c->hist[0][0], c->hist[0][1],
                    c->hist[1][0], c->hist[1][1], c->rk, c->ru, c->pf, c->pti, c->rfj, c->rtj, c->scan_tmp, c->words, c->part_mz,
                    c->part_cnt, c->rmax_bits, c->dbgF, c->dbgT, c->dbgC, c->wslot, c->wlist, c->wcount, c->wf, c->arrival,
                    c->scr, c->bflag, c->bpos, c->blist, c->flist, c->bar,
                    c->tpos, c->pour_rec, c->perm, c->cc_parent, c->cc_size, c->cc_base, c->cc_order,
                    c->cc_batch, c->cc_loc, c->cc_words, c->cc_bw, c->cc_skip};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->host_pinned) cudaFreeHost(c->host_pinned);
    for (int k = 0; k < 4; k++)
        if (c->ev[k]) cudaEventDestroy(c->ev[k]);
    if (c->ext_ready) cudaEventDestroy(c->ext_ready);
    if (c->h2d_done) cudaEventDestroy(c->h2d_done);
    if (c->ev_up) cudaEventDestroy(c->ev_up);
    if (c->ev_rad) cudaEventDestroy(c->ev_rad);
    if (c->evfork) cudaEventDestroy(c->evfork);
    if (c->evjoin) cudaEventDestroy(c->evjoin);
    for (cudaEvent_t e : c->wev) cudaEventDestroy(e);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->cstream) cudaStreamDestroy(c->cstream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return DEM_OK;
}

int dem_set_stream(dem_ctx* c, void* s) {
    if (!c) return fail(DEM_ERR_ARG, "dem_set_stream: null ctx");
    cudaStream_t ns = s ? (cudaStream_t)s : c->own_stream;
    if (ns != c->stream) {
        DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        free_graphs(c);
    }
    c->stream = ns;
    return DEM_OK;
}

int dem_set_material(dem_ctx* c, const dem_material* m) {
    if (!c || !m) return fail(DEM_ERR_ARG, "dem_set_material: null argument");
    const dem_contact* cs[2] = {&m->pp, &m->pw};
    for (const dem_contact* k : cs) {
        if (!(k->estar > 0.0) || k->mu < 0.0 || !(k->nu < 1.0) || k->damp_n < 0.0 || k->damp_t < 0.0 ||
            k->roll < 0.0 || k->roll_rel < 0.0)
            return fail(DEM_ERR_ARG, "dem_set_material: out-of-range contact parameter");
    }
    c->mat = *m;
    c->have_mat = true;
    free_graphs(c);   // parameters are baked into captured kernels
    return DEM_OK;
}

static int setup_grid(dem_ctx* c) {
    const double cs = c->cfg.cell > 0.0 ? c->cfg.cell : 2.0 * c->rmax + c->cfg.skin + 1e-4;
    if (!(cs >= 2.0 * c->rmax + c->cfg.skin))
        return fail(DEM_ERR_ARG, "cell %.6g smaller than 2*r_max+skin = %.6g", cs, 2.0 * c->rmax + c->cfg.skin);
    GridC g;
    g.ox = -c->cfg.world[0] * 0.5;
    g.oy = -c->cfg.world[1] * 0.5;
    g.oz = 0.0;
    g.cs = cs;
    g.gx = (int)(c->cfg.world[0] / cs) + 1;
    g.gy = (int)(c->cfg.world[1] / cs) + 1;
    g.gz = (int)(c->cfg.world[2] / cs) + 1;
    const long long nc = (long long)g.gx * g.gy * g.gz;
    if (nc > 0x7fffffffLL) return fail(DEM_ERR_ARG, "grid of %lld cells too large", nc);
    // the outer list: skin + ext, ext = min(skin, r_max / 10), kept while no
    // particle has moved 0.4 ext; its grid: cells of at least 2 r_max + oskin,
    // same origin
    const double ext = std::min(c->cfg.skin, 0.1 * c->rmax);
    c->oskin = c->cfg.skin + ext;
    c->odelta2 = (0.4 * ext) * (0.4 * ext);
    GridC og = g;
    og.cs = std::max(cs, 2.0 * c->rmax + c->oskin + 1e-4);
    og.gx = (int)(c->cfg.world[0] / og.cs) + 1;
    og.gy = (int)(c->cfg.world[1] / og.cs) + 1;
    og.gz = (int)(c->cfg.world[2] / og.cs) + 1;
    const long long onc = (long long)og.gx * og.gy * og.gz;
    if (onc != c->oncells) {
        free_graphs(c);
        free_cells(c);
        int rc;
        if ((rc = dalloc(&c->ccount, onc)) || (rc = dalloc(&c->cstart, onc + 1))) return rc;
        DEM_CUDA_TRY(cudaMemsetAsync(c->ccount, 0, onc * sizeof(uint), c->stream));
        c->oncells = onc;
        size_t need = scan_scratch_words(std::max<long long>(onc, c->npad + 1));
        if (need > c->scan_words) {
            DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
            cudaFree(c->scan_tmp);
            c->scan_tmp = nullptr;
            if ((rc = dalloc(&c->scan_tmp, need))) return rc;
            c->scan_words = need;
        }
    }
    const auto same = [](const GridC& a, const GridC& b) {
        return a.cs == b.cs && a.gx == b.gx && a.gy == b.gy && a.gz == b.gz;
    };
    if (!same(g, c->grid) || !same(og, c->ogrid)) free_graphs(c);
    c->grid = g;
    c->ncells = nc;
    c->ogrid = og;
    return DEM_OK;
}

static int finish_upload(dem_ctx* c) {
    // fresh start: empty previous list, zero histories, re-list on next step
    DEM_CUDA_TRY(cudaMemsetAsync(c->off[0], 0, (c->npad + 1) * sizeof(uint), c->stream));
    DEM_CUDA_TRY(cudaMemsetAsync(c->off[1], 0, (c->npad + 1) * sizeof(uint), c->stream));
    DEM_CUDA_TRY(cudaMemsetAsync(c->words, 0, sizeof(EngineWords), c->stream));
    if (c->cc_skip) DEM_CUDA_TRY(cudaMemsetAsync(c->cc_skip, 0, 2 * sizeof(uint), c->stream));
    // the outer list is rebuilt at the first re-list (new positions, radii)
    DEM_CUDA_TRY(cudaMemsetAsync(c->oflag, 0x01, sizeof(uint), c->stream));
    DEM_CUDA_TRY(cudaMemsetAsync(c->lb, 0, lb_words(c->npad) * sizeof(uint), c->stream));
    DEM_CUDA_TRY(cudaMemsetAsync(c->part_mz, 0, (size_t)c->cfg.relist_interval * c->npart * sizeof(unsigned long long),
                                 c->stream));
    DEM_CUDA_TRY(cudaMemsetAsync(c->part_cnt, 0, (size_t)c->cfg.relist_interval * c->npart * sizeof(uint), c->stream));
    c->cur = 0;
    c->sbuf = 0;
    c->hph = 0;
    c->step = 0;
    c->in_window = 0;
    c->relists = 0;
    c->last_slot = -1;
    c->uploaded = true;
    return setup_grid(c);
}

// Cell key of every particle for the upload order, (key, id) pairs: the
// cell of each coordinate is floor((p - origin) / cs) clamped to the grid
// (below the origin or not a number: cell 0), as the host computes it.
__global__ void k_cell_keys(long long n, const double* __restrict__ pos, double cs, double hx, double hy, long long gx,
                            long long gy, long long gz, uint2* __restrict__ kv) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto cell = [cs](double v, long long g) -> long long {
        const double f = v / cs;
        if (!(f >= 0.0)) return 0;
        return f >= (double)g ? g - 1 : (long long)f;
    };
    const long long cx = cell(pos[3 * i] + hx, gx), cy = cell(pos[3 * i + 1] + hy, gy), cz = cell(pos[3 * i + 2], gz);
    kv[i] = make_uint2((uint)((cz * gy + cy) * gx + cx), (uint)i);
}

__global__ void k_perm_of(long long n, const uint2* __restrict__ kv, uint* __restrict__ perm) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) perm[t] = kv[t].y;
}

// The order of a host upload: internal slot t holds the caller's particle
// perm[t], ascending (cell key, id) on the context's cell grid (any order
// that keeps neighbours together serves; this one is the re-list's).
// Computed on the device from the uploaded positions (pos: device AoS): a
// stable radix sort of (key, id) in the walk's scratch (free between
// re-lists), then the permutation goes to c->perm; the host copy that the
// id-mapping downloads use is fetched on first use (host_perm), so the
// upload does not wait for the sort.  *ordered = false (the caller's order)
// when the grid is too large (over 2^27 cells) or the particles too few.
static int device_cell_order(dem_ctx* c, const double* pos, long long n, bool* ordered) {
    c->hperm.clear();
    c->hperm_stale = false;
    *ordered = false;
    const double cs = c->cfg.cell > 0.0 ? c->cfg.cell : 2.0 * c->rmax + c->cfg.skin + 1e-4;
    if (!(cs > 0.0)) return DEM_OK;
    const long long gx = (long long)(c->cfg.world[0] / cs) + 1, gy = (long long)(c->cfg.world[1] / cs) + 1,
                    gz = (long long)(c->cfg.world[2] / cs) + 1;
    const long long nc = gx * gy * gz;
    if (nc > (1ll << 27)) return DEM_OK;
    const long long np = c->npad;
    uint2* kv = reinterpret_cast<uint2*>(c->scr);   // 2 np words
    uint2* kv2 = kv + np;                            // 2 np words
    uint* scratch = c->scr + 4 * np;                 // (kScr - 4) np words
    // the sort's histograms fit the rest of the scratch from 65 particles on;
    // fewer keep the caller's order
    if (radix_scratch_words((uint)n) > (size_t)(kScr - 4) * (size_t)np) return DEM_OK;
    int rc;
    if (!c->perm && (rc = dalloc(&c->perm, np))) return rc;
    k_cell_keys<<<grid_for(n, 256), 256, 0, c->stream>>>(n, pos, cs, 0.5 * c->cfg.world[0], 0.5 * c->cfg.world[1],
                                                         gx, gy, gz, kv);
    DEM_LAUNCH_CHECK();
    uint bits = 1;
    while (bits < 32 && (1ull << bits) < (unsigned long long)nc) bits++;
    if ((rc = radix_sort_pairs(kv, kv2, (uint)n, bits, scratch, c->stream))) return rc;
    k_perm_of<<<grid_for(n, 256), 256, 0, c->stream>>>(n, kv, c->perm);
    DEM_LAUNCH_CHECK();
    c->hperm_stale = true;
    *ordered = true;
    return DEM_OK;
}


enum UploadOrder { kOrderCaller = 0, kOrderCells = 1, kOrderGiven = 2 };

// kOrderCells (host buffers only): sort by cell; kOrderCaller: keep the
// caller's order; kOrderGiven: the buffers are already in internal order and
// `given` is its permutation (a state file's).
static int upload_impl(dem_ctx* c, const double* pos, const double* pdis, const double* angv, const double* rad,
                       bool host, int order, const uint* given) {
    if (!c || !pos || !rad) return fail(DEM_ERR_ARG, "dem_upload_state: null argument");
    // every particle the context holds is in the system again (a pour ends);
    // graphs captured for fewer particles go
    if (c->n != c->ntot) free_graphs(c);
    c->n = c->ntot;
    c->pouring = false;
    const long long n = c->n, np = c->npad;
    double* st = c->staging;
    double *spos = st, *sd = st + 3 * np, *sa = st + 6 * np, *sr = st + 9 * np;
    const double *ppos = pos, *ppd = pdis, *ppa = angv, *prad = rad;
    c->ordered = false;
    c->hperm.clear();
    c->hperm_stale = false;
    if (host) {
        // the radii first, on the second stream (after the context's earlier
        // work, which may still read the staging buffers): r_max, the solid
        // volume and the radii's validity on the device while the positions
        // copy, so that the host waits for 24 bytes instead of reducing them
        DEM_CUDA_TRY(cudaEventRecord(c->ev_up, c->stream));
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream2, c->ev_up, 0));
        DEM_CUDA_TRY(cudaMemcpyAsync(sr, rad, n * sizeof(double), cudaMemcpyHostToDevice, c->stream2));
        DEM_CUDA_TRY(cudaMemsetAsync(c->rmax_bits, 0, 3 * sizeof(unsigned long long), c->stream2));
        k_rmax<<<grid_for(n, 256), 256, 0, c->stream2>>>(n, sr, c->rmax_bits);
        k_vol<<<1, 1024, 0, c->stream2>>>(n, sr, reinterpret_cast<double*>(c->rmax_bits + 1));
        DEM_LAUNCH_CHECK();
        DEM_CUDA_TRY(cudaMemcpyAsync(c->host_pinned, c->rmax_bits, 3 * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, c->stream2));
        DEM_CUDA_TRY(cudaEventRecord(c->ev_rad, c->stream2));
        DEM_CUDA_TRY(cudaMemcpyAsync(spos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (pdis) DEM_CUDA_TRY(cudaMemcpyAsync(sd, pdis, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (angv) DEM_CUDA_TRY(cudaMemcpyAsync(sa, angv, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_rad, 0));
        // the call returns once the copies have read the caller's buffers
        // (not after the device work that follows them)
        DEM_CUDA_TRY(cudaEventRecord(c->h2d_done, c->stream));
        ppos = spos; ppd = pdis ? sd : nullptr; ppa = angv ? sa : nullptr; prad = sr;
        DEM_CUDA_TRY(cudaEventSynchronize(c->ev_rad));
        unsigned long long b[3];
        memcpy(b, c->host_pinned, sizeof(b));
        if (b[2]) {
            DEM_CUDA_TRY(cudaEventSynchronize(c->h2d_done));
            for (long long k = 0; k < n; k++)
                if (!(rad[k] > 0.0)) return fail(DEM_ERR_ARG, "dem_upload_state: radius %lld not positive", k);
        }
        double v3;
        memcpy(&c->rmax, &b[0], sizeof(double));
        memcpy(&v3, &b[1], sizeof(double));
        c->vol = 4.0 / 3.0 * M_PI * v3;
        bool cell_ordered = false;
        if (order == kOrderCells && c->reorder) {
            int rc = device_cell_order(c, spos, n, &cell_ordered);
            if (rc) return rc;
        } else if (order == kOrderGiven && given) {
            c->hperm.assign(given, given + n);
            if (!c->perm) {
                int rc = dalloc(&c->perm, np);
                if (rc) return rc;
            }
            DEM_CUDA_TRY(cudaMemcpyAsync(c->perm, c->hperm.data(), n * sizeof(uint), cudaMemcpyHostToDevice,
                                         c->stream));
        }
        c->ordered = cell_ordered || !c->hperm.empty();
    } else {
        // the caller's buffers may have been written on the legacy stream
        DEM_CUDA_TRY(cudaEventRecord(c->ext_ready, 0));
        DEM_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ext_ready, 0));
        DEM_CUDA_TRY(cudaMemsetAsync(c->rmax_bits, 0, 3 * sizeof(unsigned long long), c->stream));
        k_rmax<<<grid_for(n, 256), 256, 0, c->stream>>>(n, rad, c->rmax_bits);
        k_vol<<<1, 1024, 0, c->stream>>>(n, rad, reinterpret_cast<double*>(c->rmax_bits + 1));
        DEM_LAUNCH_CHECK();
        unsigned long long b[2] = {0, 0};
        DEM_CUDA_TRY(cudaMemcpyAsync(c->host_pinned, c->rmax_bits, sizeof(b), cudaMemcpyDeviceToHost, c->stream));
        DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        memcpy(b, c->host_pinned, sizeof(b));
        memcpy(&c->rmax, &b[0], sizeof(double));
        double v3;
        memcpy(&v3, &b[1], sizeof(double));
        c->vol = 4.0 / 3.0 * M_PI * v3;
        if (!(c->rmax > 0.0)) return fail(DEM_ERR_ARG, "dem_upload_state_device: radii not positive");
    }
    // kOrderGiven: the data are internal already (no gather), the order is recorded
    const uint* gather = (c->ordered && order == kOrderCells) ? c->perm : nullptr;
    if (c->prec == DEM_PREC_MIXED)
        k_from_aos<float><<<grid_for(n, 256), 256, 0, c->stream>>>(n, ppos, ppd, ppa, prad, (PRec<float>*)c->rec[0],
                                                                  (float*)c->rad, c->q, planes<double>(c->wh, np),
                                                                  gather);
    else
        k_from_aos<double><<<grid_for(n, 256), 256, 0, c->stream>>>(n, ppos, ppd, ppa, prad,
                                                                   (PRec<double>*)c->rec[0], (double*)c->rad, c->q,
                                                                   planes<double>(c->wh, np), gather);
    DEM_LAUNCH_CHECK();
    int rc = finish_upload(c);
    if (rc) return rc;
    if (host) DEM_CUDA_TRY(cudaEventSynchronize(c->h2d_done));   // the caller may reuse its buffers
    return DEM_OK;
}

int dem_upload_state(dem_ctx* c, const double* pos, const double* pdis, const double* angv, const double* rad) {
    NvtxRange r("dem upload");
    return upload_impl(c, pos, pdis, angv, rad, true, kOrderCells, nullptr);
}
int dem_upload_state_device(dem_ctx* c, const double* pos, const double* pdis, const double* angv, const double* rad) {
    return upload_impl(c, pos, pdis, angv, rad, false, kOrderCaller, nullptr);
}

// internal: in the internal particle order (state files); else the caller's.
static int download_common(dem_ctx* c, double* pos, double* pdis, double* angv, bool host, bool internal = false) {
    if (!c) return fail(DEM_ERR_ARG, "dem_download_state: null ctx");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_download_state: no state uploaded");
    // every particle the context holds; those not yet poured in as injected
    const long long n = c->ntot, np = c->npad, nact = c->pouring ? c->n : c->ntot;
    const int sb = c->sbuf;
    double* st = c->staging;
    double *tp = host ? st : pos, *td = host ? st + 3 * np : pdis, *ta = host ? st + 6 * np : angv;
    if (!pos) tp = nullptr;
    if (!pdis) td = nullptr;
    if (!angv) ta = nullptr;
    const uint* scatter = (c->ordered && !internal) ? c->perm : nullptr;
    if (c->prec == DEM_PREC_MIXED)
        k_to_aos<float><<<grid_for(n, 256), 256, 0, c->stream>>>(
            n, nact, (const PRec<float>*)c->rec[sb], (const PRec<float>*)c->pour_rec, tp, td, ta, scatter);
    else
        k_to_aos<double><<<grid_for(n, 256), 256, 0, c->stream>>>(
            n, nact, (const PRec<double>*)c->rec[sb], (const PRec<double>*)c->pour_rec, tp, td, ta, scatter);
    DEM_LAUNCH_CHECK();
    if (host) {
        if (pos) DEM_CUDA_TRY(cudaMemcpyAsync(pos, tp, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (pdis) DEM_CUDA_TRY(cudaMemcpyAsync(pdis, td, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (angv) DEM_CUDA_TRY(cudaMemcpyAsync(angv, ta, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DEM_OK;
}

int dem_download_state(dem_ctx* c, double* pos, double* pdis, double* angv) {
    NvtxRange r("dem download");
    return download_common(c, pos, pdis, angv, true);
}
int dem_download_state_device(dem_ctx* c, double* pos, double* pdis, double* angv) {
    return download_common(c, pos, pdis, angv, false);
}

int dem_step_n(dem_ctx* c, long long nsteps) {
    NvtxRange r("dem_step_n");
    if (!c) return fail(DEM_ERR_ARG, "dem_step_n: null ctx");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_step_n: no state uploaded");
    if (!c->have_mat) return fail(DEM_ERR_STATE, "dem_step_n: material not set");
    if (nsteps < 0) return fail(DEM_ERR_ARG, "dem_step_n: negative step count");
    const int K = c->cfg.relist_interval;
    int rc;
    while (nsteps > 0) {
        if (pour_due(c, c->step) && (rc = pour_insert(c))) return rc;
        // a whole window replays its graph unless a layer joins inside it
        // (the window then ends there: its steps run one by one)
        if (c->in_window == 0 && nsteps >= K && !c->profiling && !pour_due(c, c->step + K - 1)) {
            // whole window: replay the captured graph
            rc = launch_window_graph(c);
            if (rc) return rc;
            c->cur = 1 - c->cur;
            c->relists++;
            c->step += K;
            nsteps -= K;
            c->last_slot = K - 1;
            continue;
        }
        if (c->in_window == 0) {
            if (c->profiling) DEM_CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
            rc = relist(c, c->cur);
            if (rc) return rc;
            if (c->profiling) {
                DEM_CUDA_TRY(cudaEventRecord(c->ev[3], c->stream));
                float ms = 0.f;
                DEM_CUDA_TRY(cudaEventSynchronize(c->ev[3]));
                DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev[0], c->ev[3]));
                c->ktime[0] += ms;
                c->kcount[0]++;
            }
            c->cur = 1 - c->cur;
            c->hph = 0;
            c->relists++;
        }
        const int slot = (int)c->in_window;
        double a = 0, b = 0;
        c->observe_slot = nsteps == 1 ? slot : -1;   // the call's last step
        rc = step_kernels(c, c->cur, slot, &a, &b);
        if (rc) return rc;
        if (c->profiling) {
            c->ktime[1] += a; c->kcount[1]++;
            c->ktime[2] += b; c->kcount[2]++;
        }
        c->last_slot = slot;
        c->step++;
        nsteps--;
        c->in_window++;
        if (c->in_window == K) c->in_window = 0;
    }
    return DEM_OK;
}

int dem_set_pour(dem_ctx* c, long long nplayer, double tnewpar, long long n_active) {
    if (!c) return fail(DEM_ERR_ARG, "dem_set_pour: null ctx");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_set_pour: upload the injection states first");
    if (c->pouring) return fail(DEM_ERR_STATE, "dem_set_pour: a pour is already set (upload again to start over)");
    if (nplayer <= 0 || !(tnewpar > 0.0) || n_active < 0 || n_active > c->ntot)
        return fail(DEM_ERR_ARG, "dem_set_pour: need nplayer > 0, tnewpar > 0 and 0 <= n_active <= n");
    const long long ntot = c->ntot;
    const size_t recb = c->prec == DEM_PREC_MIXED ? sizeof(PRec<float>) : sizeof(PRec<double>);
    cudaStream_t s = c->stream;
    if (c->ordered) {
        // layers join in the caller's order: put the particles back into it
        // (the state is kept, the contact history restarts)
        std::vector<double> pos(3 * ntot), pdis(3 * ntot), angv(3 * ntot), rad(ntot), ri(ntot);
        int rc = download_common(c, pos.data(), pdis.data(), angv.data(), true);
        if (!rc) rc = host_perm(c);
        if (rc) return rc;
        if (c->prec == DEM_PREC_MIXED) {
            std::vector<float> rf(ntot);
            DEM_CUDA_TRY(cudaMemcpyAsync(rf.data(), c->rad, ntot * sizeof(float), cudaMemcpyDeviceToHost, s));
            DEM_CUDA_TRY(cudaStreamSynchronize(s));
            for (long long t = 0; t < ntot; t++) ri[t] = rf[t];
        } else {
            DEM_CUDA_TRY(cudaMemcpyAsync(ri.data(), c->rad, ntot * sizeof(double), cudaMemcpyDeviceToHost, s));
            DEM_CUDA_TRY(cudaStreamSynchronize(s));
        }
        for (long long t = 0; t < ntot; t++) rad[c->hperm[t]] = ri[t];
        const long long step = c->step, relists = c->relists;
        if ((rc = upload_impl(c, pos.data(), pdis.data(), angv.data(), rad.data(), true, kOrderCaller, nullptr)))
            return rc;
        c->step = step;
        c->relists = relists;
    }
    if (!c->pour_rec) DEM_CUDA_TRY(cudaMalloc(&c->pour_rec, (size_t)c->npad * recb));
    DEM_CUDA_TRY(cudaMemcpyAsync(c->pour_rec, c->rec[c->sbuf], (size_t)ntot * recb, cudaMemcpyDeviceToDevice, s));
    // r^3 prefix sums for the packing fraction of the particles in the system
    std::vector<double> r(ntot);
    if (c->prec == DEM_PREC_MIXED) {
        std::vector<float> rf(ntot);
        DEM_CUDA_TRY(cudaMemcpyAsync(rf.data(), c->rad, ntot * sizeof(float), cudaMemcpyDeviceToHost, s));
        DEM_CUDA_TRY(cudaStreamSynchronize(s));
        for (long long i = 0; i < ntot; i++) r[i] = rf[i];
    } else {
        DEM_CUDA_TRY(cudaMemcpyAsync(r.data(), c->rad, ntot * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    DEM_CUDA_TRY(cudaMemsetAsync(c->part_mz, 0, (size_t)c->cfg.relist_interval * c->npart * sizeof(unsigned long long),
                                 s));
    DEM_CUDA_TRY(cudaMemsetAsync(c->part_cnt, 0, (size_t)c->cfg.relist_interval * c->npart * sizeof(uint), s));
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    c->r3sum.assign(ntot + 1, 0.0);
    for (long long i = 0; i < ntot; i++) c->r3sum[i + 1] = c->r3sum[i] + r[i] * r[i] * r[i];
    if (n_active != c->n) free_graphs(c);
    c->n = n_active;
    c->vol = 4.0 / 3.0 * M_PI * c->r3sum[n_active];
    c->pour_nplayer = nplayer;
    c->pour_tnewpar = tnewpar;
    c->pouring = true;
    c->in_window = 0;   // the next step re-lists the particles in the system
    c->last_slot = -1;
    return DEM_OK;
}

int dem_active_count(dem_ctx* c, long long* n_active) {
    if (!c || !n_active) return fail(DEM_ERR_ARG, "dem_active_count: null argument");
    *n_active = c->n;
    return DEM_OK;
}

// Raw observables of the last step, as dem_scalars_enqueue leaves them in
// host memory: a header of host-side counters taken at enqueue time, the
// status words, the current list's pair count and the last step's per-block
// partials (max height, contact count).
namespace {
struct RawHead {
    long long step, relists, n, last_slot;
    double vol;
    unsigned long long npart;
    long long pad[2];
};
static_assert(sizeof(RawHead) == 64, "raw header");
constexpr size_t kRawWords = 64, kRawPairs = 80, kRawMz = 96;
size_t raw_bytes(const dem_ctx* c) { return kRawMz + c->npart * (sizeof(unsigned long long) + sizeof(uint)); }
}  // namespace

int dem_scalars_raw_bytes(dem_ctx* c, long long* bytes) {
    if (!c || !bytes) return fail(DEM_ERR_ARG, "dem_scalars_raw_bytes: null argument");
    *bytes = (long long)raw_bytes(c);
    return DEM_OK;
}

int dem_scalars_enqueue(dem_ctx* c, void* raw) {
    if (!c || !raw) return fail(DEM_ERR_ARG, "dem_scalars_enqueue: null argument");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_scalars_enqueue: no state uploaded");
    char* r = (char*)raw;
    RawHead h{};
    h.step = c->step;
    h.relists = c->relists;
    h.n = c->n;
    h.last_slot = c->last_slot;
    h.vol = c->vol;
    h.npart = c->npart;
    memcpy(r, &h, sizeof(h));
    cudaStream_t s = c->stream;
    DEM_CUDA_TRY(cudaMemcpyAsync(r + kRawWords, c->words, sizeof(EngineWords), cudaMemcpyDeviceToHost, s));
    DEM_CUDA_TRY(cudaMemcpyAsync(r + kRawPairs, c->off[c->cur] + c->n, sizeof(uint), cudaMemcpyDeviceToHost, s));
    if (c->last_slot >= 0) {
        DEM_CUDA_TRY(cudaMemcpyAsync(r + kRawMz, c->part_mz + (size_t)c->last_slot * c->npart,
                                     c->npart * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        DEM_CUDA_TRY(cudaMemcpyAsync(r + kRawMz + c->npart * sizeof(unsigned long long),
                                     c->part_cnt + (size_t)c->last_slot * c->npart, c->npart * sizeof(uint),
                                     cudaMemcpyDeviceToHost, s));
    }
    return DEM_OK;
}

int dem_scalars_from_raw(dem_ctx* c, const void* raw, dem_scalars* out) {
    if (!c || !raw || !out) return fail(DEM_ERR_ARG, "dem_scalars_from_raw: null argument");
    memset(out, 0, sizeof(*out));
    const char* r = (const char*)raw;
    RawHead h;
    memcpy(&h, r, sizeof(h));
    if (h.npart != (unsigned long long)c->npart) return fail(DEM_ERR_ARG, "dem_scalars_from_raw: not this context's");
    EngineWords w;
    memcpy(&w, r + kRawWords, sizeof(w));
    uint P;
    memcpy(&P, r + kRawPairs, sizeof(P));
    unsigned long long mzb = 0, csum = 0;
    if (h.last_slot >= 0) {
        const char* pm = r + kRawMz;
        const char* pc = pm + h.npart * sizeof(unsigned long long);
        for (size_t b = 0; b < (size_t)h.npart; b++) {
            unsigned long long m;
            uint k;
            memcpy(&m, pm + b * sizeof(m), sizeof(m));
            memcpy(&k, pc + b * sizeof(k), sizeof(k));
            mzb = std::max(mzb, m);
            csum += k;
        }
    }
    double mz;
    memcpy(&mz, &mzb, sizeof(mz));
    out->step = h.step;
    out->pairs = h.relists ? (long long)P : 0;
    out->contacts = (long long)(csum / 2);
    out->maxhz = mz;
    out->relists = h.relists;
    out->max_row = (int)w.max_row;
    // packing fraction sum (4/3) pi r^3 / (Wx Wy maxhz): dempacking.cu:768-771
    // with the monodisperse N pi/6 generalised; mean CN = pcntot/N (:768).
    out->mean_cn = h.n > 0 ? (double)csum / (double)h.n : 0.0;
    out->packing_fraction = mz > 0.0 ? h.vol / (c->cfg.world[0] * c->cfg.world[1] * mz) : 0.0;
    int status = DEM_OK;
    if (w.status & kStBarrier) {
        status = DEM_ERR_TIMEOUT;
        fail(DEM_ERR_TIMEOUT, "a bounded device wait ran out of time (sites %#x)", w.pad[0]);
    }
    else if (w.status & kStNonfinite) status = DEM_ERR_NONFINITE;
    else if (w.status & kStCapacity) status = DEM_ERR_CAPACITY;
    else if (w.status & kStSkin) status = DEM_ERR_SKIN;
    out->status = status;
    if (status == DEM_ERR_CAPACITY)
        return fail(DEM_ERR_CAPACITY, "pair list exceeded capacity %lld (rows up to %u candidates)", c->cap, w.max_row);
    if (status == DEM_ERR_NONFINITE) return fail(DEM_ERR_NONFINITE, "non-finite position or velocity");
    if (status == DEM_ERR_SKIN)
        return fail(DEM_ERR_SKIN, "a particle moved more than skin/2 = %g within a re-list window", 0.5 * c->cfg.skin);
    return DEM_OK;
}

int dem_synchronize(dem_ctx* c) {
    if (!c) return fail(DEM_ERR_ARG, "dem_synchronize: null ctx");
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DEM_OK;
}

int dem_get_scalars(dem_ctx* c, dem_scalars* out) {
    if (!c || !out) return fail(DEM_ERR_ARG, "dem_get_scalars: null argument");
    memset(out, 0, sizeof(*out));
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_get_scalars: no state uploaded");
    std::vector<unsigned long long> raw((raw_bytes(c) + 7) / 8);
    int rc = dem_scalars_enqueue(c, raw.data());
    if (rc) return rc;
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return dem_scalars_from_raw(c, raw.data(), out);
}

int dem_record_forces(dem_ctx* c, int on) {
    if (!c) return fail(DEM_ERR_ARG, "dem_record_forces: null ctx");
    if (on && !c->dbgF) {
        int rc;
        if ((rc = dalloc(&c->dbgF, 3 * c->npad)) || (rc = dalloc(&c->dbgT, 3 * c->npad)) ||
            (rc = dalloc(&c->dbgC, c->npad)))
            return rc;
    }
    if ((bool)on != c->record) free_graphs(c);
    c->record = on != 0;
    return DEM_OK;
}

int dem_download_forces(dem_ctx* c, double* force, double* torque, unsigned int* contacts) {
    if (!c) return fail(DEM_ERR_ARG, "dem_download_forces: null ctx");
    if (!c->record || !c->dbgF) return fail(DEM_ERR_STATE, "dem_download_forces: enable dem_record_forces first");
    const long long n = c->n;
    if (force) DEM_CUDA_TRY(cudaMemcpyAsync(force, c->dbgF, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (torque) DEM_CUDA_TRY(cudaMemcpyAsync(torque, c->dbgT, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (contacts) DEM_CUDA_TRY(cudaMemcpyAsync(contacts, c->dbgC, n * sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->ordered) {   // into the caller's order
        const int rc = host_perm(c);
        if (rc) return rc;
        const std::vector<uint>& pm = c->hperm;
        for (double* a : {force, torque}) {
            if (!a) continue;
            std::vector<double> t(a, a + 3 * n);
            for (long long i = 0; i < n; i++)
                for (int q = 0; q < 3; q++) a[3 * (size_t)pm[i] + q] = t[3 * (size_t)i + q];
        }
        if (contacts) {
            std::vector<uint> t(contacts, contacts + n);
            for (long long i = 0; i < n; i++) contacts[pm[i]] = t[i];
        }
    }
    return DEM_OK;
}

int dem_download_pairs(dem_ctx* c, unsigned int* lp, unsigned int* ln, double* hist, long long capn, long long* npairs) {
    if (!c || !npairs) return fail(DEM_ERR_ARG, "dem_download_pairs: null argument");
    *npairs = 0;
    if (!c->uploaded || c->relists == 0) return DEM_OK;
    const int lst = c->cur;
    uint P = 0;
    DEM_CUDA_TRY(cudaMemcpyAsync(c->host_pinned, c->off[lst] + c->n, sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    memcpy(&P, c->host_pinned, sizeof(uint));
    if ((long long)P > c->cap) return fail(DEM_ERR_CAPACITY, "dem_download_pairs: list overflowed capacity");
    *npairs = P;
    if (P == 0 || !lp || !ln) return DEM_OK;
    if ((long long)P > capn) return fail(DEM_ERR_ARG, "dem_download_pairs: host capacity %lld < %u pairs", capn, P);
    uint *dlp, *dln;
    double* dh;
    int rc;
    if ((rc = dalloc(&dlp, P)) || (rc = dalloc(&dln, P)) || (rc = dalloc(&dh, 3 * (size_t)P))) return rc;
    k_pairs_out<<<grid_for(P, 256), 256, 0, c->stream>>>(c->off[lst], c->n, c->cap, c->lp, c->ln[lst],
                                                          planes<double>(c->hist[lst][c->hph], c->cap), dlp, dln, dh);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(lp, dlp, P * sizeof(uint), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ln, dln, P * sizeof(uint), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && hist) e = cudaMemcpyAsync(hist, dh, 3 * (size_t)P * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dlp);
    cudaFree(dln);
    cudaFree(dh);
    if (e != cudaSuccess) return cuda_fail(e, "dem_download_pairs", __FILE__, __LINE__);
    if (c->ordered) {
        const int rp = host_perm(c);
        if (rp) return rp;
        // in the caller's particle ids: each pair (lower id, higher id), the
        // history in that pair's orientation (it changes sign when the two
        // swap roles), sorted by (lower, higher)
        const std::vector<uint>& pm = c->hperm;
        std::vector<uint> a(P), b(P), idx(P);
        std::vector<double> h;
        if (hist) h.assign(hist, hist + 3 * (size_t)P);
        for (uint k = 0; k < P; k++) {
            const uint u = pm[lp[k]], v = pm[ln[k]];
            a[k] = std::min(u, v);
            b[k] = std::max(u, v);
            if (hist && u > v)
                for (int q = 0; q < 3; q++) h[3 * (size_t)k + q] = -h[3 * (size_t)k + q];
            idx[k] = k;
        }
        std::sort(idx.begin(), idx.end(), [&](uint x, uint y) { return a[x] != a[y] ? a[x] < a[y] : b[x] < b[y]; });
        for (uint k = 0; k < P; k++) {
            lp[k] = a[idx[k]];
            ln[k] = b[idx[k]];
            if (hist)
                for (int q = 0; q < 3; q++) hist[3 * (size_t)k + q] = h[3 * (size_t)idx[k] + q];
        }
    }
    return DEM_OK;
}

int dem_download_cells(dem_ctx* c, unsigned int* keys, unsigned int* ids, unsigned int* cell_start,
                       unsigned int* cell_end, long long ncells_cap) {
    if (!c) return fail(DEM_ERR_ARG, "dem_download_cells: null ctx");
    if (!c->uploaded || c->relists == 0) return fail(DEM_ERR_STATE, "dem_download_cells: no list built yet");
    const long long n = c->n, nc = c->ncells;
    if ((cell_start || cell_end) && ncells_cap < nc)
        return fail(DEM_ERR_ARG, "dem_download_cells: cell capacity %lld < %lld", ncells_cap, nc);
    // each particle's cell on the configured grid at the last re-list, sorted
    // here by (cell, caller's id): the stable sort of calcHash + RadixSort
    std::vector<uint> key(n);
    DEM_CUDA_TRY(cudaMemcpyAsync(key.data(), c->ikey, n * sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (auto& k : key) k &= ~kNearWall;   // the wall-candidacy bit
    if (c->ordered) {
        const int rp = host_perm(c);
        if (rp) return rp;
    }
    std::vector<unsigned long long> kv(n);
    for (long long t = 0; t < n; t++) {
        const uint id = c->ordered ? c->hperm[t] : (uint)t;
        kv[t] = ((unsigned long long)key[t] << 32) | id;
    }
    std::sort(kv.begin(), kv.end());
    for (long long t = 0; t < n; t++) {
        if (keys) keys[t] = (uint)(kv[t] >> 32);
        if (ids) ids[t] = (uint)(kv[t] & 0xffffffffu);
    }
    if (cell_start || cell_end) {
        for (long long cc = 0; cc < nc; cc++) {
            if (cell_start) cell_start[cc] = kEmpty;
            if (cell_end) cell_end[cc] = kEmpty;
        }
        for (long long t = 0; t < n; t++) {
            const uint k = (uint)(kv[t] >> 32);
            if (k >= (uint)nc) return fail(DEM_ERR_STATE, "dem_download_cells: cell key %u outside the grid", k);
            if (t == 0 || (uint)(kv[t - 1] >> 32) != k)
                if (cell_start) cell_start[k] = (uint)t;
            if (t == n - 1 || (uint)(kv[t + 1] >> 32) != k)
                if (cell_end) cell_end[k] = (uint)(t + 1);
        }
    }
    return DEM_OK;
}

int dem_grid_info(dem_ctx* c, unsigned int grid[3], double* cell, long long* ncells) {
    if (!c) return fail(DEM_ERR_ARG, "dem_grid_info: null ctx");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_grid_info: no state uploaded");
    if (grid) { grid[0] = c->grid.gx; grid[1] = c->grid.gy; grid[2] = c->grid.gz; }
    if (cell) *cell = c->grid.cs;
    if (ncells) *ncells = c->ncells;
    return DEM_OK;
}

int dem_set_profiling(dem_ctx* c, int on) {
    if (!c) return fail(DEM_ERR_ARG, "dem_set_profiling: null ctx");
    c->profiling = on != 0;
    for (int k = 0; k < 3; k++) { c->ktime[k] = 0; c->kcount[k] = 0; }
    return DEM_OK;
}

int dem_kernel_times(dem_ctx* c, double out[3]) {
    if (!c || !out) return fail(DEM_ERR_ARG, "dem_kernel_times: null argument");
    for (int k = 0; k < 3; k++) out[k] = c->kcount[k] ? c->ktime[k] / c->kcount[k] : 0.0;
    return DEM_OK;
}

int dem_set_window_timing(dem_ctx* c, int on) {
    if (!c) return fail(DEM_ERR_ARG, "dem_set_window_timing: null ctx");
    const size_t need = 4 + 2 * (size_t)c->cfg.relist_interval;
    if (on && c->wev.size() < need) {
        for (size_t k = c->wev.size(); k < need; k++) {
            cudaEvent_t e = nullptr;
            DEM_CUDA_TRY(cudaEventCreate(&e));
            c->wev.push_back(e);
        }
    }
    c->wtiming = on != 0;
    return DEM_OK;
}

int dem_check_barrier_timeout(dem_ctx* c, double* waited_ms) {
    if (!c || !waited_ms) return fail(DEM_ERR_ARG, "dem_check_barrier_timeout: null argument");
    *waited_ms = 0.0;
    if (c->in_window != 0) return fail(DEM_ERR_STATE, "dem_check_barrier_timeout: call at a re-list boundary");
    unsigned long long* spent = nullptr;
    int rc = dalloc(&spent, 1);
    if (rc) return rc;
    cudaStream_t s = c->stream;
    cudaError_t e = cudaMemsetAsync(c->bar, 0, kBarWords * sizeof(uint), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(spent, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        k_barrier_check<<<1, 32, 0, s>>>(c->bar, c->words, spent);
        e = cudaGetLastError();
    }
    unsigned long long ns = 0;
    EngineWords w{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ns, spent, sizeof(ns), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&w, c->words, sizeof(w), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(spent);
    if (e != cudaSuccess) return cuda_fail(e, "dem_check_barrier_timeout", __FILE__, __LINE__);
    *waited_ms = (double)ns * 1e-6;
    if (!(w.status & kStBarrier))
        return fail(DEM_ERR_STATE, "dem_check_barrier_timeout: the wait did not report its timeout");
    return DEM_OK;
}

int dem_window_work(dem_ctx* c, long long* bound, long long* wall_candidates, long long* pairs, int* batched) {
    if (!c) return fail(DEM_ERR_ARG, "dem_window_work: null ctx");
    if (bound) *bound = 0;
    if (wall_candidates) *wall_candidates = 0;
    if (pairs) *pairs = 0;
    if (batched) *batched = 0;
    if (!c->uploaded || c->relists == 0) return DEM_OK;
    uint v[4] = {0, 0, 0, 1};
    uint* hp = (uint*)c->host_pinned;
    DEM_CUDA_TRY(cudaMemcpyAsync(hp, c->bpos + c->n, sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaMemcpyAsync(hp + 1, c->wcount, sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    DEM_CUDA_TRY(cudaMemcpyAsync(hp + 2, c->off[c->cur] + c->n, sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    if (use_batches(c))
        DEM_CUDA_TRY(cudaMemcpyAsync(hp + 3, c->cc_words + 1, sizeof(uint), cudaMemcpyDeviceToHost, c->stream));
    else
        hp[3] = 1u;
    DEM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    memcpy(v, hp, sizeof(v));
    if (bound) *bound = v[0];
    if (wall_candidates) *wall_candidates = v[1];
    if (pairs) *pairs = (long long)v[2] <= c->cap ? v[2] : 0;
    if (batched) *batched = !use_batches(c) ? -1 : (v[3] == 0u ? 1 : 0);
    return DEM_OK;
}

int dem_window_kernel_times(dem_ctx* c, double out[5]) {
    if (!c || !out) return fail(DEM_ERR_ARG, "dem_window_kernel_times: null argument");
    for (int k = 0; k < 5; k++) out[k] = 0.0;
    if (!c->wtiming_ran) return fail(DEM_ERR_STATE, "dem_window_kernel_times: no timed window has run");
    const int K = c->cfg.relist_interval;
    float ms = 0.f;
    if (c->wtiming_path == 1) {   // window kernel
        DEM_CUDA_TRY(cudaEventSynchronize(c->wev[2]));
        DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->wev[0], c->wev[1]));
        out[0] = ms;
        DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->wev[1], c->wev[2]));
        out[4] = ms;
        return DEM_OK;
    }
    DEM_CUDA_TRY(cudaEventSynchronize(c->wev[3 + 2 * (K - 1)]));
    DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->wev[0], c->wev[1]));
    out[0] = ms;
    for (int s = 0; s < K; s++) {
        cudaEvent_t prev = s == 0 ? c->wev[1] : c->wev[3 + 2 * (s - 1)];
        DEM_CUDA_TRY(cudaEventElapsedTime(&ms, prev, c->wev[2 + 2 * s]));
        out[1] += ms / K;
        DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->wev[2 + 2 * s], c->wev[3 + 2 * s]));
        out[2] += ms / K;
    }
    if (c->wtiming_path == 2) {   // forked free-particle kernel
        DEM_CUDA_TRY(cudaEventSynchronize(c->wev[3 + 2 * K]));
        DEM_CUDA_TRY(cudaEventElapsedTime(&ms, c->wev[2 + 2 * K], c->wev[3 + 2 * K]));
        out[3] = ms;
    }
    return DEM_OK;
}


// ------------------------------------------------------ checkpoint / resume
// The reference's restart path (dempacking.cu:361-367, commented out there)
// would re-read preflow.dat, which has neither the pair nor the wall history.
// This file holds the whole engine state at a re-list boundary: particle
// state, displacement-since-list words, wall history and the previous pair
// list with its FP64 tangential history (the next re-list carries from it),
// the step counters, the material and a pour in progress (particles not yet
// in the system are stored with their injection states).  Native byte order,
// this library only.
namespace {
struct StateHeader {
    char magic[8];
    int version, precision, force_mode, relist_interval;
    long long n, step, relists, npairs;
    double dt, skin, cell, density, world[3], rmax, vol;
    int have_mat, pouring;
    dem_material mat;
    long long n_active, pour_nplayer;
    double pour_tnewpar;
    long long ordered;   // the particle order follows (n uint32 after the header)
};
constexpr char kStateMagic[8] = {'D', 'E', 'M', 'B', '2', '0', '0', 'S'};
constexpr int kStateVersion = 3;

int write_all(FILE* f, const void* p, size_t bytes) {
    return fwrite(p, 1, bytes, f) == bytes ? DEM_OK : fail(DEM_ERR_IO, "dem_save_state: write failed");
}
int read_all(FILE* f, void* p, size_t bytes) {
    return fread(p, 1, bytes, f) == bytes ? DEM_OK : fail(DEM_ERR_IO, "dem_load_state: truncated state file");
}
}  // namespace

int dem_save_state(dem_ctx* c, const char* path) {
    if (!c || !path) return fail(DEM_ERR_ARG, "dem_save_state: null argument");
    if (!c->uploaded) return fail(DEM_ERR_STATE, "dem_save_state: no state uploaded");
    if (c->in_window != 0)
        return fail(DEM_ERR_STATE, "dem_save_state: save at a re-list boundary (step a multiple of relist_interval)");
    // particle sections: every particle held; list: the particles in the system
    const long long n = c->ntot, na = c->n, np = c->npad;
    std::vector<double> pos(3 * n), pdis(3 * n), angv(3 * n), rad(n), wh(3 * n);
    std::vector<float4> q(n);
    int rc = download_common(c, pos.data(), pdis.data(), angv.data(), true, true);   // internal order
    if (rc) return rc;
    uint P = 0;
    cudaStream_t s = c->stream;
    DEM_CUDA_TRY(cudaMemcpyAsync(&P, c->off[c->cur] + na, sizeof(uint), cudaMemcpyDeviceToHost, s));
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    if ((long long)P > c->cap) P = 0;   // an overflowed list carries nothing
    std::vector<uint> off(na + 1), ln(P);
    std::vector<double> hist(3 * (size_t)P);
    if (c->prec == DEM_PREC_MIXED) {
        std::vector<float> rf(n);
        DEM_CUDA_TRY(cudaMemcpyAsync(rf.data(), c->rad, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        DEM_CUDA_TRY(cudaStreamSynchronize(s));
        for (long long i = 0; i < n; i++) rad[i] = rf[i];
    } else {
        DEM_CUDA_TRY(cudaMemcpyAsync(rad.data(), c->rad, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    DEM_CUDA_TRY(cudaMemcpyAsync(q.data(), c->q, n * sizeof(float4), cudaMemcpyDeviceToHost, s));
    for (int a = 0; a < 3; a++)
        DEM_CUDA_TRY(cudaMemcpyAsync(wh.data() + a * n, c->wh + a * np, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    DEM_CUDA_TRY(cudaMemcpyAsync(off.data(), c->off[c->cur], (na + 1) * sizeof(uint), cudaMemcpyDeviceToHost, s));
    if (P) {
        DEM_CUDA_TRY(cudaMemcpyAsync(ln.data(), c->ln[c->cur], P * sizeof(uint), cudaMemcpyDeviceToHost, s));
        const double* h = c->hist[c->cur][c->hph];
        for (int a = 0; a < 3; a++)
            DEM_CUDA_TRY(cudaMemcpyAsync(hist.data() + (size_t)a * P, h + a * c->cap, P * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
    } else {
        std::fill(off.begin(), off.end(), 0u);
    }
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    StateHeader hd = {};
    memcpy(hd.magic, kStateMagic, 8);
    hd.version = kStateVersion;
    hd.precision = c->prec;
    hd.force_mode = c->mode;
    hd.relist_interval = c->cfg.relist_interval;
    hd.n = n;
    hd.step = c->step;
    hd.relists = c->relists;
    hd.npairs = P;
    hd.dt = c->cfg.dt; hd.skin = c->cfg.skin; hd.cell = c->cfg.cell; hd.density = c->cfg.density;
    for (int a = 0; a < 3; a++) hd.world[a] = c->cfg.world[a];
    hd.rmax = c->rmax;
    hd.vol = c->vol;
    hd.have_mat = c->have_mat ? 1 : 0;
    hd.mat = c->mat;
    hd.pouring = c->pouring ? 1 : 0;
    hd.n_active = na;
    hd.pour_nplayer = c->pour_nplayer;
    hd.pour_tnewpar = c->pour_tnewpar;
    hd.ordered = c->ordered ? 1 : 0;
    if (c->ordered && (rc = host_perm(c))) return rc;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    rc = write_all(f, &hd, sizeof(hd));
    if (!rc && c->ordered) rc = write_all(f, c->hperm.data(), n * sizeof(uint));
    if (!rc) rc = write_all(f, pos.data(), pos.size() * sizeof(double));
    if (!rc) rc = write_all(f, pdis.data(), pdis.size() * sizeof(double));
    if (!rc) rc = write_all(f, angv.data(), angv.size() * sizeof(double));
    if (!rc) rc = write_all(f, rad.data(), rad.size() * sizeof(double));
    if (!rc) rc = write_all(f, q.data(), q.size() * sizeof(float4));
    if (!rc) rc = write_all(f, wh.data(), wh.size() * sizeof(double));
    if (!rc) rc = write_all(f, off.data(), off.size() * sizeof(uint));
    if (!rc && P) rc = write_all(f, ln.data(), ln.size() * sizeof(uint));
    if (!rc && P) rc = write_all(f, hist.data(), hist.size() * sizeof(double));
    if (fclose(f) != 0 && !rc) rc = fail(DEM_ERR_IO, "dem_save_state: close failed");
    return rc;
}

int dem_load_state(dem_ctx* c, const char* path) {
    if (!c || !path) return fail(DEM_ERR_ARG, "dem_load_state: null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    StateHeader hd;
    int rc = read_all(f, &hd, sizeof(hd));
    if (!rc && (memcmp(hd.magic, kStateMagic, 8) != 0 || hd.version != kStateVersion))
        rc = fail(DEM_ERR_IO, "dem_load_state: %s is not a state file of this library", path);
    if (!rc && (hd.n != c->ntot || hd.precision != c->prec || hd.force_mode != c->mode ||
                hd.relist_interval != c->cfg.relist_interval))
        rc = fail(DEM_ERR_ARG, "dem_load_state: the context differs from the saved one (n %lld/%lld, precision, "
                  "force mode or relist_interval)", hd.n, c->ntot);
    if (!rc && (hd.n_active < 0 || hd.n_active > hd.n || (!hd.pouring && hd.n_active != hd.n) ||
                (hd.pouring && (hd.pour_nplayer <= 0 || !(hd.pour_tnewpar > 0.0) || hd.ordered))))
        rc = fail(DEM_ERR_IO, "dem_load_state: %s holds an inconsistent pour", path);
    if (!rc && (hd.npairs < 0 || hd.npairs > c->cap))
        rc = fail(DEM_ERR_CAPACITY, "dem_load_state: %lld saved pairs exceed the pair capacity", hd.npairs);
    if (rc) { fclose(f); return rc; }
    const long long n = c->ntot, na = hd.n_active, np = c->npad, P = hd.npairs;
    std::vector<double> pos(3 * n), pdis(3 * n), angv(3 * n), rad(n), wh(3 * n), hist(3 * (size_t)P);
    std::vector<float4> q(n);
    std::vector<uint> off(na + 1), ln(P), order;
    if (hd.ordered) {   // the particle order: a permutation of 0 .. n-1
        order.resize(n);
        rc = read_all(f, order.data(), n * sizeof(uint));
        std::vector<unsigned char> seen(n, 0);
        for (long long t = 0; !rc && t < n; t++) {
            if ((long long)order[t] >= n || seen[order[t]]) {
                rc = fail(DEM_ERR_IO, "dem_load_state: %s holds a malformed particle order", path);
                break;
            }
            seen[order[t]] = 1;
        }
        if (rc) { fclose(f); return rc; }
    }
    rc = read_all(f, pos.data(), pos.size() * sizeof(double));
    if (!rc) rc = read_all(f, pdis.data(), pdis.size() * sizeof(double));
    if (!rc) rc = read_all(f, angv.data(), angv.size() * sizeof(double));
    if (!rc) rc = read_all(f, rad.data(), rad.size() * sizeof(double));
    if (!rc) rc = read_all(f, q.data(), q.size() * sizeof(float4));
    if (!rc) rc = read_all(f, wh.data(), wh.size() * sizeof(double));
    if (!rc) rc = read_all(f, off.data(), off.size() * sizeof(uint));
    if (!rc && P) rc = read_all(f, ln.data(), ln.size() * sizeof(uint));
    if (!rc && P) rc = read_all(f, hist.data(), hist.size() * sizeof(double));
    fclose(f);
    if (rc) return rc;
    // the list drives device indexing: rows must be well formed (offsets from
    // 0 to P, non-decreasing; partners j > i, ascending, among the particles
    // in the system)
    bool ok = off[0] == 0u && (long long)off[na] == P;
    for (long long i = 0; ok && i < na; i++) {
        if (off[i + 1] < off[i]) { ok = false; break; }
        for (uint k = off[i]; k < off[i + 1]; k++)
            if (ln[k] <= (uint)i || (long long)ln[k] >= na || (k > off[i] && ln[k] <= ln[k - 1])) { ok = false; break; }
    }
    if (!ok) return fail(DEM_ERR_IO, "dem_load_state: %s holds a malformed pair list", path);
    if (hd.have_mat && (rc = dem_set_material(c, &hd.mat))) return rc;
    // the sections are in the saved context's internal order
    if ((rc = upload_impl(c, pos.data(), pdis.data(), angv.data(), rad.data(), true,
                          hd.ordered ? kOrderGiven : kOrderCaller, hd.ordered ? order.data() : nullptr)))
        return rc;
    // particles not yet poured in wait with the injection states just uploaded
    if (hd.pouring && (rc = dem_set_pour(c, hd.pour_nplayer, hd.pour_tnewpar, na))) return rc;
    // the upload started afresh (list buffer 0 current, empty); put back the
    // rest of the saved state
    cudaStream_t s = c->stream;
    DEM_CUDA_TRY(cudaMemcpyAsync(c->q, q.data(), n * sizeof(float4), cudaMemcpyHostToDevice, s));
    for (int a = 0; a < 3; a++)
        DEM_CUDA_TRY(cudaMemcpyAsync(c->wh + a * np, wh.data() + a * n, n * sizeof(double), cudaMemcpyHostToDevice, s));
    DEM_CUDA_TRY(cudaMemcpyAsync(c->off[0], off.data(), (na + 1) * sizeof(uint), cudaMemcpyHostToDevice, s));
    std::vector<uint> lp(P);   // each pair's row (the lower particle), as a re-list writes it
    for (long long i = 0; i < na; i++)
        for (uint k = off[i]; k < off[i + 1]; k++) lp[k] = (uint)i;
    if (P) {
        DEM_CUDA_TRY(cudaMemcpyAsync(c->lp, lp.data(), P * sizeof(uint), cudaMemcpyHostToDevice, s));
        DEM_CUDA_TRY(cudaMemcpyAsync(c->ln[0], ln.data(), P * sizeof(uint), cudaMemcpyHostToDevice, s));
        for (int a = 0; a < 3; a++)
            DEM_CUDA_TRY(cudaMemcpyAsync(c->hist[0][0] + a * c->cap, hist.data() + (size_t)a * P, P * sizeof(double),
                                         cudaMemcpyHostToDevice, s));
    }
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    c->step = hd.step;
    c->relists = hd.relists;
    c->rmax = hd.rmax;
    c->vol = hd.vol;
    return DEM_OK;
}

}  // extern "C"
