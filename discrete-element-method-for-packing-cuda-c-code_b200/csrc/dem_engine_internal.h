// dem_engine_internal.h -- the engine context and the launchers shared by
// dem_engine.cu (forward step) and dem_adjoint.cu (its reverse mode).
#pragma once
#include <vector>
#include "dem_common.cuh"
#include "dem_law.cuh"

namespace dem {

enum : uint {
    kStCapacity = 1u,
    kStNonfinite = 2u,
    kStSkin = 4u,
    kStBarrier = 8u,   // a bounded wait (window-kernel grid barrier, scan look-back) ran out of time
};

// device words: [0] status bits, [1] max row count, pad[0]: which bounded
// waits gave up (kStBarrier)
struct EngineWords {
    uint status;
    uint max_row;
    uint pad[2];
};

template <typename Real> struct Planes3 { Real* x; Real* y; Real* z; };

// Particle record: FP64 position and per-step displacement, rotation (per-step
// angle) and radius in the working precision.  One record per particle, so a
// gathered particle costs 2 (mixed: 64 B) or 3 (FP64: 96 B) 32-byte sectors
// instead of one per field.
template <typename Real> struct PRec;
template <> struct alignas(64) PRec<float> {
    double x, y, z, dx, dy, dz;
    float ax, ay, az, r;
};
template <> struct alignas(32) PRec<double> {
    double x, y, z, dx, dy, dz;
    double ax, ay, az, r, pad0, pad1;
};
static_assert(sizeof(PRec<float>) == 64 && sizeof(PRec<double>) == 96, "record layout");

// Record access by 16-byte vectors; COH: L2-coherent loads (.cg) for data that
// other blocks of the same launch write.
template <bool COH, typename T> __device__ __forceinline__ T ldv(const T* p) {
    if constexpr (COH) return __ldcg(p);
    else return *p;
}
template <bool COH>
__device__ __forceinline__ void ld_rec(const PRec<float>* p, V3<double>& x, V3<double>& d, V3<float>& a, float& r) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 v0 = ldv<COH>(q), v1 = ldv<COH>(q + 1), v2 = ldv<COH>(q + 2);
    const float4 v3 = ldv<COH>(reinterpret_cast<const float4*>(p) + 3);
    x = mk(v0.x, v0.y, v1.x);
    d = mk(v1.y, v2.x, v2.y);
    a = mk(v3.x, v3.y, v3.z);
    r = v3.w;
}
template <bool COH>
__device__ __forceinline__ void ld_rec(const PRec<double>* p, V3<double>& x, V3<double>& d, V3<double>& a,
                                       double& r) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 v0 = ldv<COH>(q), v1 = ldv<COH>(q + 1), v2 = ldv<COH>(q + 2), v3 = ldv<COH>(q + 3),
                  v4 = ldv<COH>(q + 4);
    x = mk(v0.x, v0.y, v1.x);
    d = mk(v1.y, v2.x, v2.y);
    a = mk(v3.x, v3.y, v4.x);
    r = v4.y;
}
template <bool COH, typename Real> __device__ __forceinline__ V3<double> ld_pos(const PRec<Real>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 v0 = ldv<COH>(q), v1 = ldv<COH>(q + 1);
    return mk(v0.x, v0.y, v1.x);
}
__device__ __forceinline__ void st_rec(PRec<float>* p, V3<double> x, V3<double> d, V3<float> a, float r) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(x.x, x.y);
    q[1] = make_double2(x.z, d.x);
    q[2] = make_double2(d.y, d.z);
    reinterpret_cast<float4*>(p)[3] = make_float4(a.x, a.y, a.z, r);
}
__device__ __forceinline__ void st_rec(PRec<double>* p, V3<double> x, V3<double> d, V3<double> a, double r) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(x.x, x.y);
    q[1] = make_double2(x.z, d.x);
    q[2] = make_double2(d.y, d.z);
    q[3] = make_double2(a.x, a.y);
    q[4] = make_double2(a.z, r);
}

struct GridC {
    double ox, oy, oz;   // world origin
    double cs;
    int gx, gy, gz;      // grid size
};

struct StepPartials { unsigned long long* maxhz_bits; uint* contacts; };

// Tape written by the window kernel for the adjoint's recompute (see
// StepArgs in dem_engine.cu); ta is Real.
struct WindowTape {
    double *tx, *td, *twh, *tF, *tT, *th;
    void* ta;
    int step0;
    uint* tc;   // per particle and step: its pair contacts
};

struct ParticleCommon {
    double dt, hx, hy;
    float half_skin2;
    int first;
    int observe;   // write this step's per-block observables (max height, contacts)
};

// Cluster batches: batches of whole components, at most BatchCap<Real>::P
// particles and ::Q listed pairs each (what one block of k_batch holds in
// shared memory).  A batch takes the components whose first slot falls
// in one window of `target` slots; the re-list chooses target per window as
// the bound particles over the batch kernel's resident blocks (one round of
// blocks), at least kBatchMin and at most P minus the largest component.
constexpr uint kBatchMin = 32;
constexpr uint kDenseSkip = 32;          // re-lists without the component pass after one larger than a block
// Blocks of 256 threads holding up to 256 (FP64: 192) particles and 320
// pairs: three (FP64: two) resident per SM, so that one block's barrier
// waits overlap another's steps.
constexpr int kBatchThreads = 256;       // k_batch: one particle per thread
template <typename Real> struct BatchCap;
template <> struct BatchCap<float> { static constexpr uint P = 256, Q = 320; };
template <> struct BatchCap<double> { static constexpr uint P = 192, Q = 320; };

// Exclusive scan of in[0, m) into out over the block (m <= a few thousand);
// returns the total to every thread.  tmp: 33 words of shared memory.
__device__ __forceinline__ uint block_exscan(const uint* in, uint* out, uint m, uint* tmp) {
    const uint per = (m + blockDim.x - 1) / blockDim.x;
    const uint b = threadIdx.x * per, e = min(b + per, m);
    uint sum = 0;
    for (uint k = b; k < e; k++) sum += in[k];
    const uint lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)lane >= o) inc += v;
    }
    if (lane == 31) tmp[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint acc = 0;
        for (uint w = 0; w < (blockDim.x >> 5); w++) { const uint t = tmp[w]; tmp[w] = acc; acc += t; }
        tmp[32] = acc;
    }
    __syncthreads();
    uint run = tmp[warp] + inc - sum;
    for (uint k = b; k < e; k++) { const uint v = in[k]; out[k] = run; run += v; }
    const uint total = tmp[32];
    __syncthreads();
    return total;
}

}  // namespace dem

using dem::EngineWords;
using dem::GridC;
using dem::uint;
namespace dem { struct AdjWork; }

struct dem_ctx {
    dem_config cfg{};
    int prec = DEM_PREC_MIXED;
    int mode = DEM_FORCE_PCCP;
    long long n = 0, npad = 0, cap = 0;   // n: particles in the system (the first n of ntot)
    long long ntot = 0;                    // particles the context holds (dem_config.n)
    // poured packing: particles n .. ntot-1 wait in pour_rec (their injection
    // records) and join nplayer at a time (dem_set_pour)
    bool pouring = false;
    long long pour_nplayer = 0;
    double pour_tnewpar = 0.0;
    void* pour_rec = nullptr;              // PRec<Real>[npad]
    std::vector<double> r3sum;             // r3sum[k] = sum of r^3 over the first k particles
    // particle order: the host upload sorts the particles by cell (locality of
    // every gather and scatter); internal slot t holds the caller's particle
    // perm[t].  Results leave in the caller's order.
    bool reorder = true;                   // host uploads sort by cell (DEM_B200_REORDER=0: off)
    bool ordered = false;
    uint* perm = nullptr;                  // device copy (npad)
    std::vector<uint> hperm;               // host copy (n), fetched on first use after an upload
    bool hperm_stale = false;              // the device copy is newer than hperm
    cudaEvent_t h2d_done = nullptr;        // a host upload's copies have read the caller's buffers
    cudaEvent_t ev_up = nullptr, ev_rad = nullptr;   // a host upload: its start; its radii reduced
    int device = 0;
    cudaStream_t stream = 0;
    cudaStream_t own_stream = 0;      // non-blocking; used unless dem_set_stream gives one
    cudaEvent_t ext_ready = nullptr;  // orders legacy-stream work before device uploads
    dem_material mat{};
    bool have_mat = false;
    // grid: the configured one (cell keys of dem_download_cells), and the
    // outer list's (cells >= 2 r_max + oskin), whose cell arrays the re-list uses
    GridC grid{};
    long long ncells = 0;
    GridC ogrid{};
    long long oncells = 0;
    double rmax = 0.0;
    double vol = 0.0;        // sum (4/3) pi r^3
    // state: [current buffer]; the second buffer exists in PP mode only
    void* rec[2] = {nullptr, nullptr};     // PRec<Real>[npad] per state buffer
    int sbuf = 0;
    void* rad = nullptr;     // Real
    float4* q = nullptr;
    double* wh = nullptr;    // 3 planes
    double* staging = nullptr;   // 10n doubles
    // list: the outer build's cell arrays (outer grid)
    uint* key = nullptr;
    uint* sid = nullptr;     // unordered within cells (scatter)
    uint* skeyu = nullptr;
    void* sposu = nullptr;
    uint* ccount = nullptr;
    uint* cstart = nullptr;
    uint* njgi = nullptr;
    uint* njli = nullptr;
    uint* arrival = nullptr; // per particle: slot among its cell's members (hash order)
    uint* scr = nullptr;     // per particle: the walk's first kScr row candidates
    uint* tpos = nullptr;    // per particle: its slot in the cell-sorted order
    uint* bflag = nullptr;   // per particle: 1 = bound this window (a listed pair or a wall candidacy)
    uint* bpos = nullptr;    // exclusive scan of bflag; bpos[n] = number of bound particles
    uint* blist = nullptr;   // bound particle ids, ascending
    uint* flist = nullptr;   // free particle ids, ascending
    // outer candidate list: rows of every particle within r_i + r_j + oskin
    // at the build (both directions), kept while every particle stays within
    // odelta of its position then (oskin, odelta: set with the grid)
    double oskin = 0.0, odelta2 = 0.0;
    uint* coff = nullptr;    // np + 1: row offsets
    uint* cln = nullptr;     // ccap: candidates
    long long ccap = 0;
    uint* ocnt = nullptr;    // np: row lengths (build)
    double* xo = nullptr;    // 3 planes: positions at the build
    uint* oflag = nullptr;   // [0] nonzero: the list is invalid (rebuild at the next re-list)
    uint* ikey = nullptr;    // np: each particle's cell on the configured grid at the last re-list
    cudaStream_t cstream = 0;        // captures the outer build into its conditional node
    bool outer_cond = true;          // DEM_B200_OUTER_COND=0: build in every re-list
    unsigned bound_grid = 0;         // blocks of the re-list passes over the bound particles (grid-stride)
    uint* lb = nullptr;              // the candidate pass's look-back: [0] tile ticket, then 3 64-bit words per tile
    cudaStream_t stream2 = 0;        // free-particle branch of the window graph
    cudaEvent_t evfork = nullptr, evjoin = nullptr;
    int prio_hi = 0;                 // the device's highest stream priority (the batch kernel's launches)
    int win_minb = 1;                // window-kernel blocks per SM (DEM_B200_WINDOW_MINB)
    bool free_in_window = false;     // capturing: the free particles run as one window kernel
    bool free_early = false;         // enqueueing a batched window: the re-list forks its free particles
    int free_fork = 1;               // where (DEM_B200_FREE_FORK): 0 in the window, 1 after the candidate pass, 2 after the fill
    uint* bar = nullptr;             // window-kernel grid barrier: [0] arrival counter
    unsigned win_grid = 1;           // window-kernel blocks (all co-resident)
    bool win_kernel = true;          // whole PCCP windows as one cooperative launch
    int win_split = 0;               // window kernels: bound items per thread of the bound blocks (0: no split)
    int wtiming_path = 0;            // last timed window: 0 per-step, 1 window kernel, 2 per-step + forked free
    uint* off[2] = {nullptr, nullptr};
    uint* roff = nullptr;
    uint* ln[2] = {nullptr, nullptr};
    uint* lp = nullptr;
    double* hist[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [list buffer][phase], 3 planes of cap
    int hph = 0;             // history phase of the current list (PP ping-pong)
    uint* rk = nullptr;
    uint* carry = nullptr;   // optional carry-map output of relist (adjoint recompute)
    // cluster batches (PCCP windows): the window's bound particles grouped by
    // connected component of the pair list; small components are packed into
    // batches that one block steps through the whole window in shared memory
    bool batching = true;            // DEM_B200_BATCH=0: the grid-barrier window kernel for every window
    uint* cc_parent = nullptr;       // np: union-find parent, then the component root (its smallest id)
    uint* cc_size = nullptr;         // np: per root: bound particles of the component
    uint* cc_pairs = nullptr;        // np: per root: listed pairs of the component
    uint* cc_fill = nullptr;         // np: per root: slots handed out so far
    uint* cc_base = nullptr;         // np: per root: the component's first slot
    uint* cc_bw = nullptr;           // 3 (nbatch_max + 2): per batch first slot, particles, pairs
    uint* cc_order = nullptr;        // np: bound particle ids, grouped by component
    uint* cc_batch = nullptr;        // nbatch_max + 1: first slot of each batch
    uint* cc_loc = nullptr;          // np: a batch particle's index inside its block
    uint* cc_skip = nullptr;         // [0] re-lists left that skip the component pass (a dense bed)
    uint* cc_words = nullptr;        // [0] slots handed out, [1] 1 = a batch too large (or the list overflowed),
                                     // [2] largest component, [3] batch window (slots)
    long long nbatch_max = 0;
    unsigned batch_grid = 1;         // blocks of the batch kernel
    size_t batch_smem = 0;           // its dynamic shared memory
    uint* wslot = nullptr;   // per particle: wall-candidate slot of this window or kEmpty
    uint* wlist = nullptr;   // wall candidates (particle ids)
    uint* wcount = nullptr;  // number of wall candidates (device)
    void* wf = nullptr;      // per candidate: wall force, wall torque (R4 each)
    uint* ru = nullptr;      // per pair: its slot in the reverse rows
    void* pf = nullptr;      // per pair (row slot): force on lo, .w = contact
    void* pti = nullptr;     // per pair (row slot): torque on lo
    void* rfj = nullptr;     // per reverse slot: force on hi, .w = contact
    void* rtj = nullptr;     // per reverse slot: torque on hi
    unsigned pair_grid = 1;  // one wave of the pair kernel
    bool pdl = true;         // programmatic launches: window steps, re-list, reverse sweep
    uint* scan_tmp = nullptr;
    size_t scan_words = 0;
    // scalars
    EngineWords* words = nullptr;
    unsigned long long* part_mz = nullptr;   // relist_interval x npart
    uint* part_cnt = nullptr;                // relist_interval x npart
    unsigned nblk = 0;                       // blocks of the particle kernel
    size_t fpart = 0;                        // partials per slot of the particle kernels (>= nblk, window grid)
    size_t npart = 0;                        // partials per slot: fpart + nblk (the free kernel's)
    unsigned long long* rmax_bits = nullptr;
    void* host_pinned = nullptr;     // mirror for scalars
    // debug force record
    bool record = false;
    double* dbgF = nullptr;
    double* dbgT = nullptr;
    uint* dbgC = nullptr;
    // schedule
    int cur = 0;
    long long step = 0, in_window = 0, relists = 0;
    int last_slot = -1;
    int observe_slot = -1;   // window slot whose step writes the observables
    bool uploaded = false;
    // window graphs keyed by (previous list buffer, state buffer, history
    // phase, with timing events)
    cudaGraphExec_t gexec[2][2][2][2] = {};
    // timing events inside window graphs: [0] window start, [1] after the
    // re-list, [2 + 2s] after the pair launch of slot s, [3 + 2s] after its
    // particle launch
    bool wtiming = false;
    bool wtiming_capture = false;
    bool wtiming_ran = false;
    std::vector<cudaEvent_t> wev;
    // profiling
    bool profiling = false;
    double ktime[3] = {0, 0, 0};
    long long kcount[3] = {0, 0, 0};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    dem::AdjWork* adj = nullptr;     // adjoint workspace (dem_adjoint.cu)
};


namespace dem {
// Launchers (dem_engine.cu).  relist(): list build from the current state,
// carrying history from list buffer `src` into 1-src; when c->carry is set,
// carry[k] receives the previous slot of new pair k (kEmpty if new).
// step_kernels(): one DEM step on list buffer `lst`, window slot `slot`.
// window_kernel(): all steps of a window on list buffer `lst` (PCCP, window
// kernel enabled), optionally writing the adjoint tape.
int relist(dem_ctx* c, int src);
int step_kernels(dem_ctx* c, int lst, int slot, double* ms_pair, double* ms_part);
int window_kernel(dem_ctx* c, int lst, const WindowTape* tape);
// Whether PCCP windows run as cluster batches (set at dem_create).
bool use_batches(const dem_ctx* c);
// Drops the adjoint's cached graphs (with the engine's: they hold its parameters).
void adjoint_drop_graphs(dem_ctx* c);
// The host copy of the particle order (c->hperm), fetched from the device
// (one copy and a stream wait) when an upload computed a new one.
int host_perm(dem_ctx* c);
template <typename Real> Planes3<Real> planes(void* base, long long npad) {
    Real* b = (Real*)base;
    return Planes3<Real>{b, b + npad, b + 2 * npad};
}
template <typename T> int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    DEM_CUDA_TRY(cudaMalloc((void**)p, count * sizeof(T)));
    return DEM_OK;
}
}  // namespace dem
