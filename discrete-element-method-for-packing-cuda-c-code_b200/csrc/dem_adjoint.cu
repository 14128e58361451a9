// dem_adjoint.cu -- reverse mode of the DEM step over a window of steps
// (force + walls + integrator), with checkpoints every K steps and
// recomputation in between.  No counterpart in the reference.
//
//   1. forward:  the engine runs the window; every K steps it saves a
//      checkpoint (state, wall history, and the previous list with its
//      tangential history, from which the next re-list carries).
//   2. objective at the final state: packing fraction
//      sum (4/3) pi r^3 / (Wx Wy max z) or potential energy
//      sum m z + sum (2/5) estar sqrt(R*) delta^2.5 (pairs and walls); its
//      gradient seeds the adjoint state.
//   3. for each segment, last first: restore the checkpoint, recompute the
//      segment (PCCP: re-list + window kernel per window, writing the tape of
//      the bound particles -- state, force, torque, wall and pair history --
//      and every re-list's list, carry map and bound/free lists; one CUDA
//      graph per segment); then sweep the steps backwards (one CUDA graph
//      per segment, on its own stream):
//        k_adj_free_window  free particles: the window's steps in closed form
//        k_adj_pairs + k_adj_bound  bound particles, per step: each listed
//                     pair's law reversed once, then each particle's
//                     integrator reverse with its pairs' shares in list
//                     order and its walls' VJP (dem_law_adj.cuh) -- no
//                     atomics, deterministic (k_adj_step: the same in one
//                     particle-parallel kernel, DEM_B200_ADJ=pp)
//        k_adj_carry  at a re-list, the history adjoints of the new list go
//                     back to the carried pairs of the previous list
//      Two tape sets: segment g-1 is recomputed into one while segment g is
//      reversed from the other.
// The reverse runs in FP64 on the recorded FP64/FP32 trajectory.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "dem_engine_internal.h"
#include "dem_law_adj.cuh"

namespace dem {

namespace {
constexpr int kB = 256;
constexpr int kPairB = 32;    // block size of k_adj_step; pbar holds one 12-slot row per block
constexpr int kAB = 128;      // block size of k_adj_pairs and k_adj_bound
constexpr int kPC = 20;       // doubles per pair of the two-phase reverse step's shares
constexpr long long kScatterPrime = 2654435761ll;

struct Ck {
    void* rec = nullptr;     // np particle records
    float4* q = nullptr;     // np
    double* wh = nullptr;    // 3 np
    uint* off = nullptr;     // np + 1 (previous list)
    uint* ln = nullptr;      // cap
    double* hist = nullptr;  // 3 cap
    int cur = 0, sbuf = 0, hph = 0;
};

struct ListRec {
    uint *off = nullptr, *ln = nullptr, *lp = nullptr, *roff = nullptr, *rk = nullptr, *carry = nullptr;
    uint* bflag = nullptr;   // bound (1) / free (0) particles of the window
    uint* blist = nullptr;   // bound particle ids (n)
    uint* flist = nullptr;   // free particle ids (n)
    uint* nb = nullptr;      // number of bound particles (device word)
};
}  // namespace

// Graphs of the adjoint, indexed by the tape set and the parities at the
// segment start (recompute: list buffer; reverse sweep: hb, in): a graph
// holds the set's addresses and the material.  Kept across calls of the same
// segment length; dropped with the engine's graphs (material, particle count,
// grid) and when the tape is reallocated.
struct SegmentGraphs {
    cudaGraphExec_t g[2][2][2] = {};
    void drop() {
        for (auto& set : g)
            for (auto& row : set)
                for (cudaGraphExec_t& e : row)
                    if (e) {
                        cudaGraphExecDestroy(e);
                        e = nullptr;
                    }
    }
    ~SegmentGraphs() { drop(); }
};

// The tape of one segment's recompute: per step the bound particles' state
// before the step, wall history, total force and torque, pair contacts and
// every listed pair's history; per window its list.
struct TapeSet {
    std::vector<ListRec> lists;
    double *tx = nullptr, *td = nullptr, *twh = nullptr, *tF = nullptr, *tT = nullptr, *th = nullptr;
    uint* tc = nullptr;   // per step and particle: its pair contacts in the forward
    void* ta = nullptr;
};

struct AdjWork {
    long long seg = 0, nck = 0, nwin = 0;
    std::vector<Ck> ck;
    // two tape sets: the recompute of segment g-1 (context stream) fills one
    // while the reverse of segment g (reverse stream) reads the other
    TapeSet set[2];
    cudaStream_t rs = nullptr;                       // the reverse sweep's stream
    cudaEvent_t filled[2] = {nullptr, nullptr};      // set k's recompute done
    cudaEvent_t freed[2] = {nullptr, nullptr};       // set k's reverse done
    cudaEvent_t joined = nullptr;
    SegmentGraphs fgraph, rgraph;    // recompute and reverse graphs
    long long graph_every = 0;       // the segment length they were captured for
    // the set selected for the code below (select_set)
    ListRec* lists = nullptr;
    double *tx = nullptr, *td = nullptr, *twh = nullptr, *tF = nullptr, *tT = nullptr, *th = nullptr;
    uint* tc = nullptr;
    void* ta = nullptr;
    // state adjoints, two sets (ping-pong per reversed step); the objective
    // seeds set 0 (Xb, Db, Ab alias it)
    double* Xb2[2] = {nullptr, nullptr};
    double* Db2[2] = {nullptr, nullptr};
    double* Ab2[2] = {nullptr, nullptr};
    double *Xb = nullptr, *Db = nullptr, *Ab = nullptr, *Wb = nullptr, *Rb = nullptr;
    double* Hb[2] = {nullptr, nullptr};
    double* pbar = nullptr;      // npb x 12 (one row per reverse-step block: pair params 0-5, wall params 6-11)
    double* PC = nullptr;        // kPC per pair slot: the shares a pair's reverse sends to lo and hi
    uint* pon = nullptr;         // per pair slot: 1 if PC holds this step's shares
    double* WS = nullptr;        // 10 per particle: its walls' shares (pair phase)
    uint* wson = nullptr;        // per particle: 1 if WS holds this step's shares
    unsigned grid_pairs = 1, grid_bound = 1;   // blocks of k_adj_pairs / k_adj_bound
    bool pair_parallel = true;   // two-phase reverse step (DEM_B200_ADJ=pp: k_adj_step)
    double* objp = nullptr;      // 3 per k_obj_potential block: energy, d/d estar (pair, wall)
    double* Pobj = nullptr;      // 3 np: the final positions for the objective
    long long npb = 0;
    double* obj = nullptr;       // [0] value, [1..] scratch
    unsigned long long* zmax = nullptr;  // [0] max z bits, [1] argmax
    unsigned long long* save_mz = nullptr;   // observables of the forward's last step
    uint* save_cnt = nullptr;
};

namespace {

void free_ck(Ck& k) {
    void* p[] = {k.rec, k.q, k.wh, k.off, k.ln, k.hist};
    for (void* x : p)
        if (x) cudaFree(x);
    k = Ck();
}

size_t rsz(const dem_ctx* c) { return c->prec == DEM_PREC_MIXED ? sizeof(float) : sizeof(double); }

void select_set(AdjWork* w, int k) {
    TapeSet& t = w->set[k];
    w->lists = t.lists.data();
    w->tx = t.tx; w->td = t.td; w->twh = t.twh; w->tF = t.tF; w->tT = t.tT; w->th = t.th; w->tc = t.tc; w->ta = t.ta;
}

void free_set(TapeSet& t) {
    void* p[] = {t.tx, t.td, t.twh, t.tF, t.tT, t.th, t.ta, t.tc};
    for (void* x : p)
        if (x) cudaFree(x);
    for (ListRec& l : t.lists) {
        void* q[] = {l.off, l.ln, l.lp, l.roff, l.rk, l.carry, l.bflag, l.blist, l.flist, l.nb};
        for (void* x : q)
            if (x) cudaFree(x);
    }
    t = TapeSet();
}
size_t recsz(const dem_ctx* c) { return c->prec == DEM_PREC_MIXED ? sizeof(PRec<float>) : sizeof(PRec<double>); }

int adj_grids(dem_ctx* c);

int ensure_work(dem_ctx* c, long long seg, long long nck) {
    AdjWork* w = c->adj;
    if (!w) {
        w = new AdjWork();
        c->adj = w;
    }
    const long long np = c->npad, cap = c->cap;
    const int K = c->cfg.relist_interval;
    int rc;
    if (!w->Xb) {
        if ((rc = dalloc(&w->Xb2[0], 3 * np)) || (rc = dalloc(&w->Db2[0], 3 * np)) ||
            (rc = dalloc(&w->Ab2[0], 3 * np)) || (rc = dalloc(&w->Xb2[1], 3 * np)) ||
            (rc = dalloc(&w->Db2[1], 3 * np)) || (rc = dalloc(&w->Ab2[1], 3 * np)) || (rc = dalloc(&w->Wb, 3 * np)) ||
            (rc = dalloc(&w->Rb, np)) || (rc = dalloc(&w->Hb[0], 3 * cap)) || (rc = dalloc(&w->Hb[1], 3 * cap)) ||
            (rc = dalloc(&w->obj, 16)) ||
            (rc = dalloc(&w->objp, 3 * (size_t)grid_for(c->n, kB))) ||
            (rc = dalloc(&w->zmax, 2)) ||
            (rc = dalloc(&w->save_mz, c->npart)) || (rc = dalloc(&w->save_cnt, c->npart)) ||
            (rc = dalloc(&w->Pobj, 3 * np)))
            return rc;
        const char* ap = getenv("DEM_B200_ADJ");   // "pp": the particle-parallel reverse step
        w->pair_parallel = !(ap && ap[0] == 'p');
        if ((rc = adj_grids(c))) return rc;
        w->npb = std::max<long long>(grid_for(c->n, kPairB), std::max(w->grid_pairs, w->grid_bound));
        if ((rc = dalloc(&w->pbar, (size_t)w->npb * 12))) return rc;
        if (w->pair_parallel && ((rc = dalloc(&w->PC, (size_t)kPC * cap)) || (rc = dalloc(&w->pon, cap)) ||
                                 (rc = dalloc(&w->WS, 10 * (size_t)np)) || (rc = dalloc(&w->wson, np))))
            return rc;
        w->Xb = w->Xb2[0];
        w->Db = w->Db2[0];
        w->Ab = w->Ab2[0];
    }
    if (!w->rs) {
        DEM_CUDA_TRY(cudaStreamCreateWithFlags(&w->rs, cudaStreamNonBlocking));
        for (int k = 0; k < 2; k++) {
            DEM_CUDA_TRY(cudaEventCreateWithFlags(&w->filled[k], cudaEventDisableTiming));
            DEM_CUDA_TRY(cudaEventCreateWithFlags(&w->freed[k], cudaEventDisableTiming));
        }
        DEM_CUDA_TRY(cudaEventCreateWithFlags(&w->joined, cudaEventDisableTiming));
    }
    if (seg > w->seg) {
        cudaStreamSynchronize(w->rs);
        w->fgraph.drop();
        w->rgraph.drop();
        const long long nw = (seg + K - 1) / K;
        for (TapeSet& t : w->set) {
            free_set(t);
            if ((rc = dalloc(&t.tx, 3 * np * seg)) || (rc = dalloc(&t.td, 3 * np * seg)) ||
                (rc = dalloc(&t.twh, 3 * np * seg)) || (rc = dalloc(&t.tF, 3 * np * seg)) ||
                (rc = dalloc(&t.tT, 3 * np * seg)) || (rc = dalloc(&t.th, 3 * cap * seg)) ||
                (rc = dalloc(&t.tc, np * seg)))
                return rc;
            DEM_CUDA_TRY(cudaMalloc(&t.ta, 3 * np * seg * rsz(c)));
            t.lists.resize(nw);
            for (ListRec& l : t.lists)
                if ((rc = dalloc(&l.off, np + 1)) || (rc = dalloc(&l.ln, cap)) || (rc = dalloc(&l.lp, cap)) ||
                    (rc = dalloc(&l.roff, np + 1)) || (rc = dalloc(&l.rk, cap)) || (rc = dalloc(&l.carry, cap)) ||
                    (rc = dalloc(&l.bflag, np)) || (rc = dalloc(&l.blist, np)) || (rc = dalloc(&l.flist, np)) ||
                    (rc = dalloc(&l.nb, 1)))
                    return rc;
        }
        w->seg = seg;
        w->nwin = nw;
    }
    if (nck > (long long)w->ck.size()) {
        size_t old = w->ck.size();
        w->ck.resize(nck);
        for (size_t k = old; k < (size_t)nck; k++) {
            Ck& x = w->ck[k];
            if ((rc = dalloc(&x.q, np)) || (rc = dalloc(&x.wh, 3 * np)) || (rc = dalloc(&x.off, np + 1)) ||
                (rc = dalloc(&x.ln, cap)) || (rc = dalloc(&x.hist, 3 * cap)))
                return rc;
            DEM_CUDA_TRY(cudaMalloc(&x.rec, np * recsz(c)));
        }
    }
    w->nck = nck;
    return DEM_OK;
}

int copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes) DEM_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    return DEM_OK;
}

// Checkpoint = state of the current buffers + the previous list (the one the
// next re-list carries history from).
int save_ck(dem_ctx* c, Ck& k) {
    const long long np = c->npad, cap = c->cap;
    cudaStream_t s = c->stream;
    int rc;
    if ((rc = copy(k.rec, c->rec[c->sbuf], np * recsz(c), s)) || (rc = copy(k.q, c->q, np * sizeof(float4), s)) ||
        (rc = copy(k.wh, c->wh, 3 * np * sizeof(double), s)) ||
        (rc = copy(k.off, c->off[c->cur], (np + 1) * sizeof(uint), s)) ||
        (rc = copy(k.ln, c->ln[c->cur], cap * sizeof(uint), s)) ||
        (rc = copy(k.hist, c->hist[c->cur][c->hph], 3 * cap * sizeof(double), s)))
        return rc;
    k.cur = c->cur;
    k.sbuf = c->sbuf;
    k.hph = c->hph;
    return DEM_OK;
}

int restore_ck(dem_ctx* c, const Ck& k) {
    const long long np = c->npad, cap = c->cap;
    cudaStream_t s = c->stream;
    c->cur = k.cur;
    c->sbuf = k.sbuf;
    c->hph = k.hph;
    int rc;
    if ((rc = copy(c->rec[c->sbuf], k.rec, np * recsz(c), s)) || (rc = copy(c->q, k.q, np * sizeof(float4), s)) ||
        (rc = copy(c->wh, k.wh, 3 * np * sizeof(double), s)) ||
        (rc = copy(c->off[c->cur], k.off, (np + 1) * sizeof(uint), s)) ||
        (rc = copy(c->ln[c->cur], k.ln, cap * sizeof(uint), s)) ||
        (rc = copy(c->hist[c->cur][c->hph], k.hist, 3 * cap * sizeof(double), s)))
        return rc;
    return DEM_OK;
}

// ------------------------------------------------------------- kernels
template <typename Real> __device__ __forceinline__ V3d ldA(const Real* a, long long np, long long i) {
    return mk((double)a[i], (double)a[np + i], (double)a[2 * np + i]);
}
__device__ __forceinline__ V3d ld3(const double* a, long long np, long long i) {
    return mk(a[i], a[np + i], a[2 * np + i]);
}
__device__ __forceinline__ void st3(double* a, long long np, long long i, V3d v) {
    a[i] = v.x; a[np + i] = v.y; a[2 * np + i] = v.z;
}

// Integrator reverse of particle i (neiglist.cu:356-360 read backwards):
//   d' = d + F dt^2/m,  x' = x + d',  a' = a + T dt^2/I,  F_z includes -m.
// Given the step's taped total force f and torque t and the adjoints (xb,
// db, ab) of the state after the step, returns the adjoint of d' (dtot = db +
// xb) and of the step's force and torque, and adds the mass / inertia terms
// to the radius adjoint.
template <typename Real>
__device__ __forceinline__ void integ_rev(Real rr, V3d f, V3d t, double dt, double density, V3d xb, V3d db, V3d ab,
                                          V3d& dtot, V3d& fb, V3d& tb, double& rb) {
    const double r = (double)rr;
    const double m = density * 8.0 * r * r * r, I = 0.4 * m * (r * r);
    const double dmdr = density * 24.0 * r * r, dIdr = 0.4 * (dmdr * r * r + 2.0 * m * r);
    dtot = db + xb;
    const double k = dt * dt / m, kI = dt * dt / I;
    fb = k * dtot;
    tb = kI * ab;
    double mb = -dot(dtot, f) * k / m;   // d/dm of F dt^2/m
    mb += -fb.z;                          // gravity F_z = ... - m
    const double Ib = -dot(ab, t) * kI / I;
    rb += mb * dmdr + Ib * dIdr;
}

// Force / torque adjoints of partner j from the after-step adjoints (the
// first half of integ_rev, no side effects).
template <typename Real>
__device__ __forceinline__ void partner_fb(Real rr, long long np, long long j, double dt, double density,
                                           const double* __restrict__ Xa, const double* __restrict__ Da,
                                           const double* __restrict__ Aa, V3d& fb, V3d& tb) {
    const double r = (double)rr;
    const double m = density * 8.0 * r * r * r, I = 0.4 * m * (r * r);
    fb = (dt * dt / m) * (ld3(Da, np, j) + ld3(Xa, np, j));
    tb = (dt * dt / I) * ld3(Aa, np, j);
}

struct AdjList {
    const uint *off, *ln, *lp, *roff, *rk;
};

// The window's free particles (flist[t], t < n - nb), all K steps of the
// window reversed at once.  A free particle feels its weight only: per step
// d' = d - g dt^2 and x' = x + d', so the reverse keeps the position and
// rotation adjoints and adds the position adjoint to the displacement adjoint
// once per step (d_bar += K x_bar); no parameter or radius depends on it
// (F/m = -g) and its wall-history adjoint is zero.  No bound particle reads a
// free particle's adjoints inside the window, so they are read from set `in`
// at the window's end and written to the set current after its K reversed
// steps.
__global__ void k_adj_free_window(long long n, long long np, int K, const uint* __restrict__ flist,
                                  const uint* __restrict__ nbp, const double* Xi, const double* Di, const double* Ai,
                                  double* Xo, double* Do, double* Ao, double* __restrict__ Wb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n - (long long)*nbp) return;
    const long long i = flist[t];
    const V3d xb = ld3(Xi, np, i), db = ld3(Di, np, i), ab = ld3(Ai, np, i);
    st3(Xo, np, i, xb);
    st3(Do, np, i, db + (double)K * xb);
    st3(Ao, np, i, ab);
    st3(Wb, np, i, zero3<double>());
}

// One reversed step of the window's bound particles (blist[u], u < nb),
// particle-parallel: the integrator reverse of particle i, then every pair it
// belongs to and its walls, evaluated forward with tape and reversed; each
// particle keeps its own share of the input adjoints, the pair's history
// adjoint and its parameter adjoints are kept by the lower index only.  State
// adjoints ping-pong: (Xa, Da, Aa) after the step are read (also for the
// partners' force adjoints), (Xo, Do, Ao) before the step are written; no
// atomics, deterministic.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// L2 prefetch of partner j's taped state and radius and of pair k's history.
template <typename Real>
__device__ __forceinline__ void prefetch_partner(uint j, uint k, long long np, long long cap,
                                                 const double* __restrict__ tx, const double* __restrict__ td,
                                                 const Real* __restrict__ ta, const double* __restrict__ th,
                                                 const Real* __restrict__ R) {
    for (int c = 0; c < 3; c++) {
        prefetch_l2(tx + c * np + j);
        prefetch_l2(td + c * np + j);
        prefetch_l2(ta + c * np + j);
        prefetch_l2(th + c * cap + k);
    }
    prefetch_l2(R + j);
}

template <typename Real>
__global__ void __launch_bounds__(kPairB) k_adj_step(
    long long n, long long np, long long cap, AdjList L, const uint* __restrict__ blist, const uint* __restrict__ nbp,
    const double* __restrict__ tx, const double* __restrict__ td, const Real* __restrict__ ta,
    const double* __restrict__ twh, const double* __restrict__ th, const double* __restrict__ tF,
    const double* __restrict__ tT, const uint* __restrict__ tc, const Real* __restrict__ R, LawParams<double> pp,
    LawParams<double> pw,
    double dt, double density, double hx, double hy, const double* __restrict__ Hout, double* __restrict__ Hin,
    const double* __restrict__ Xa, const double* __restrict__ Da, const double* __restrict__ Aa,
    double* __restrict__ Xo, double* __restrict__ Do, double* __restrict__ Ao, double* __restrict__ Wb,
    double* __restrict__ Rb, double* __restrict__ pbar) {
    __shared__ double sp[12][kPairB / 32];
    const double inv_dt = 1.0 / dt;
    const long long u0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nb = (long long)*nbp;
    LawBar bp, bw;
    lawbar_zero(bp);
    lawbar_zero(bw);
    // Before pdl_wait: what the recompute wrote (list, tape) -- the particle,
    // its taped state, force, torque, wall history and pair-contact count,
    // and its row bounds.  The previous reversed step (the predecessor)
    // writes only adjoints, and it triggers this launch only after its own
    // wait, so everything older than it is complete.
    // Bound particles in a scattered order (u0 -> u0 * p mod nb, p a prime
    // above any particle count: a bijection): with the particles stored in
    // cell order, neighbours with many contacts -- long FP64 chains -- would
    // otherwise fill the same warps (measured: 25 % longer reverse sweeps);
    // scattered, every warp gets a mix.
    long long i = 0;
    Real rr = (Real)0;
    V3d xi = zero3<double>(), di = zero3<double>(), ai = zero3<double>(), fi = zero3<double>(), ti = zero3<double>(),
        hw = zero3<double>();
    uint total = 0, o0 = 0, o1 = 0, q0 = 0, q1 = 0, nc = 0;
    if (u0 < nb) {
        i = blist[(u0 * kScatterPrime) % nb];
        rr = R[i];
        xi = ld3(tx, np, i); di = ld3(td, np, i); ai = ldA<Real>(ta, np, i);
        fi = mk(tF[3 * i], tF[3 * i + 1], tF[3 * i + 2]);
        ti = mk(tT[3 * i], tT[3 * i + 1], tT[3 * i + 2]);
        hw = ld3(twh, np, i);
        nc = tc[i];
        total = L.off[n];
        o0 = L.off[i]; o1 = L.off[i + 1]; q0 = L.roff[i]; q1 = L.roff[i + 1];
        if (nc != 0 && (long long)total <= cap) {
            // a sphere in contact: the first partner of each row has its taped
            // state and the pair's history brought into L2 while the
            // predecessor finishes (tape data only; no registers held)
            if (o1 > o0) prefetch_partner(L.ln[o0], o0, np, cap, tx, td, ta, th, R);
            if (q1 > q0) {
                const uint k = L.rk[q0];
                if (k < total) prefetch_partner(L.lp[k], k, np, cap, tx, td, ta, th, R);
            }
        }
    }
    pdl_wait();
    pdl_trigger();
    if (u0 < nb) {
        const V3d xa = ld3(Xa, np, i), aa = ld3(Aa, np, i);
        V3d dtot, fbi, tbi;
        double rb = 0.0;
        integ_rev<Real>(rr, fi, ti, dt, density, xa, ld3(Da, np, i), aa, dtot, fbi, tbi, rb);
        V3d xb = zero3<double>(), dbv = zero3<double>(), ab = zero3<double>();
        const double ri = (double)rr;
        double dum = 0.0;
        if ((long long)total <= cap && nc == 0) {
            // no pair contact in the forward step: every listed pair of the
            // sphere was inert (zero force, history reset), so only the
            // history adjoints of its own row are cleared; no partner is read
            for (uint k = o0; k < o1; k++) { Hin[k] = 0.0; Hin[cap + k] = 0.0; Hin[2 * cap + k] = 0.0; }
        } else if ((long long)total <= cap) {
            for (uint k = o0; k < o1; k++) {
                const uint j = L.ln[k];
                const V3d hin = mk(th[k], th[cap + k], th[2 * cap + k]);
                PairTape t;
                V3d Fi, Ti, Tj, ho;
                if (!pair_fwd(xi, ld3(tx, np, j), di, ld3(td, np, j), ai, ldA<Real>(ta, np, j), ri, (double)R[j], hin,
                              pp, inv_dt, density, t, Fi, Ti, Tj, ho)) {
                    Hin[k] = 0.0; Hin[cap + k] = 0.0; Hin[2 * cap + k] = 0.0;
                    continue;
                }
                V3d fbj, tbj;
                partner_fb<Real>(R[j], np, j, dt, density, Xa, Da, Aa, fbj, tbj);
                V3d hinb = zero3<double>(), xjb = zero3<double>(), djb = zero3<double>(), ajb = zero3<double>();
                pair_rev(t, pp, inv_dt, density, fbi - fbj, tbi, tbj, mk(Hout[k], Hout[cap + k], Hout[2 * cap + k]), xb,
                         xjb, dbv, djb, ab, ajb, rb, dum, hinb, bp);
                Hin[k] = hinb.x; Hin[cap + k] = hinb.y; Hin[2 * cap + k] = hinb.z;
            }
            for (uint u = q0; u < q1; u++) {
                const uint k = L.rk[u];
                if (k >= total) continue;
                const uint j = L.lp[k];
                const V3d hin = mk(th[k], th[cap + k], th[2 * cap + k]);
                PairTape t;
                V3d Fi, Ti, Tj, ho;
                if (!pair_fwd(ld3(tx, np, j), xi, ld3(td, np, j), di, ldA<Real>(ta, np, j), ai, (double)R[j], ri, hin,
                              pp, inv_dt, density, t, Fi, Ti, Tj, ho))
                    continue;
                V3d fbj, tbj;
                partner_fb<Real>(R[j], np, j, dt, density, Xa, Da, Aa, fbj, tbj);
                LawBar scratch;
                lawbar_zero(scratch);
                V3d hinb = zero3<double>(), xlb = zero3<double>(), dlb = zero3<double>(), alb = zero3<double>();
                pair_rev(t, pp, inv_dt, density, fbj - fbi, tbj, tbi, mk(Hout[k], Hout[cap + k], Hout[2 * cap + k]),
                         xlb, xb, dlb, dbv, alb, ab, dum, rb, hinb, scratch);
            }
        }
        // walls (the stored slot is the history input; it is zero whenever
        // the particle did not touch a wall at the previous step)
        V3d hwb = zero3<double>();
        wall_vjp(hx, hy, xi, di, ai, ri, density, hw, pw, inv_dt, fbi, tbi, ld3(Wb, np, i), xb, dbv, ab, rb, hwb, bw);
        st3(Wb, np, i, hwb);
        st3(Xo, np, i, xa + xb);
        st3(Do, np, i, dtot + dbv);
        st3(Ao, np, i, aa + ab);
        Rb[i] += rb;
    }
    // parameter adjoints: block sums accumulated into this block's slot
    double v[12] = {bp.estar, bp.mu, bp.cn, bp.ct, bp.roll, bp.roll_rel,
                    bw.estar, bw.mu, bw.cn, bw.ct, bw.roll, bw.roll_rel};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sp[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) x += sp[threadIdx.x][w];
        pbar[(size_t)blockIdx.x * 12 + threadIdx.x] += x;
    }
}

// One reversed step of the bound particles in two pair-parallel phases (the
// default; k_adj_step above is the particle-parallel form, DEM_B200_ADJ=pp).
//
// Phase A (k_adj_pairs), one thread per listed pair (lo, hi): the pair law is
// evaluated forward from the tape and reversed once, with the force adjoint
// of each side taken from the after-step state adjoints (the first half of
// the integrator reverse); the pair's input-history adjoint goes to Hin, its
// parameter adjoints into this block's row of pbar (slots 0-5), and the
// adjoints it sends to lo and hi into PC (kPC doubles per pair: lo's x, d, a
// and radius, then hi's), with pon[k] = 1.  A pair whose two spheres had no
// pair contact in the forward step (taped count 0 on either side) only clears
// its history adjoint.  Phase B (k_adj_bound), one thread per bound particle:
// the integrator reverse, the sum of its pairs' shares (own row, then reverse
// row, in list order: deterministic), the walls (parameter adjoints into
// slots 6-11 of its block's row), and the state adjoints before the step.
// The chain of one thread is one pair's law instead of all of a sphere's
// pairs twice over; no atomics.
__device__ __forceinline__ void block_sum6(const double v[6], double* row) {
    __shared__ double sp[6][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sp[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) x += sp[threadIdx.x][w];
        row[threadIdx.x] += x;
    }
    __syncthreads();   // sp may be reused by the next call
}

template <typename Real>
__global__ void __launch_bounds__(kAB) k_adj_pairs(
    long long n, long long np, long long cap, AdjList L, const double* __restrict__ tx, const double* __restrict__ td,
    const Real* __restrict__ ta, const double* __restrict__ th, const uint* __restrict__ tc, const Real* __restrict__ R,
    LawParams<double> pp, double dt, double density, const double* __restrict__ Hout, double* __restrict__ Hin,
    const double* __restrict__ Xa, const double* __restrict__ Da, const double* __restrict__ Aa,
    double* __restrict__ PC, uint* __restrict__ pon, double* __restrict__ pbar, const uint* __restrict__ blist,
    const uint* __restrict__ nbp, const double* __restrict__ twh, LawParams<double> pw, double hx, double hy,
    double* __restrict__ WS, uint* __restrict__ wson, double* __restrict__ Wb) {
    const double inv_dt = 1.0 / dt;
    LawBar bp, bw;
    lawbar_zero(bp);
    lawbar_zero(bw);
    // the list and the tape (the recompute's) may be read before the wait;
    // the state and history adjoints are the predecessors'
    const uint total = L.off[n];
    const long long nb = (long long)*nbp;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long npr = (long long)total <= cap ? (long long)total : 0ll;
    pdl_wait();
    pdl_trigger();
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < npr + nb; k += stride) {
        if (k >= npr) {
            // a bound particle's walls: their VJP needs only the particle's
            // force adjoints, so it runs beside the pairs; its shares go to
            // WS for the particle phase, its history adjoint to Wb
            const uint i = blist[k - npr];
            V3d fbi, tbi;
            partner_fb<Real>(R[i], np, i, dt, density, Xa, Da, Aa, fbi, tbi);
            V3d xw = zero3<double>(), dw = zero3<double>(), aw = zero3<double>(), hwb = zero3<double>();
            double rw = 0.0;
            const int hit = wall_vjp(hx, hy, ld3(tx, np, i), ld3(td, np, i), ldA<Real>(ta, np, i), (double)R[i],
                                     density, ld3(twh, np, i), pw, inv_dt, fbi, tbi, ld3(Wb, np, i), xw, dw, aw, rw,
                                     hwb, bw);
            st3(Wb, np, i, hwb);
            if (hit) {
                double* c = WS + 10 * (size_t)i;
                c[0] = xw.x; c[1] = xw.y; c[2] = xw.z; c[3] = dw.x; c[4] = dw.y; c[5] = dw.z;
                c[6] = aw.x; c[7] = aw.y; c[8] = aw.z; c[9] = rw;
            }
            wson[i] = hit ? 1u : 0u;
            continue;
        }
        {
            const uint lo = L.lp[k], hi = L.ln[k];
            bool on = tc[lo] != 0 && tc[hi] != 0;
            PairTape t;
            if (on) {
                const V3d hin = mk(th[k], th[cap + k], th[2 * cap + k]);
                V3d Fi, Ti, Tj, ho;
                on = pair_fwd(ld3(tx, np, lo), ld3(tx, np, hi), ld3(td, np, lo), ld3(td, np, hi), ldA<Real>(ta, np, lo),
                              ldA<Real>(ta, np, hi), (double)R[lo], (double)R[hi], hin, pp, inv_dt, density, t, Fi,
                              Ti, Tj, ho) != 0;
            }
            if (!on) {
                Hin[k] = 0.0; Hin[cap + k] = 0.0; Hin[2 * cap + k] = 0.0;
                pon[k] = 0u;
                continue;
            }
            V3d fbl, tbl, fbh, tbh;
            partner_fb<Real>(R[lo], np, lo, dt, density, Xa, Da, Aa, fbl, tbl);
            partner_fb<Real>(R[hi], np, hi, dt, density, Xa, Da, Aa, fbh, tbh);
            V3d xl = zero3<double>(), xh = zero3<double>(), dl = zero3<double>(), dh = zero3<double>(),
                al = zero3<double>(), ah = zero3<double>(), hinb = zero3<double>();
            double rl = 0.0, rh = 0.0;
            pair_rev(t, pp, inv_dt, density, fbl - fbh, tbl, tbh, mk(Hout[k], Hout[cap + k], Hout[2 * cap + k]), xl, xh,
                     dl, dh, al, ah, rl, rh, hinb, bp);
            Hin[k] = hinb.x; Hin[cap + k] = hinb.y; Hin[2 * cap + k] = hinb.z;
            double* c = PC + (size_t)kPC * k;
            c[0] = xl.x; c[1] = xl.y; c[2] = xl.z; c[3] = dl.x; c[4] = dl.y; c[5] = dl.z;
            c[6] = al.x; c[7] = al.y; c[8] = al.z; c[9] = rl;
            c[10] = xh.x; c[11] = xh.y; c[12] = xh.z; c[13] = dh.x; c[14] = dh.y; c[15] = dh.z;
            c[16] = ah.x; c[17] = ah.y; c[18] = ah.z; c[19] = rh;
            pon[k] = 1u;
        }
    }
    const double v[6] = {bp.estar, bp.mu, bp.cn, bp.ct, bp.roll, bp.roll_rel};
    block_sum6(v, pbar + (size_t)blockIdx.x * 12);
    const double vw[6] = {bw.estar, bw.mu, bw.cn, bw.ct, bw.roll, bw.roll_rel};
    block_sum6(vw, pbar + (size_t)blockIdx.x * 12 + 6);
}

__device__ __forceinline__ void add_share(const double* __restrict__ c, V3d& xb, V3d& db, V3d& ab, double& rb) {
    xb += mk(c[0], c[1], c[2]);
    db += mk(c[3], c[4], c[5]);
    ab += mk(c[6], c[7], c[8]);
    rb += c[9];
}

template <typename Real>
__global__ void __launch_bounds__(kAB) k_adj_bound(
    long long n, long long np, long long cap, AdjList L, const uint* __restrict__ blist, const uint* __restrict__ nbp,
    const double* __restrict__ tF, const double* __restrict__ tT, const Real* __restrict__ R, double dt,
    double density, const double* __restrict__ PC, const uint* __restrict__ pon, const double* __restrict__ WS,
    const uint* __restrict__ wson, const double* __restrict__ Xa, const double* __restrict__ Da,
    const double* __restrict__ Aa, double* __restrict__ Xo, double* __restrict__ Do, double* __restrict__ Ao,
    double* __restrict__ Rb) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nb = (long long)*nbp;
    const uint total = L.off[n];
    // the list and the tape of a particle (the first one before the wait)
    long long i = 0;
    Real rr = (Real)0;
    V3d fi, ti;
    uint o0 = 0, o1 = 0, q0 = 0, q1 = 0;
    auto load = [&]() {
        i = blist[u];
        rr = R[i];
        fi = mk(tF[3 * i], tF[3 * i + 1], tF[3 * i + 2]);
        ti = mk(tT[3 * i], tT[3 * i + 1], tT[3 * i + 2]);
        o0 = L.off[i]; o1 = L.off[i + 1]; q0 = L.roff[i]; q1 = L.roff[i + 1];
    };
    if (u < nb) load();
    pdl_wait();
    pdl_trigger();
    for (bool first = true; u < nb; u += stride, first = false) {
        if (!first) load();
        const V3d xa = ld3(Xa, np, i), aa = ld3(Aa, np, i);
        V3d dtot, fbi, tbi;
        double rb = 0.0;
        integ_rev<Real>(rr, fi, ti, dt, density, xa, ld3(Da, np, i), aa, dtot, fbi, tbi, rb);
        V3d xb = zero3<double>(), dbv = zero3<double>(), ab = zero3<double>();
        if ((long long)total <= cap) {
            for (uint k = o0; k < o1; k++)
                if (pon[k]) add_share(PC + (size_t)kPC * k, xb, dbv, ab, rb);
            for (uint q = q0; q < q1; q++) {
                const uint k = L.rk[q];
                if (k < total && pon[k]) add_share(PC + (size_t)kPC * k + 10, xb, dbv, ab, rb);
            }
        }
        if (wson[i]) add_share(WS + 10 * (size_t)i, xb, dbv, ab, rb);   // its walls (the pair phase's items)
        st3(Xo, np, i, xa + xb);
        st3(Do, np, i, dtot + dbv);
        st3(Ao, np, i, aa + ab);
        Rb[i] += rb;
    }
}

// Grids of the two-phase reverse step: one round of resident blocks,
// striding over the pairs / bound particles (a grid sized for the capacity
// is mostly blocks without work, each of which still takes a slot on an SM
// every step).
int adj_grids(dem_ctx* c) {
    AdjWork* w = c->adj;
    const bool mx = c->prec == DEM_PREC_MIXED;
    int nsm = 0, bp = 0, bb = 0;
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    if (e == cudaSuccess)
        e = mx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bp, k_adj_pairs<float>, kAB, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bp, k_adj_pairs<double>, kAB, 0);
    if (e == cudaSuccess)
        e = mx ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, k_adj_bound<float>, kAB, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bb, k_adj_bound<double>, kAB, 0);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint kernel set-up", __FILE__, __LINE__);
    w->grid_pairs = (unsigned)std::max(1, nsm * std::max(bp, 1));
    w->grid_bound = (unsigned)std::max(1, nsm * std::max(bb, 1));
    return DEM_OK;
}

// History adjoint across a re-list: new pair k carried old pair carry[k].
__global__ void k_adj_carry(const uint* __restrict__ off, long long n, long long cap, const uint* __restrict__ carry,
                            const double* __restrict__ Hnew, double* __restrict__ Hold) {
    const uint total = off[n];
    if ((long long)total > cap) return;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < (long long)total;
         k += (long long)gridDim.x * blockDim.x) {
        const uint t = carry[k];
        if (t == kEmpty || (long long)t >= cap) continue;
        Hold[t] = Hnew[k];
        Hold[cap + t] = Hnew[cap + k];
        Hold[2 * cap + t] = Hnew[2 * cap + k];
    }
}

// Records the input of one recomputed step: state planes, wall history and
// the pair history of the current list (count read on the device).
template <typename Real>
__global__ void k_tape(long long n, long long np, long long cap, const PRec<Real>* __restrict__ S,
                       const double* __restrict__ W, const uint* __restrict__ off, const double* __restrict__ H,
                       double* __restrict__ tx, double* __restrict__ td, Real* __restrict__ ta,
                       double* __restrict__ twh, double* __restrict__ th) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long i = t0; i < np; i += stride) {
        V3<double> x, d;
        V3<Real> a;
        Real r;
        ld_rec<false>(S + i, x, d, a, r);
        st3(tx, np, i, x);
        st3(td, np, i, d);
        ta[i] = a.x; ta[np + i] = a.y; ta[2 * np + i] = a.z;
    }
    for (long long k = t0; k < 3 * np; k += stride) twh[k] = W[k];
    long long total = off[n];
    if (total > cap) total = cap;
    for (long long k = t0; k < total; k += stride) {
        th[k] = H[k];
        th[cap + k] = H[cap + k];
        th[2 * cap + k] = H[2 * cap + k];
    }
}

// ------------------------------------------------------------ objectives
template <typename Real>
__global__ void k_zmax(long long n, const double* __restrict__ Z, unsigned long long* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double z = i < n ? Z[i] : 0.0;
    unsigned long long b = (unsigned long long)__double_as_longlong(z > 0.0 ? z : 0.0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
        b = ob > b ? ob : b;
    }
    if ((threadIdx.x & 31) == 0 && b) atomicMax(out, b);
}
__global__ void k_zargmax(long long n, const double* __restrict__ Z, unsigned long long* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double z = Z[i];
    unsigned long long b = (unsigned long long)__double_as_longlong(z > 0.0 ? z : 0.0);
    if (b == out[0]) atomicMin(&out[1], (unsigned long long)i);
}

// Packing fraction phi = Vs / (Wx Wy H): dphi/dz_argmax = -phi/H,
// dphi/dr_i = 4 pi r_i^2 / (Wx Wy H).
template <typename Real>
__global__ void k_obj_packing(long long n, long long np, const Real* __restrict__ R, double area, double vs,
                              const unsigned long long* zm, double* Xb, double* Rb, double* obj) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double H;
    memcpy(&H, &zm[0], sizeof(double));
    if (!(H > 0.0)) return;
    const double phi = vs / (area * H);
    const double r = (double)R[i];
    Rb[i] += 4.0 * M_PI * r * r / (area * H);
    if ((unsigned long long)i == zm[1]) {
        Xb[2 * np + i] += -phi / H;
        obj[0] = phi;
    }
}

// Potential energy sum m z + elastic (2/5) estar sqrt(R*) delta^2.5 of pairs
// and walls at the final state; gradient into Xb, Rb and estar adjoints.
template <typename Real>
__global__ void k_obj_potential(long long n, long long np, long long cap, AdjList L, const double* __restrict__ P,
                                const Real* __restrict__ R, double estar, double estar_w, double density, double hx,
                                double hy, double* Xb, double* Rb, double* part) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double U = 0.0, eb = 0.0, ebw = 0.0;
    if (i < n) {
        const V3d x = ld3(P, np, i);
        const double r = (double)R[i];
        const double m = density * 8.0 * r * r * r;
        U += m * x.z;
        V3d xb = mk(0.0, 0.0, m);
        double rb = density * 24.0 * r * r * x.z;
        // walls
        double dl[5] = {r - x.z, r - (x.x + hx), r - (hx - x.x), r - (x.y + hy), r - (hy - x.y)};
        for (int w = 0; w < 5; w++) {
            if (!(dl[w] > 0.0)) continue;
            const double d = dl[w], sr = sqrt(r), d15 = d * sqrt(d), d25 = d * d15;
            U += 0.4 * estar_w * sr * d25;
            const double fne = estar_w * sr * d15;
            xb += fne * wall_normal(w);
            rb += fne + 0.4 * estar_w * d25 / (2.0 * sr);
            ebw += 0.4 * sr * d25;
        }
        const uint total = L.off[n];
        if ((long long)total <= cap) {
            for (int side = 0; side < 2; side++) {
                const uint b = side ? L.roff[i] : L.off[i], e = side ? L.roff[i + 1] : L.off[i + 1];
                for (uint u = b; u < e; u++) {
                    const uint k = side ? L.rk[u] : u;
                    if (k >= total) continue;
                    const uint j = side ? L.lp[k] : L.ln[k];
                    const V3d xj = ld3(P, np, j);
                    const double rj = (double)R[j];
                    const V3d D = xj - x;
                    const double dist = sqrt(dot(D, D));
                    const double d = (r + rj) - dist;
                    if (!(d > 0.0 && dist > 0.0)) continue;
                    const double Rs = r * rj / (r + rj), sR = sqrt(Rs), d15 = d * sqrt(d), d25 = d * d15;
                    const double fne = estar * sR * d15;
                    xb += (fne / dist) * D;                       // d delta / d x_i = n
                    const double dRdr = rj * rj / ((r + rj) * (r + rj));
                    rb += fne + 0.4 * estar * d25 * dRdr / (2.0 * sR);
                    if (!side) {                                   // counted once, by the lower index
                        U += 0.4 * estar * sR * d25;
                        eb += 0.4 * sR * d25;
                    }
                }
            }
        }
        st3(Xb, np, i, ld3(Xb, np, i) + xb);
        Rb[i] += rb;
    }
    // block sums in a fixed order (no atomics: the same bits on every run),
    // summed over the blocks on the host
    __shared__ double sw[3][kB / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        U += __shfl_xor_sync(0xffffffffu, U, o);
        eb += __shfl_xor_sync(0xffffffffu, eb, o);
        ebw += __shfl_xor_sync(0xffffffffu, ebw, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sw[0][warp] = U; sw[1][warp] = eb; sw[2][warp] = ebw; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double x = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sw[threadIdx.x][q];
        part[3 * (size_t)blockIdx.x + threadIdx.x] = x;
    }
}

// Reversed step t of the segment for the bound particles: state adjoints
// read from set `in` (after the step), written to set 1 - in (before it).
template <typename Real> int adj_step(dem_ctx* c, long long t, const ListRec& l, int hb, int in) {
    AdjWork* w = c->adj;
    const long long np = c->npad, cap = c->cap;
    AdjList L{l.off, l.ln, l.lp, l.roff, l.rk};
    if (w->pair_parallel) {
        // both phases programmatic: each waits for its predecessor before it
        // reads an adjoint (tape and list loads overlap the predecessor's tail)
        const bool pdl = c->pdl;
        const double* tx = w->tx + 3 * np * t;
        const double* td = w->td + 3 * np * t;
        const Real* ta = (const Real*)w->ta + 3 * np * t;
        DEM_CUDA_TRY(launch_ex(k_adj_pairs<Real>, w->grid_pairs, kAB, w->rs, pdl, c->n, np, cap, L, tx, td, ta,
                               (const double*)w->th + 3 * cap * t, (const uint*)w->tc + np * t, (const Real*)c->rad,
                               make_law<double>(c->mat.pp), c->cfg.dt, c->cfg.density, (const double*)w->Hb[hb],
                               w->Hb[1 - hb], (const double*)w->Xb2[in], (const double*)w->Db2[in],
                               (const double*)w->Ab2[in], w->PC, w->pon, w->pbar, l.blist, l.nb,
                               (const double*)w->twh + 3 * np * t, make_law<double>(c->mat.pw), c->cfg.world[0] * 0.5,
                               c->cfg.world[1] * 0.5, w->WS, w->wson, w->Wb));
        DEM_CUDA_TRY(launch_ex(k_adj_bound<Real>, w->grid_bound, kAB, w->rs, pdl, c->n, np, cap, L, l.blist, l.nb,
                               (const double*)w->tF + 3 * np * t, (const double*)w->tT + 3 * np * t,
                               (const Real*)c->rad, c->cfg.dt, c->cfg.density, (const double*)w->PC,
                               (const uint*)w->pon, (const double*)w->WS, (const uint*)w->wson,
                               (const double*)w->Xb2[in], (const double*)w->Db2[in], (const double*)w->Ab2[in],
                               w->Xb2[1 - in], w->Db2[1 - in], w->Ab2[1 - in], w->Rb));
        return DEM_OK;
    }
    // a reversed step that directly follows another is launched programmatic
    // (its tape loads overlap the predecessor's tail); the first step of a
    // window follows the free-particle kernel and is launched plainly
    const bool pdl = c->pdl && (t % c->cfg.relist_interval) != c->cfg.relist_interval - 1;
    DEM_CUDA_TRY(launch_ex(
        k_adj_step<Real>, (unsigned)w->npb, kPairB, w->rs, pdl, c->n, np, cap, L, l.blist, l.nb,
        w->tx + 3 * np * t, w->td + 3 * np * t, (const Real*)w->ta + 3 * np * t, w->twh + 3 * np * t,
        w->th + 3 * cap * t, w->tF + 3 * np * t, w->tT + 3 * np * t, (const uint*)w->tc + np * t, (const Real*)c->rad,
        make_law<double>(c->mat.pp), make_law<double>(c->mat.pw), c->cfg.dt, c->cfg.density, c->cfg.world[0] * 0.5,
        c->cfg.world[1] * 0.5, (const double*)w->Hb[hb], w->Hb[1 - hb], (const double*)w->Xb2[in],
        (const double*)w->Db2[in], (const double*)w->Ab2[in], w->Xb2[1 - in], w->Db2[1 - in], w->Ab2[1 - in], w->Wb,
        w->Rb, w->pbar));
    return DEM_OK;
}

template <typename Real>
__global__ void k_rec_positions(long long np, const PRec<Real>* __restrict__ S, double* __restrict__ P) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) st3(P, np, i, ld_pos<false>(S + i));
}

template <typename Real> int objective(dem_ctx* c, int which) {
    AdjWork* w = c->adj;
    const long long n = c->n, np = c->npad, cap = c->cap;
    cudaStream_t s = c->stream;
    double* P = w->Pobj;   // final positions as planes
    k_rec_positions<Real><<<grid_for(np, kB), kB, 0, s>>>(np, (const PRec<Real>*)c->rec[c->sbuf], P);
    DEM_CUDA_TRY(cudaMemsetAsync(w->obj, 0, 16 * sizeof(double), s));
    if (which == DEM_OBJ_PACKING) {
        unsigned long long init[2] = {0ull, ~0ull};
        DEM_CUDA_TRY(cudaMemcpyAsync(w->zmax, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_zmax<Real><<<grid_for(n, kB), kB, 0, s>>>(n, P + 2 * np, w->zmax);
        k_zargmax<<<grid_for(n, kB), kB, 0, s>>>(n, P + 2 * np, w->zmax);
        k_obj_packing<Real><<<grid_for(n, kB), kB, 0, s>>>(n, np, (const Real*)c->rad,
                                                           c->cfg.world[0] * c->cfg.world[1], c->vol, w->zmax, w->Xb,
                                                           w->Rb, w->obj);
    } else {
        AdjList L{c->off[c->cur], c->ln[c->cur], c->lp, c->roff, c->rk};
        k_obj_potential<Real><<<grid_for(n, kB), kB, 0, s>>>(n, np, cap, L, P, (const Real*)c->rad, c->mat.pp.estar,
                                                             c->mat.pw.estar, c->cfg.density, c->cfg.world[0] * 0.5,
                                                             c->cfg.world[1] * 0.5, w->Xb, w->Rb, w->objp);
    }
    DEM_LAUNCH_CHECK();
    return DEM_OK;
}

// The list of the window just built (no host sync: the pair arrays are
// copied at capacity; kernels read the pair count on the device) with its
// bound / free particle lists.
int list_snapshot(dem_ctx* c, ListRec& l) {
    cudaStream_t s = c->stream;
    const long long np = c->npad, cap = c->cap;
    int rc;
    if ((rc = copy(l.off, c->off[c->cur], (np + 1) * sizeof(uint), s)) ||
        (rc = copy(l.roff, c->roff, (np + 1) * sizeof(uint), s)) ||
        (rc = copy(l.ln, c->ln[c->cur], cap * sizeof(uint), s)) || (rc = copy(l.lp, c->lp, cap * sizeof(uint), s)) ||
        (rc = copy(l.rk, c->rk, cap * sizeof(uint), s)) || (rc = copy(l.bflag, c->bflag, np * sizeof(uint), s)) ||
        (rc = copy(l.blist, c->blist, np * sizeof(uint), s)) || (rc = copy(l.flist, c->flist, np * sizeof(uint), s)) ||
        (rc = copy(l.nb, c->bpos + c->n, sizeof(uint), s)))
        return rc;
    return DEM_OK;
}

// The recompute of one segment with the window kernel: per window, the
// re-list (recording the carry map), the list snapshot and the window kernel
// writing the tape.  Advances c->cur as the re-lists do.
int recompute_segment(dem_ctx* c, long long every) {
    AdjWork* w = c->adj;
    const int K = c->cfg.relist_interval;
    int rc;
    for (long long t = 0; t < every; t += K) {
        c->carry = w->lists[t / K].carry;
        rc = relist(c, c->cur);
        c->carry = nullptr;
        if (rc) return rc;
        c->cur = 1 - c->cur;
        c->hph = 0;
        if ((rc = list_snapshot(c, w->lists[t / K]))) return rc;
        WindowTape tape{w->tx, w->td, w->twh, w->tF, w->tT, w->th, w->ta, (int)t, w->tc};
        if ((rc = window_kernel(c, c->cur, &tape))) return rc;
    }
    return DEM_OK;
}

// The reversed steps of one segment (steps every-1 .. 0) from the selected
// tape set, enqueued on the reverse stream; hb / in advance as the steps swap
// their buffers.
int reverse_segment(dem_ctx* c, long long every, int& hb, int& in) {
    AdjWork* w = c->adj;
    const int K = c->cfg.relist_interval;
    const long long cap = c->cap;
    const bool mixed = c->prec == DEM_PREC_MIXED;
    cudaStream_t s = w->rs;
    int rc;
    const long long np = c->npad;
    for (long long t = every - 1; t >= 0; t--) {
        const ListRec& l = w->lists[t / K];
        if (t % K == K - 1) {   // the window's free particles, all its steps at once
            const int out = (K & 1) ? 1 - in : in;
            k_adj_free_window<<<grid_for(c->n, kB), kB, 0, s>>>(c->n, np, K, l.flist, l.nb, w->Xb2[in], w->Db2[in],
                                                                w->Ab2[in], w->Xb2[out], w->Db2[out], w->Ab2[out],
                                                                w->Wb);
            DEM_LAUNCH_CHECK();
        }
        rc = mixed ? adj_step<float>(c, t, l, hb, in) : adj_step<double>(c, t, l, hb, in);
        if (rc) return rc;
        in = 1 - in;   // set `in` now holds the adjoints of the state before the step
        hb = 1 - hb;   // Hb[hb] now holds the adjoint of this step's input history
        if (t % K == 0) {
            // input history came from the re-list carry: route it to the
            // previous list's output history
            DEM_CUDA_TRY(cudaMemsetAsync(w->Hb[1 - hb], 0, 3 * cap * sizeof(double), s));
            k_adj_carry<<<148 * 4, kB, 0, s>>>(l.off, c->n, cap, l.carry, w->Hb[hb], w->Hb[1 - hb]);
            DEM_LAUNCH_CHECK();
            hb = 1 - hb;
        }
    }
    return DEM_OK;
}

void reverse_parities(long long every, int K, int& hb, int& in) {
    for (long long t = every - 1; t >= 0; t--) {
        in = 1 - in;
        hb = 1 - hb;
        if (t % K == 0) hb = 1 - hb;
    }
}

// Captures what `enqueue` puts on stream s as a graph (once) and launches it.
template <typename F> int run_captured(cudaStream_t s, cudaGraphExec_t& ge, F enqueue) {
    if (!ge) {
        cudaGraph_t gr = nullptr;
        DEM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue();
        cudaError_t e = cudaStreamEndCapture(s, &gr);
        if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture (adjoint)", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&ge, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate (adjoint)", __FILE__, __LINE__);
    }
    DEM_CUDA_TRY(cudaGraphLaunch(ge, s));
    return DEM_OK;
}

}  // namespace
}  // namespace dem

using namespace dem;

extern "C" int dem_adjoint_window(dem_ctx* c, long long nsteps, int every, int which, dem_adjoint_result* out,
                                  double* d_radii) {
    if (!c || !out) return fail(DEM_ERR_ARG, "dem_adjoint_window: null argument");
    memset(out, 0, sizeof(*out));
    if (!c->uploaded || !c->have_mat) return fail(DEM_ERR_STATE, "dem_adjoint_window: upload state and material first");
    const int K = c->cfg.relist_interval;
    if (which != DEM_OBJ_PACKING && which != DEM_OBJ_POTENTIAL)
        return fail(DEM_ERR_ARG, "dem_adjoint_window: unknown objective %d", which);
    if (nsteps <= 0 || every <= 0 || every % K || nsteps % every)
        return fail(DEM_ERR_ARG, "dem_adjoint_window: need nsteps %% every == 0 and every %% relist_interval == 0");
    if (c->in_window != 0) return fail(DEM_ERR_STATE, "dem_adjoint_window: start at a re-list boundary");
    if (c->profiling) return fail(DEM_ERR_STATE, "dem_adjoint_window: switch profiling off");
    if (c->n != c->ntot)
        return fail(DEM_ERR_STATE, "dem_adjoint_window: layers are still to be poured in (%lld of %lld in the system)",
                    c->n, c->ntot);
    const long long nseg = nsteps / every;
    int rc = ensure_work(c, every, nseg + 1);
    if (rc) return rc;
    AdjWork* w = c->adj;
    cudaStream_t s = c->stream;
    const long long np = c->npad, cap = c->cap;
    const bool mixed = c->prec == DEM_PREC_MIXED;
    const bool rec0 = c->record;
    // ---------------------------------------------------- forward + checkpoints
    DEM_CUDA_TRY(cudaEventRecord(c->ev[0], s));
    const long long step0 = c->step, relists0 = c->relists;
    {
        NvtxRange fwd_range("dem adjoint forward");
        for (long long g = 0; g < nseg; g++) {
            if ((rc = save_ck(c, w->ck[g]))) return rc;
            if ((rc = dem_step_n(c, every))) return rc;
        }
    }
    if ((rc = save_ck(c, w->ck[nseg]))) return rc;
    const size_t last = (size_t)(K - 1) * c->npart;
    if ((rc = copy(w->save_mz, c->part_mz + last, c->npart * sizeof(unsigned long long), s)) ||
        (rc = copy(w->save_cnt, c->part_cnt + last, c->npart * sizeof(uint), s)))
        return rc;
    DEM_CUDA_TRY(cudaEventRecord(c->ev[1], s));
    // --------------------------------------------------------------- objective
    DEM_CUDA_TRY(cudaMemsetAsync(w->Xb, 0, 3 * np * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->Db, 0, 3 * np * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->Ab, 0, 3 * np * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->Wb, 0, 3 * np * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->Rb, 0, np * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->Hb[0], 0, 3 * cap * sizeof(double), s));
    DEM_CUDA_TRY(cudaMemsetAsync(w->pbar, 0, (size_t)w->npb * 12 * sizeof(double), s));
    rc = mixed ? objective<float>(c, which) : objective<double>(c, which);
    if (rc) return rc;
    // ------------------------------------------------------- reverse segments
    // Recompute path: the window kernel writing the tape of the bound
    // particles (PCCP), else per-step kernels with the force record.
    const bool win_path = c->mode == DEM_FORCE_PCCP && c->win_kernel;
    if (!win_path) dem_record_forces(c, 1);
    c->observe_slot = -1;   // the recompute writes no observables
    int hb = 0;   // Hb[hb]: adjoint of the pair history output by the step being reversed
    int in = 0;   // state-adjoint set of the state after the step being reversed
    if (w->graph_every != every) {
        w->fgraph.drop();
        w->rgraph.drop();
        w->graph_every = every;
    }
    SegmentGraphs& fgraph = w->fgraph;
    SegmentGraphs& rgraph = w->rgraph;
    // Segment g is recomputed into tape set g & 1 on the context's stream and
    // reversed from it on the reverse stream, so the recompute of segment g-1
    // (into the other set) runs beside the reverse of segment g: the two are
    // independent (the reverse reads only its tape and the adjoints).
    for (long long g = nseg - 1; g >= 0; g--) {
        const int k = (int)(g & 1);
        NvtxRange seg_range("dem adjoint segment (recompute + reverse)");
        // the set's previous reader, the reverse of segment g + 2, is done
        if (g + 2 <= nseg - 1) DEM_CUDA_TRY(cudaStreamWaitEvent(s, w->freed[k], 0));
        if ((rc = restore_ck(c, w->ck[g]))) return rc;
        select_set(w, k);
        // recompute the segment, recording what the reverse sweep needs
        if (win_path) {
            // one graph per tape set and list-buffer parity at the segment
            // start (the capture only records: c->cur is advanced after the
            // launch)
            const int cur0 = c->cur;
            rc = run_captured(s, fgraph.g[k][cur0][0], [&]() {
                const int r = recompute_segment(c, every);
                c->cur = cur0;
                return r;
            });
            if (rc) return rc;
            for (long long t = 0; t < every; t += K) c->cur = 1 - c->cur;
            c->hph = 0;
        }
        for (long long t = 0; !win_path && t < every; t++) {
            const int slot = (int)(t % K);
            if (slot == 0) {
                c->carry = w->lists[t / K].carry;
                rc = relist(c, c->cur);
                c->carry = nullptr;
                if (rc) return rc;
                c->cur = 1 - c->cur;
                c->hph = 0;
                if ((rc = list_snapshot(c, w->lists[t / K]))) return rc;
            }
            if (mixed)
                k_tape<float><<<148 * 4, kB, 0, s>>>(c->n, np, cap, (const PRec<float>*)c->rec[c->sbuf], c->wh,
                                                     c->off[c->cur],
                                                     c->hist[c->cur][c->hph], w->tx + 3 * np * t, w->td + 3 * np * t,
                                                     (float*)w->ta + 3 * np * t, w->twh + 3 * np * t,
                                                     w->th + 3 * cap * t);
            else
                k_tape<double><<<148 * 4, kB, 0, s>>>(c->n, np, cap, (const PRec<double>*)c->rec[c->sbuf], c->wh,
                                                      c->off[c->cur],
                                                      c->hist[c->cur][c->hph], w->tx + 3 * np * t,
                                                      w->td + 3 * np * t, (double*)w->ta + 3 * np * t,
                                                      w->twh + 3 * np * t, w->th + 3 * cap * t);
            DEM_LAUNCH_CHECK();
            // the step writes its total force and torque straight into the tape
            double* keepF = c->dbgF;
            double* keepT = c->dbgT;
            uint* keepC = c->dbgC;
            c->dbgF = w->tF + 3 * np * t;
            c->dbgT = w->tT + 3 * np * t;
            c->dbgC = w->tc + np * t;   // per-particle pair contacts
            double a, b;
            rc = step_kernels(c, c->cur, slot, &a, &b);
            c->dbgF = keepF;
            c->dbgT = keepT;
            c->dbgC = keepC;
            if (rc) return rc;
        }
        DEM_CUDA_TRY(cudaEventRecord(w->filled[k], s));
        // the reverse sweep step by step, after the recompute: one graph per
        // tape set and (hb, in) parity at the segment start
        DEM_CUDA_TRY(cudaStreamWaitEvent(w->rs, w->filled[k], 0));
        const int hb0 = hb, in0 = in;
        rc = run_captured(w->rs, rgraph.g[k][hb0][in0], [&]() {
            int h = hb0, i = in0;
            return reverse_segment(c, every, h, i);
        });
        if (rc) return rc;
        reverse_parities(every, K, hb, in);
        DEM_CUDA_TRY(cudaEventRecord(w->freed[k], w->rs));
    }
    DEM_CUDA_TRY(cudaEventRecord(w->joined, w->rs));
    DEM_CUDA_TRY(cudaStreamWaitEvent(s, w->joined, 0));
    DEM_CUDA_TRY(cudaEventRecord(c->ev[2], s));
    // ------------------------------------------------------------ results
    std::vector<double> pb((size_t)w->npb * 12);
    double obj[3] = {0.0, 0.0, 0.0};   // value, and the elastic energy's direct d/d estar (pair, wall)
    const size_t nob = (size_t)grid_for(c->n, kB);
    std::vector<double> op(which == DEM_OBJ_POTENTIAL ? 3 * nob : 0);
    DEM_CUDA_TRY(cudaMemcpyAsync(pb.data(), w->pbar, pb.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (which == DEM_OBJ_POTENTIAL)
        DEM_CUDA_TRY(cudaMemcpyAsync(op.data(), w->objp, op.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    else
        DEM_CUDA_TRY(cudaMemcpyAsync(obj, w->obj, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (d_radii) DEM_CUDA_TRY(cudaMemcpyAsync(d_radii, w->Rb, c->n * sizeof(double), cudaMemcpyDeviceToHost, s));
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    if (d_radii && c->ordered) {   // into the caller's particle order
        const int rp = host_perm(c);
        if (rp) return rp;
        std::vector<double> t(d_radii, d_radii + c->n);
        for (long long i = 0; i < c->n; i++) d_radii[c->hperm[i]] = t[i];
    }
    for (size_t b = 0; b < op.size() / 3; b++)   // block sums of the energy objective, in block order
        for (int q = 0; q < 3; q++) obj[q] += op[3 * b + q];
    double acc[12] = {0};
    for (size_t b = 0; b < (size_t)w->npb; b++)
        for (int k = 0; k < 12; k++) acc[k] += pb[b * 12 + k];
    out->value = obj[0];
    out->d_pp = dem_contact{acc[0], acc[1], 0.0, acc[2], acc[3], acc[4], acc[5]};
    out->d_pw = dem_contact{acc[6], acc[7], 0.0, acc[8], acc[9], acc[10], acc[11]};
    if (which == DEM_OBJ_POTENTIAL) {
        // direct dependence of the elastic energy on estar
        out->d_pp.estar += obj[1];
        out->d_pw.estar += obj[2];
    }
    float f1 = 0.f, f2 = 0.f;
    DEM_CUDA_TRY(cudaEventElapsedTime(&f1, c->ev[0], c->ev[1]));
    DEM_CUDA_TRY(cudaEventElapsedTime(&f2, c->ev[1], c->ev[2]));
    out->forward_ms = f1;
    out->adjoint_ms = f2;
    // leave the context at the end of the window, as dem_step_n(nsteps) would
    if ((rc = restore_ck(c, w->ck[nseg]))) return rc;
    if ((rc = copy(c->part_mz + last, w->save_mz, c->npart * sizeof(unsigned long long), s)) ||
        (rc = copy(c->part_cnt + last, w->save_cnt, c->npart * sizeof(uint), s)))
        return rc;
    dem_record_forces(c, rec0 ? 1 : 0);
    DEM_CUDA_TRY(cudaStreamSynchronize(s));
    c->step = step0 + nsteps;
    c->relists = relists0 + nsteps / K;
    c->in_window = 0;
    c->last_slot = K - 1;
    return DEM_OK;
}

namespace dem {
void adjoint_drop_graphs(dem_ctx* c) {
    if (!c->adj) return;
    c->adj->fgraph.drop();
    c->adj->rgraph.drop();
}
}  // namespace dem

extern "C" int dem_adjoint_release(dem_ctx* c) {
    if (!c || !c->adj) return DEM_OK;
    AdjWork* w = c->adj;
    cudaStreamSynchronize(c->stream);
    for (Ck& k : w->ck) free_ck(k);
    if (w->rs) cudaStreamSynchronize(w->rs);
    void* p[] = {w->Xb2[0], w->Db2[0], w->Ab2[0], w->Xb2[1], w->Db2[1], w->Ab2[1], w->Wb, w->Rb, w->Hb[0], w->Hb[1],
                 w->pbar, w->obj, w->zmax, w->save_mz, w->save_cnt, w->Pobj, w->objp, w->PC, w->pon, w->WS, w->wson};
    for (void* x : p)
        if (x) cudaFree(x);
    for (TapeSet& t : w->set) free_set(t);
    for (cudaEvent_t e : {w->filled[0], w->filled[1], w->freed[0], w->freed[1], w->joined})
        if (e) cudaEventDestroy(e);
    if (w->rs) cudaStreamDestroy(w->rs);
    delete w;
    c->adj = nullptr;
    return DEM_OK;
}
