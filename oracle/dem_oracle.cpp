/*
 * dem_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain FP64 C++/OpenMP restatement of the reference's DEM packing time step
 * (clera-gan/Discrete-Element-Method-for-Packing-CUDA-C-code).  It is the
 * checker for the CUDA library: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.  The product (libdem_b200.so) never
 * links or calls it.
 *
 * Parity pinning.  The reference ships no tests or golden outputs, and its
 * force laws (calforceij, calforceiw), four kernels (neighborarrayD,
 * pairlistD, sumallforceiD, outputporositycnD) and its SDK sort/scan are not
 * in the repository.  What exists (calcHashD, findCellStartD, addTwoArraysD,
 * vprojec, vscale, calculateforcepairD's bookkeeping, calculateforceiwD's
 * gravity/bookkeeping, updatepositionD) is pinned against golden vectors
 * produced by running those reference kernels themselves (tests/golden/).
 * The missing pieces follow the published Hertz-Mindlin model with rolling
 * friction (Zhou et al., Physica A 269 (1999) 536; Gan, Zhou & Yu, Powder
 * Technol. 301 (2016) 1172) and are pinned by physics known-answer tests
 * only: for them parity is unpinned against the reference itself.
 *
 * Build: g++ -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 * -ffp-contract=off keeps every product and sum rounded separately so the
 * FP32 list tests below reproduce the GPU's __fmul_rn/__fadd_rn bit for bit.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned int uint;
static const uint EMPTY = 0xffffffffu;

extern "C" {

/* ------------------------------------------------------------------ misc */
int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------- vector helpers */
static inline void v_cross(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double v_dot(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Single-precision length of cutil_math.h:1082-1093: sqrtf of the double dot
 * product.  The reference uses it in vprojec (neiglist.cu:140,142) and for the
 * re-list trigger (neiglist.cu:359). */
double ref_length(const double v[3]) {
    return (double)sqrtf((float)v_dot(v, v));
}

/* vprojec  -- neiglist.cu:133-146.  r = (-u) x (u x p): the component of p
 * perpendicular to unit u; with ityp != 0 the result is further scaled by
 * sqrt(|p|/|r|) (single-precision lengths) unless |p| < 0.001 or |p| > 100|r|. */
void ref_vprojec(const double p[3], const double u[3], double r[3], uint ityp) {
    double q[3], mu[3] = {-u[0], -u[1], -u[2]};
    v_cross(u, p, q);
    v_cross(mu, q, r);
    if (ityp == 0) return;
    double pmag = ref_length(p);
    if (pmag < 0.001) return;
    double rmag = ref_length(r);
    if (pmag > rmag * 100) return;
    double pr = sqrt(pmag / rmag);
    r[0] *= pr; r[1] *= pr; r[2] *= pr;
}

/* vscale -- neiglist.cu:148-153: vec *= p1/p2. */
void ref_vscale(double v[3], double p1, double p2) {
    double ratio = p1 / p2;
    v[0] *= ratio; v[1] *= ratio; v[2] *= ratio;
}

/* ------------------------------------------------------------ contact law
 * Published Hertz-Mindlin sphere model with viscous damping, Coulomb limit
 * and rolling resistance (the force law the reference calls as calforceij /
 * calforceiw, neiglist.cu:208,287; not in the repository).  Reduced units.
 *   n      unit vector from i to j (for a wall: from the particle to the wall)
 *   delta  overlap > 0
 *   U      per-step displacement of j's contact point relative to i's
 *   Wr     per-step relative rotation a_i - a_j
 *   xi     tangential history (in: previous, out: updated)
 * Outputs the force on i (Fi), the tangential part of it (Ft), the rolling
 * torque on i (Mr) and the elastic normal force magnitude (*fne).
 *   fn_e  = estar sqrt(R*) delta^1.5                       (Hertz, 4/3 in estar)
 *   fn    = fn_e - cn sqrt(6 m* (3/4 estar) sqrt(R* delta)) (U.n)/dt
 *   xi    = xi - (xi.n) n + U_t                 (rotate into the tangent plane)
 *   xmax  = mu (2-nu)/(2(1-nu)) delta,  s = min(|xi|,xmax)/xmax
 *   ft_e  = mu fn_e (1-(1-s)^1.5)
 *   Ft    = ft_e xi/|xi| + ct sqrt(6 mu m* fn_e sqrt(1-s)/xmax) U_t/dt,
 *           |Ft| <= mu fn_e (rescaled when above), |xi| <= xmax (rescaled)
 *   Mr    = -(roll + roll_rel R*) fn_e (Wr/|Wr|)
 *   Fi    = -fn n + Ft
 */
struct OContact { double estar, mu, nu, cn, ct, roll, roll_rel; };

static void law(double delta, const double n[3], double rstar, double mstar,
                const double U[3], const double Wr[3], double xi[3], double dt,
                const OContact& p, double Fi[3], double Ft[3], double Mr[3], double* fne)
{
    const double fn_e = p.estar * sqrt(rstar) * delta * sqrt(delta);
    const double Un = v_dot(U, n);
    const double cn_c = p.cn * sqrt(4.5 * mstar * p.estar * sqrt(rstar * delta));
    const double fn = fn_e - cn_c * (Un / dt);
    double Ut[3] = {U[0] - Un * n[0], U[1] - Un * n[1], U[2] - Un * n[2]};
    const double xn = v_dot(xi, n);
    xi[0] = xi[0] - xn * n[0] + Ut[0];
    xi[1] = xi[1] - xn * n[1] + Ut[1];
    xi[2] = xi[2] - xn * n[2] + Ut[2];
    if (p.mu > 0.0) {
        const double xmax = p.mu * (2.0 - p.nu) / (2.0 * (1.0 - p.nu)) * delta;
        const double xim = sqrt(v_dot(xi, xi));
        const double s = std::min(xim, xmax) / xmax;
        const double oms = 1.0 - s;
        const double ft_e = p.mu * fn_e * (1.0 - oms * sqrt(oms));
        const double ct_c = p.ct * sqrt(6.0 * p.mu * mstar * fn_e * sqrt(oms) / xmax);
        const double el = xim > 0.0 ? ft_e / xim : 0.0;
        for (int c = 0; c < 3; c++) Ft[c] = el * xi[c] + ct_c * (Ut[c] / dt);
        const double ftm = sqrt(v_dot(Ft, Ft));
        const double cap = p.mu * fn_e;
        if (ftm > cap) { const double sc = cap / ftm; for (int c = 0; c < 3; c++) Ft[c] *= sc; }
        if (xim > xmax) { const double sc = xmax / xim; for (int c = 0; c < 3; c++) xi[c] *= sc; }
    } else {
        Ft[0] = Ft[1] = Ft[2] = 0.0;
        xi[0] = xi[1] = xi[2] = 0.0;
    }
    const double rl = p.roll + p.roll_rel * rstar;
    const double w = sqrt(v_dot(Wr, Wr));
    if (w > 1e-30 && rl > 0.0) {
        const double sc = -(rl * fn_e / w);
        for (int c = 0; c < 3; c++) Mr[c] = sc * Wr[c];
    } else {
        Mr[0] = Mr[1] = Mr[2] = 0.0;
    }
    for (int c = 0; c < 3; c++) Fi[c] = -fn * n[c] + Ft[c];
    *fne = fn_e;
}

/* One pair: geometry + law.  Returns 1 when touching.  Ti/Tj torques on i/j. */
static int pair_force(const double xi_[3], const double xj_[3], const double di[3], const double dj[3],
                      const double ai[3], const double aj[3], double ri, double rj, double mi, double mj,
                      double hist[3], double dt, const OContact& p,
                      double Fi[3], double Ti[3], double Tj[3], double* ftmag)
{
    double D[3] = {xj_[0] - xi_[0], xj_[1] - xi_[1], xj_[2] - xi_[2]};
    const double d2 = v_dot(D, D);
    const double dist = sqrt(d2);
    const double delta = (ri + rj) - dist;
    if (!(delta > 0.0) || dist <= 0.0) {
        for (int c = 0; c < 3; c++) { Fi[c] = Ti[c] = Tj[c] = 0.0; hist[c] = 0.0; }
        *ftmag = 0.0;
        return 0;
    }
    double n[3] = {D[0] / dist, D[1] / dist, D[2] / dist};
    const double rstar = ri * rj / (ri + rj);
    const double mstar = mi * mj / (mi + mj);
    double ra[3] = {ri * ai[0] + rj * aj[0], ri * ai[1] + rj * aj[1], ri * ai[2] + rj * aj[2]};
    double rxn[3];
    v_cross(ra, n, rxn);
    double U[3] = {(dj[0] - di[0]) - rxn[0], (dj[1] - di[1]) - rxn[1], (dj[2] - di[2]) - rxn[2]};
    double Wr[3] = {ai[0] - aj[0], ai[1] - aj[1], ai[2] - aj[2]};
    double Ft[3], Mr[3], fne;
    law(delta, n, rstar, mstar, U, Wr, hist, dt, p, Fi, Ft, Mr, &fne);
    double nxf[3];
    v_cross(n, Ft, nxf);
    for (int c = 0; c < 3; c++) {
        Ti[c] = ri * nxf[c] + Mr[c];
        Tj[c] = rj * nxf[c] - Mr[c];
    }
    *ftmag = sqrt(v_dot(Ft, Ft));
    return 1;
}

/* Flat walls x=+-Wx/2, y=+-Wy/2, z=0 (open top; world origin (-Wx/2,-Wy/2,0),
 * dempacking.cu:333-339).  Walls are visited in the order floor, x-, x+, y-,
 * y+.  The reference keeps one wall-history slot per particle
 * (neiglist.cu:263-264,290-301); it belongs to the wall with the largest
 * overlap (the first one on a tie); any other touching wall uses a history
 * that starts from zero this step.  Returns 1 if any wall is touched. */
static int wall_force(const double ws[3], const double x[3], const double d[3], const double a[3],
                      double r, double m, double hist[3], double* fricpw, double dt,
                      const OContact& p, double F[3], double T[3])
{
    const double hx = ws[0] * 0.5, hy = ws[1] * 0.5;
    double dl[5];
    dl[0] = r - x[2];
    dl[1] = r - (x[0] + hx);
    dl[2] = r - (hx - x[0]);
    dl[3] = r - (x[1] + hy);
    dl[4] = r - (hy - x[1]);
    static const double nrm[5][3] = {{0, 0, -1}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}};
    int prim = -1;
    for (int w = 0; w < 5; w++)
        if (dl[w] > 0.0 && (prim < 0 || dl[w] > dl[prim])) prim = w;
    F[0] = F[1] = F[2] = 0.0;
    T[0] = T[1] = T[2] = 0.0;
    if (prim < 0) {
        hist[0] = hist[1] = hist[2] = 0.0;
        *fricpw = 0.0;
        return 0;
    }
    double newhist[3] = {0, 0, 0};
    double newfr = 0.0;
    for (int w = 0; w < 5; w++) {
        if (!(dl[w] > 0.0)) continue;
        const double* n = nrm[w];
        double axn[3];
        v_cross(a, n, axn);
        double U[3] = {-d[0] - r * axn[0], -d[1] - r * axn[1], -d[2] - r * axn[2]};
        double Wr[3] = {a[0], a[1], a[2]};
        double h[3] = {0, 0, 0};
        if (w == prim) { h[0] = hist[0]; h[1] = hist[1]; h[2] = hist[2]; }
        double Fi[3], Ft[3], Mr[3], fne;
        law(dl[w], n, r, m, U, Wr, h, dt, p, Fi, Ft, Mr, &fne);
        double nxf[3];
        v_cross(n, Ft, nxf);
        for (int c = 0; c < 3; c++) {
            F[c] += Fi[c];
            T[c] += r * nxf[c] + Mr[c];
        }
        if (w == prim) {
            newhist[0] = h[0]; newhist[1] = h[1]; newhist[2] = h[2];
            newfr = sqrt(v_dot(Ft, Ft));
        }
    }
    hist[0] = newhist[0]; hist[1] = newhist[1]; hist[2] = newhist[2];
    *fricpw = newfr;
    return 1;
}

/* Exposed for known-answer tests: force on i, torques, updated history. */
int orc_pair_force(const double* xi, const double* xj, const double* di, const double* dj,
                   const double* ai, const double* aj, double ri, double rj, double mi, double mj,
                   double* hist, double dt, const double* par7,
                   double* Fi, double* Ti, double* Tj)
{
    OContact p{par7[0], par7[1], par7[2], par7[3], par7[4], par7[5], par7[6]};
    double ft;
    return pair_force(xi, xj, di, dj, ai, aj, ri, rj, mi, mj, hist, dt, p, Fi, Ti, Tj, &ft);
}
int orc_wall_force(const double* ws, const double* x, const double* d, const double* a,
                   double r, double m, double* hist, double dt, const double* par7,
                   double* F, double* T)
{
    OContact p{par7[0], par7[1], par7[2], par7[3], par7[4], par7[5], par7[6]};
    double fr;
    return wall_force(ws, x, d, a, r, m, hist, &fr, dt, p, F, T);
}

/* =========================================================================
 * Reference-compatible restatements (host arrays, reference layout)
 * =======================================================================*/
static double g_cua = 1.0, g_cub = 1.55;          /* neiglist.cu:27-28 */
static OContact g_pp{0, 0, 0, 0, 0, 0, 0}, g_pw{0, 0, 0, 0, 0, 0, 0};

/* Par/ParW (neiglist.cu:32-49): estar, ufric, vpois, dampn, dampt, upp. */
void ref_set_material(const double* par6, const double* parw6) {
    g_pp = OContact{par6[0], par6[1], par6[2], par6[3], par6[4], par6[5], 0.0};
    g_pw = OContact{parw6[0], parw6[1], parw6[2], parw6[3], parw6[4], parw6[5], 0.0};
}
void ref_set_cutoff(double cua, double cub) { g_cua = cua; g_cub = cub; }

/* calcGridPos / calcGridAddress -- neiglist.cu:54-75.  The clamp is
 * max(0, min(int, uint-1)): CUDA's min(int, unsigned) compares as unsigned,
 * so a negative cell coordinate becomes gridSize-1, not 0. */
static inline uint ref_grid_address(const double p[3], const uint gs[3], const double cs[3], const double o[3]) {
    long long g[3];
    for (int c = 0; c < 3; c++) {
        int gp = (int)floor((p[c] - o[c]) / cs[c]);
        uint ug = (uint)gp;
        uint lim = gs[c] - 1u;
        uint mn = ug < lim ? ug : lim;
        g[c] = (long long)mn;   /* max(0, mn): mn is unsigned, never < 0 */
    }
    return (uint)(g[2] * gs[1] * gs[0] + g[1] * gs[0] + g[0]);
}

/* calcHash -- particleSystem.cu:27-45 / calcHashD neiglist.cu:77-97. */
void ref_calcHash(const double* pos, uint* hash, const uint* gs, const double* cs, const double* o, int n) {
    #pragma omp parallel for
    for (int i = 0; i < n; i++) {
        hash[2 * i] = ref_grid_address(pos + 3 * i, gs, cs, o);
        hash[2 * i + 1] = (uint)i;
    }
}

/* RadixSort(.., n, bits) -- dempacking.cu:553: stable sort by key. */
void ref_radix_sort(uint* kv, uint n, uint bits) {
    std::vector<std::pair<uint, uint>> v(n);
    const uint mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
    for (uint i = 0; i < n; i++) v[i] = {kv[2 * i], kv[2 * i + 1]};
    std::stable_sort(v.begin(), v.end(), [mask](const std::pair<uint, uint>& a, const std::pair<uint, uint>& b) {
        return (a.first & mask) < (b.first & mask);
    });
    for (uint i = 0; i < n; i++) { kv[2 * i] = v[i].first; kv[2 * i + 1] = v[i].second; }
}

/* findCellStart -- particleSystem.cu:49-64 / neiglist.cu:102-120. */
void ref_findCellStart(const uint* hash, uint* cellStart, int n, uint ncells) {
    for (uint c = 0; c < ncells; c++) cellStart[c] = EMPTY;
    for (int i = 0; i < n; i++) {
        uint cell = hash[2 * i];
        if (i == 0 || cell != hash[2 * (i - 1)]) cellStart[cell] = (uint)i;
    }
}

/* neighborarray -- particleSystem.cu:67-97 (neighborarrayD not in the
 * repository).  27-cell walk around i's cell using cellStart and the key
 * change as cell end; candidate when |x_i-x_j|^2 < cub^2.  Row layout: j>i
 * ascending, then j<i ascending.  Returns the number of rows that overflowed. */
int ref_neighborarray(const double* pos, const uint* hash, const uint* cellStart, const uint* gs,
                      const double* cs, const double* o, int maxppc, int n,
                      uint* Anei, uint* njgi, uint* njli)
{
    int overflow = 0;
    const double cub2 = g_cub * g_cub;
    #pragma omp parallel for reduction(+:overflow)
    for (int i = 0; i < n; i++) {
        const double* pi = pos + 3 * i;
        uint a = ref_grid_address(pi, gs, cs, o);
        long long gx = a % gs[0], gy = (a / gs[0]) % gs[1], gz = a / (gs[0] * gs[1]);
        std::vector<uint> up, lo;
        for (long long z = gz - 1; z <= gz + 1; z++) {
            if (z < 0 || z >= gs[2]) continue;
            for (long long y = gy - 1; y <= gy + 1; y++) {
                if (y < 0 || y >= gs[1]) continue;
                for (long long x = gx - 1; x <= gx + 1; x++) {
                    if (x < 0 || x >= gs[0]) continue;
                    uint c = (uint)((z * gs[1] + y) * gs[0] + x);
                    uint t = cellStart[c];
                    if (t == EMPTY) continue;
                    for (; t < (uint)n && hash[2 * t] == c; t++) {
                        uint j = hash[2 * t + 1];
                        if (j == (uint)i) continue;
                        const double* pj = pos + 3 * j;
                        double dx = pj[0] - pi[0], dy = pj[1] - pi[1], dz = pj[2] - pi[2];
                        double d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 < cub2) (j > (uint)i ? up : lo).push_back(j);
                    }
                }
            }
        }
        std::sort(up.begin(), up.end());
        std::sort(lo.begin(), lo.end());
        size_t tot = up.size() + lo.size();
        if (tot > (size_t)maxppc) overflow++;
        uint* row = Anei + (size_t)i * maxppc;
        for (int s = 0; s < maxppc; s++) row[s] = EMPTY;
        size_t s = 0;
        size_t nu = std::min(up.size(), (size_t)maxppc);
        for (size_t k = 0; k < nu; k++) row[s++] = up[k];
        size_t nl = std::min(lo.size(), (size_t)maxppc - nu);
        for (size_t k = 0; k < nl; k++) row[s++] = lo[k];
        njgi[i] = (uint)nu;
        njli[i] = (uint)nl;
    }
    return overflow;
}

/* prefixsum -- particleSystem.cu:126-140. */
uint ref_prefixsum(uint n, const uint* njgi, uint* sjgi, uint* oldsjgi) {
    memcpy(oldsjgi, sjgi, n * sizeof(uint));
    uint acc = 0;
    for (uint i = 0; i < n; i++) { acc += njgi[i]; sjgi[i] = acc; }
    return n ? sjgi[n - 1] : 0;
}

/* pairlist -- particleSystem.cu:143-191 (pairlistD not in the repository). */
void ref_pairlist(const uint* sjgi, const uint* oldsjgi, const uint* oldLn, const uint* Anei,
                  const uint* njgi, const uint* njli, const double* olddispt, const double* oldfricp,
                  int maxppc, int maxcn, uint n, uint* Aref, uint* Lp, uint* Ln,
                  double* dispt, double* fricp)
{
    const size_t capN = (size_t)n * maxppc, capP = (size_t)n * maxcn;
    for (size_t k = 0; k < capN; k++) Aref[k] = EMPTY;
    for (size_t k = 0; k < capP; k++) { Lp[k] = EMPTY; Ln[k] = EMPTY; fricp[k] = 0.0; }
    for (size_t k = 0; k < 3 * capP; k++) dispt[k] = 0.0;
    #pragma omp parallel for
    for (long long ii = 0; ii < (long long)n; ii++) {
        uint i = (uint)ii;
        uint base = sjgi[i] - njgi[i];
        uint os = i > 0 ? oldsjgi[i - 1] : 0u, oe = oldsjgi[i];
        if (oe > capP) oe = (uint)capP;
        if (os > oe) os = oe;
        const uint* row = Anei + (size_t)i * maxppc;
        for (uint s = 0; s < njgi[i]; s++) {
            uint k = base + s, j = row[s];
            Lp[k] = i; Ln[k] = j;
            Aref[(size_t)i * maxppc + s] = k;
            for (uint t = os; t < oe; t++) {
                if (oldLn[t] == j) {
                    dispt[3 * k] = olddispt[3 * t];
                    dispt[3 * k + 1] = olddispt[3 * t + 1];
                    dispt[3 * k + 2] = olddispt[3 * t + 2];
                    fricp[k] = oldfricp[t];
                    break;
                }
            }
        }
        for (uint s = njgi[i]; s < njgi[i] + njli[i]; s++) {
            uint j = row[s];
            uint kk = EMPTY;
            const uint* rowj = Anei + (size_t)j * maxppc;
            for (uint t = 0; t < njgi[j]; t++)
                if (rowj[t] == i) { kk = sjgi[j] - njgi[j] + t; break; }
            Aref[(size_t)i * maxppc + s] = kk;
        }
    }
}

/* calculateforcepair -- particleSystem.cu:194-240 / neiglist.cu:156-233. */
void ref_calculateforcepair(const double* pos, const double* pdis, const double* angv, const double* rad,
                            const double* rmass, const uint* Lp, const uint* Ln, uint* oldLn,
                            double* dispt, double* fricp, double* olddispt, double* oldfricp, double dt,
                            double* forcepair, double* torqpairi, double* torqpairj, uint* contactpair,
                            uint total)
{
    #pragma omp parallel for
    for (long long kk = 0; kk < (long long)total; kk++) {
        size_t k = (size_t)kk;
        uint i = Lp[k], j = Ln[k];
        double h[3] = {dispt[3 * k], dispt[3 * k + 1], dispt[3 * k + 2]};
        double F[3], Ti[3], Tj[3], ft;
        int c = pair_force(pos + 3 * i, pos + 3 * j, pdis + 3 * i, pdis + 3 * j, angv + 3 * i, angv + 3 * j,
                           rad[i], rad[j], rmass[i], rmass[j], h, dt, g_pp, F, Ti, Tj, &ft);
        for (int q = 0; q < 3; q++) {
            forcepair[3 * k + q] = c ? F[q] : 0.0;
            torqpairi[3 * k + q] = c ? Ti[q] : 0.0;
            torqpairj[3 * k + q] = c ? Tj[q] : 0.0;
            dispt[3 * k + q] = c ? h[q] : 0.0;
            olddispt[3 * k + q] = h[q];
        }
        fricp[k] = c ? ft : 0.0;
        oldfricp[k] = c ? ft : 0.0;
        contactpair[k] = c ? 1u : 0u;
        oldLn[k] = j;
    }
}

/* sumallforcei -- particleSystem.cu:243-277 (sumallforceiD not in the
 * repository): gather through Aref in row order. */
void ref_sumallforcei(int maxppc, int n, const uint* njgi, const uint* njli, const double* forcepair,
                      const double* torqpairi, const double* torqpairj, const uint* contactpair,
                      const uint* Aref, double* forcei, double* torquei, uint* contacti)
{
    #pragma omp parallel for
    for (int i = 0; i < n; i++) {
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        uint cnt = 0;
        const uint* row = Aref + (size_t)i * maxppc;
        for (uint s = 0; s < njgi[i] + njli[i]; s++) {
            uint k = row[s];
            if (k == EMPTY) continue;
            if (s < njgi[i]) {
                for (int q = 0; q < 3; q++) { F[q] += forcepair[3 * k + q]; T[q] += torqpairi[3 * k + q]; }
            } else {
                for (int q = 0; q < 3; q++) { F[q] -= forcepair[3 * k + q]; T[q] += torqpairj[3 * k + q]; }
            }
            cnt += contactpair[k];
        }
        for (int q = 0; q < 3; q++) { forcei[3 * i + q] = F[q]; torquei[3 * i + q] = T[q]; }
        contacti[i] = cnt;
    }
}

/* calculateforceiw -- particleSystem.cu:279-313 / neiglist.cu:238-306. */
void ref_calculateforceiw(const double* ws, const double* pos, const double* pdis, const double* angv,
                          const double* rad, const double* rmass, double dt, uint total, int n,
                          double* disptw, double* fricpw, double* forcei, double* torquei)
{
    #pragma omp parallel for
    for (int i = 0; i < n; i++) {
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        if (total != 0) {
            for (int q = 0; q < 3; q++) { F[q] = forcei[3 * i + q]; T[q] = torquei[3 * i + q]; }
        }
        F[2] += -rmass[i];
        double h[3] = {disptw[3 * i], disptw[3 * i + 1], disptw[3 * i + 2]};
        double fr = fricpw[i];
        double Fw[3], Tw[3];
        int hit = wall_force(ws, pos + 3 * i, pdis + 3 * i, angv + 3 * i, rad[i], rmass[i], h, &fr, dt, g_pw, Fw, Tw);
        if (hit) {
            for (int q = 0; q < 3; q++) { F[q] += Fw[q]; T[q] += Tw[q]; disptw[3 * i + q] = h[q]; }
            fricpw[i] = fr;
        } else {
            for (int q = 0; q < 3; q++) disptw[3 * i + q] = 0.0;
            fricpw[i] = 0.0;
        }
        for (int q = 0; q < 3; q++) { forcei[3 * i + q] = F[q]; torquei[3 * i + q] = T[q]; }
    }
}

/* updateposition -- particleSystem.cu:315-384 / neiglist.cu:308-409 with
 * adamp = bdamp = 1 (neiglist.cu:354-355).  Returns iall; *maxhz =
 * max(0, max z) as the host loop at particleSystem.cu:372-379. */
uint ref_updateposition(const double* ws, int n, double* pos, double* pdis, double* angv,
                        const double* rmass, const double* inert, const double* forcei,
                        const double* torquei, double* qi, double dt, double* maxhz)
{
    (void)ws;
    const double ann = 0.5 * (g_cub - g_cua);
    uint iall = 0;
    double mz = 0.0;
    for (int i = 0; i < n; i++) {
        for (int q = 0; q < 3; q++) {
            pdis[3 * i + q] = pdis[3 * i + q] + forcei[3 * i + q] * dt * dt / rmass[i];
            pos[3 * i + q] += pdis[3 * i + q];
            qi[3 * i + q] += pdis[3 * i + q];
        }
        double rmov = ref_length(qi + 3 * i);
        for (int q = 0; q < 3; q++)
            angv[3 * i + q] = angv[3 * i + q] + torquei[3 * i + q] * dt * dt / inert[i];
        mz = std::max(mz, pos[3 * i + 2]);
        if (rmov > ann) iall = 1;
    }
    *maxhz = mz;
    return iall;
}

/* outputporositycn -- particleSystem.cu:386-422. */
uint ref_outputporositycn(uint n, const uint* contacti) {
    uint s = 0;
    for (uint i = 0; i < n; i++) s += contacti[i];
    return s;
}

/* =========================================================================
 * Engine restatement (the context API's semantics: CSR half list with
 * per-pair cut-off r_i+r_j+skin, fixed re-list interval, FP32 or FP64 list)
 * =======================================================================*/
struct OGrid {
    double o[3], cs;
    uint gs[3];
    float of[3], csf;
};
static OGrid make_grid(const double* world, double cs) {
    OGrid g;
    g.o[0] = -world[0] * 0.5; g.o[1] = -world[1] * 0.5; g.o[2] = 0.0;
    g.cs = cs; g.csf = (float)cs;
    for (int c = 0; c < 3; c++) { g.gs[c] = (uint)((int)(world[c] / cs) + 1); g.of[c] = (float)g.o[c]; }
    return g;
}
static inline int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

/* Cell coordinate of a position.  FP64 list: floor((x-o)/cs).  FP32 list:
 * xf = (float)(x - o) (FP64 difference rounded once), floorf(xf / (float)cs). */
static inline void cell_of(const OGrid& g, const double* p, int fp32, int c3[3]) {
    for (int c = 0; c < 3; c++) {
        /* the quotient is clamped to [-1, G] before floor so that far-away
         * positions cannot overflow the int (same as the GPU) */
        int v;
        const int G = (int)g.gs[c];
        if (fp32) {
            float xf = (float)(p[c] - g.o[c]);
            float q = xf / g.csf;
            q = q < -1.0f ? -1.0f : (q > (float)G ? (float)G : q);
            v = (int)floorf(q);
        } else {
            double q = (p[c] - g.o[c]) / g.cs;
            q = q < -1.0 ? -1.0 : (q > (double)G ? (double)G : q);
            v = (int)floor(q);
        }
        c3[c] = clampi(v, G - 1);
    }
}

int orc_grid_size(const double* world, double cs, uint* gs_out) {
    OGrid g = make_grid(world, cs);
    gs_out[0] = g.gs[0]; gs_out[1] = g.gs[1]; gs_out[2] = g.gs[2];
    return 0;
}

/* keys[i] = (gz*Gy + gy)*Gx + gx */
void orc_hash(long long n, const double* pos, const double* world, double cs, int fp32, uint* keys) {
    OGrid g = make_grid(world, cs);
    #pragma omp parallel for
    for (long long i = 0; i < n; i++) {
        int c3[3];
        cell_of(g, pos + 3 * i, fp32, c3);
        keys[i] = ((uint)c3[2] * g.gs[1] + (uint)c3[1]) * g.gs[0] + (uint)c3[0];
    }
}

/* Stable sort of ids by key; cell ranges [start, end) (EMPTY if empty). */
void orc_sort_cells(long long n, const uint* keys, uint ncells, uint* skeys, uint* sids,
                    uint* cstart, uint* cend) {
    std::vector<uint> idx(n);
    for (long long i = 0; i < n; i++) idx[i] = (uint)i;
    std::stable_sort(idx.begin(), idx.end(), [keys](uint a, uint b) { return keys[a] < keys[b]; });
    for (long long t = 0; t < n; t++) { sids[t] = idx[t]; skeys[t] = keys[idx[t]]; }
    for (uint c = 0; c < ncells; c++) { cstart[c] = EMPTY; cend[c] = EMPTY; }
    for (long long t = 0; t < n; t++) {
        uint c = skeys[t];
        if (t == 0 || skeys[t - 1] != c) cstart[c] = (uint)t;
        if (t == n - 1 || skeys[t + 1] != c) cend[c] = (uint)(t + 1);
    }
}

/* Candidate test.  FP64: (dx^2+dy^2)+dz^2 < ((ri+rj)+skin)^2.  FP32: the same
 * with xf = (float)(x-o), (float)r, (float)skin, every op rounded to FP32. */
static inline bool candidate(const double* pi, const double* pj, double ri, double rj, double skin,
                             const OGrid& g, int fp32) {
    if (fp32) {
        float dx = (float)(pj[0] - g.o[0]) - (float)(pi[0] - g.o[0]);
        float dy = (float)(pj[1] - g.o[1]) - (float)(pi[1] - g.o[1]);
        float dz = (float)(pj[2] - g.o[2]) - (float)(pi[2] - g.o[2]);
        float d2 = dx * dx + dy * dy;
        d2 = d2 + dz * dz;
        float cut = ((float)ri + (float)rj) + (float)skin;
        return d2 < cut * cut;
    }
    double dx = pj[0] - pi[0], dy = pj[1] - pi[1], dz = pj[2] - pi[2];
    double d2 = dx * dx + dy * dy;
    d2 = d2 + dz * dz;
    double cut = (ri + rj) + skin;
    return d2 < cut * cut;
}

/* Half list in CSR: pairs of i at [off[i], off[i+1]) with j>i ascending.
 * History of (i,j) carried from the previous list (old_off/old_ln/old_hist)
 * when present, else zero.  Returns the pair count, or -(needed) when cap is
 * too small.  *max_row receives the largest per-particle candidate count. */
long long orc_build_list(long long n, const double* pos, const double* rad, const double* world,
                         double cs, double skin, int fp32,
                         const uint* old_off, const uint* old_ln, const double* old_hist,
                         uint* off, uint* ln, double* hist, long long cap, int* max_row)
{
    OGrid g = make_grid(world, cs);
    const uint ncells = g.gs[0] * g.gs[1] * g.gs[2];
    std::vector<uint> keys(n), skeys(n), sids(n), cst(ncells), cen(ncells);
    orc_hash(n, pos, world, cs, fp32, keys.data());
    orc_sort_cells(n, keys.data(), ncells, skeys.data(), sids.data(), cst.data(), cen.data());
    std::vector<std::vector<uint>> up(n);
    std::vector<int> rowc(n, 0);
    #pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < n; i++) {
        int c3[3];
        cell_of(g, pos + 3 * i, fp32, c3);
        int cnt = 0;
        for (int z = c3[2] - 1; z <= c3[2] + 1; z++) {
            if (z < 0 || z >= (int)g.gs[2]) continue;
            for (int y = c3[1] - 1; y <= c3[1] + 1; y++) {
                if (y < 0 || y >= (int)g.gs[1]) continue;
                for (int x = c3[0] - 1; x <= c3[0] + 1; x++) {
                    if (x < 0 || x >= (int)g.gs[0]) continue;
                    uint c = ((uint)z * g.gs[1] + (uint)y) * g.gs[0] + (uint)x;
                    if (cst[c] == EMPTY) continue;
                    for (uint t = cst[c]; t < cen[c]; t++) {
                        uint j = sids[t];
                        if (j == (uint)i) continue;
                        if (candidate(pos + 3 * i, pos + 3 * j, rad[i], rad[j], skin, g, fp32)) {
                            cnt++;
                            if (j > (uint)i) up[i].push_back(j);
                        }
                    }
                }
            }
        }
        std::sort(up[i].begin(), up[i].end());
        rowc[i] = cnt;
    }
    int mr = 0;
    long long total = 0;
    for (long long i = 0; i < n; i++) { mr = std::max(mr, rowc[i]); total += (long long)up[i].size(); }
    if (max_row) *max_row = mr;
    if (total > cap) return -total;
    off[0] = 0;
    for (long long i = 0; i < n; i++) off[i + 1] = off[i] + (uint)up[i].size();
    #pragma omp parallel for
    for (long long i = 0; i < n; i++) {
        uint k = off[i];
        for (uint j : up[i]) {
            ln[k] = j;
            double h[3] = {0, 0, 0};
            if (old_off && old_ln && old_hist) {
                const uint* b = old_ln + old_off[i];
                const uint* e = old_ln + old_off[i + 1];
                const uint* f = std::lower_bound(b, e, j);
                if (f != e && *f == j) {
                    size_t t = (size_t)(f - old_ln);
                    h[0] = old_hist[3 * t]; h[1] = old_hist[3 * t + 1]; h[2] = old_hist[3 * t + 2];
                }
            }
            hist[3 * (size_t)k] = h[0]; hist[3 * (size_t)k + 1] = h[1]; hist[3 * (size_t)k + 2] = h[2];
            k++;
        }
    }
    return total;
}

/* Engine state in host AoS double arrays. */
struct OState {
    long long n;
    double *pos, *pdis, *angv, *rad;
    double *whist;         /* wall history 3n */
    double *q;             /* displacement since last list 3n */
};

/* One engine force step for a given list.  Force/torque/contacts outputs are
 * per particle (AoS); the pair history is updated in place.  Summation order:
 * own pairs (k ascending), pairs where i is the j side (k ascending), gravity,
 * walls. */
static void engine_forces(const OState& s, const double* world, double dt, double density,
                          const OContact& pp, const OContact& pw,
                          long long P, const uint* off, const uint* ln, double* hist,
                          double* force, double* torque, uint* contacts)
{
    const long long n = s.n;
    std::vector<double> pf(3 * P), pti(3 * P), ptj(3 * P);
    std::vector<uint> pc(P);
    std::vector<uint> lp(P);
    for (long long i = 0; i < n; i++)
        for (uint k = off[i]; k < off[i + 1]; k++) lp[k] = (uint)i;
    #pragma omp parallel for
    for (long long k = 0; k < P; k++) {
        uint i = lp[k], j = ln[k];
        double mi = density * 8.0 * s.rad[i] * s.rad[i] * s.rad[i];
        double mj = density * 8.0 * s.rad[j] * s.rad[j] * s.rad[j];
        double ft;
        pc[k] = (uint)pair_force(s.pos + 3 * i, s.pos + 3 * j, s.pdis + 3 * i, s.pdis + 3 * j,
                                 s.angv + 3 * i, s.angv + 3 * j, s.rad[i], s.rad[j], mi, mj,
                                 hist + 3 * k, dt, pp, &pf[3 * k], &pti[3 * k], &ptj[3 * k], &ft);
    }
    /* reverse CSR: pairs with Ln == j, k ascending */
    std::vector<uint> roff(n + 1, 0), rk(P);
    for (long long k = 0; k < P; k++) roff[ln[k] + 1]++;
    for (long long i = 0; i < n; i++) roff[i + 1] += roff[i];
    {
        std::vector<uint> fill(roff.begin(), roff.end() - 1);
        for (long long k = 0; k < P; k++) rk[fill[ln[k]]++] = (uint)k;
    }
    #pragma omp parallel for
    for (long long i = 0; i < n; i++) {
        double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
        uint c = 0;
        for (uint k = off[i]; k < off[i + 1]; k++) {
            for (int q = 0; q < 3; q++) { F[q] += pf[3 * k + q]; T[q] += pti[3 * k + q]; }
            c += pc[k];
        }
        for (uint t = roff[i]; t < roff[i + 1]; t++) {
            uint k = rk[t];
            for (int q = 0; q < 3; q++) { F[q] -= pf[3 * k + q]; T[q] += ptj[3 * k + q]; }
            c += pc[k];
        }
        const double r = s.rad[i];
        const double m = density * 8.0 * r * r * r;
        F[2] += -m;
        double Fw[3], Tw[3], fr;
        wall_force(world, s.pos + 3 * i, s.pdis + 3 * i, s.angv + 3 * i, r, m, s.whist + 3 * i, &fr, dt, pw, Fw, Tw);
        for (int q = 0; q < 3; q++) { F[q] += Fw[q]; T[q] += Tw[q]; }
        for (int q = 0; q < 3; q++) { force[3 * i + q] = F[q]; torque[3 * i + q] = T[q]; }
        contacts[i] = c;
    }
}

/* Integrator of neiglist.cu:356-360 (adamp = bdamp = 1):
 * pdis += F dt dt / m; pos += pdis; q += pdis; angv += T dt dt / I,
 * m = density 8 r^3, I = 0.4 m r^2 (dempacking.cu:311-312). */
static void engine_integrate(OState& s, double dt, double density, const double* force, const double* torque,
                             double skin, double* maxhz, int* skin_violation)
{
    const long long n = s.n;
    double mz = 0.0;
    int viol = 0;
    #pragma omp parallel for reduction(max:mz) reduction(|:viol)
    for (long long i = 0; i < n; i++) {
        const double r = s.rad[i];
        const double m = density * 8.0 * r * r * r;
        const double I = 0.4 * m * (r * r);
        for (int q = 0; q < 3; q++) {
            s.pdis[3 * i + q] = s.pdis[3 * i + q] + force[3 * i + q] * dt * dt / m;
            s.pos[3 * i + q] += s.pdis[3 * i + q];
            s.q[3 * i + q] += s.pdis[3 * i + q];
            s.angv[3 * i + q] = s.angv[3 * i + q] + torque[3 * i + q] * dt * dt / I;
        }
        mz = std::max(mz, s.pos[3 * i + 2]);
        double q2 = v_dot(s.q + 3 * i, s.q + 3 * i);
        if (q2 > 0.25 * skin * skin) viol |= 1;
    }
    *maxhz = mz;
    *skin_violation = viol;
}

/* Full engine loop.  params: [dt, skin, cell, density] ; mat: 14 doubles (pp 7,
 * pw 7) ; relist every `interval` steps starting at step 0.  State arrays are
 * updated in place; whist (3n) must be zero on entry for a fresh start.
 * out_scalars per step (if not NULL): [maxhz, contacts, pairs] * nsteps.
 * Returns 0, or 3 when the pair capacity was exceeded, 5 on a skin violation. */
int orc_run_list(long long n, double* pos, double* pdis, double* angv, const double* rad, double* whist,
                 const double* world, const double* params, const double* mat, int fp32_list,
                 long long nsteps, int interval, long long cap, double* out_scalars,
                 double* last_force, double* last_torque, uint* last_contacts,
                 uint* out_off, uint* out_ln, double* out_hist, long long* out_P);

int orc_run(long long n, double* pos, double* pdis, double* angv, const double* rad, double* whist,
            const double* world, const double* params, const double* mat, int fp32_list,
            long long nsteps, int interval, long long cap, double* out_scalars,
            double* last_force, double* last_torque, uint* last_contacts)
{
    return orc_run_list(n, pos, pdis, angv, rad, whist, world, params, mat, fp32_list, nsteps, interval, cap,
                        out_scalars, last_force, last_torque, last_contacts, nullptr, nullptr, nullptr, nullptr);
}

/* orc_run that also returns the final list (CSR offsets, j per pair and the
 * FP64 tangential history after the last step). */
int orc_run_list(long long n, double* pos, double* pdis, double* angv, const double* rad, double* whist,
                 const double* world, const double* params, const double* mat, int fp32_list,
                 long long nsteps, int interval, long long cap, double* out_scalars,
                 double* last_force, double* last_torque, uint* last_contacts,
                 uint* out_off, uint* out_ln, double* out_hist, long long* out_P)
{
    const double dt = params[0], skin = params[1], cs = params[2], density = params[3];
    OContact pp{mat[0], mat[1], mat[2], mat[3], mat[4], mat[5], mat[6]};
    OContact pw{mat[7], mat[8], mat[9], mat[10], mat[11], mat[12], mat[13]};
    std::vector<double> q(3 * n, 0.0), F(3 * n), T(3 * n);
    std::vector<uint> C(n);
    OState s{n, pos, pdis, angv, const_cast<double*>(rad), whist, q.data()};
    std::vector<uint> off(n + 1, 0), ln, ooff(n + 1, 0), oln;
    std::vector<double> hist, ohist;
    long long P = 0;
    int status = 0;
    bool have_old = false;
    for (long long st = 0; st < nsteps; st++) {
        if (st % interval == 0) {
            ln.assign(cap > 0 ? cap : 1, 0);
            hist.assign(3 * (cap > 0 ? cap : 1), 0.0);
            int mr;
            long long got = orc_build_list(n, pos, rad, world, cs, skin, fp32_list,
                                           have_old ? ooff.data() : nullptr, have_old ? oln.data() : nullptr,
                                           have_old ? ohist.data() : nullptr,
                                           off.data(), ln.data(), hist.data(), cap, &mr);
            if (got < 0) return 3;
            P = got;
            std::fill(q.begin(), q.end(), 0.0);
        }
        engine_forces(s, world, dt, density, pp, pw, P, off.data(), ln.data(), hist.data(),
                      F.data(), T.data(), C.data());
        double mz;
        int viol;
        engine_integrate(s, dt, density, F.data(), T.data(), skin, &mz, &viol);
        if (viol && !status) status = 5;
        /* keep the history of this step as "old list" for the next re-list */
        ooff = off;
        oln.assign(ln.begin(), ln.begin() + P);
        ohist.assign(hist.begin(), hist.begin() + 3 * P);
        have_old = true;
        if (out_scalars) {
            long long csum = 0;
            for (long long i = 0; i < n; i++) csum += C[i];
            out_scalars[3 * st] = mz;
            out_scalars[3 * st + 1] = (double)(csum / 2);
            out_scalars[3 * st + 2] = (double)P;
        }
    }
    if (last_force) memcpy(last_force, F.data(), 3 * n * sizeof(double));
    if (last_torque) memcpy(last_torque, T.data(), 3 * n * sizeof(double));
    if (last_contacts) memcpy(last_contacts, C.data(), n * sizeof(uint));
    if (out_P) *out_P = P;
    if (out_off) memcpy(out_off, off.data(), (n + 1) * sizeof(uint));
    if (out_ln && P) memcpy(out_ln, ln.data(), P * sizeof(uint));
    if (out_hist && P) memcpy(out_hist, hist.data(), 3 * P * sizeof(double));
    return status;
}

/* Poured packing: the reference's layer injection (dempacking.cu:376-461).
 * The arrays hold all ntot particles; entries from N on are the injection
 * states of particles not yet in the system, N starting at n_active.  Before
 * step it (1-based; time = dt*it, :375-376): while N < ntot and
 * time > (float)N*tnewpar/float(nplayer) (:379-381) the next nplayer
 * particles join (N += nplayer, capped at ntot: :459-460) and the step
 * re-lists (m_hiall = 1: :461); the fixed re-list cadence restarts there.
 * A new particle brings no tangential history: its rows of the previous list
 * are empty (the reference re-uploads its old-list arrays with the new count,
 * :522-533, leaving the new rows to whatever the host arrays held; empty rows
 * are the physical reading).  out_nact (if not NULL): N of each step.
 * Returns 0, 3 (pair capacity) or 5 (skin violation). */
int orc_run_pour(long long ntot, double* pos, double* pdis, double* angv, const double* rad, double* whist,
                 const double* world, const double* params, const double* mat, int fp32_list,
                 long long nsteps, int interval, long long cap, long long nplayer, double tnewpar,
                 long long n_active, long long* out_nact, double* out_scalars,
                 uint* out_off, uint* out_ln, double* out_hist, long long* out_P)
{
    const double dt = params[0], skin = params[1], cs = params[2], density = params[3];
    OContact pp{mat[0], mat[1], mat[2], mat[3], mat[4], mat[5], mat[6]};
    OContact pw{mat[7], mat[8], mat[9], mat[10], mat[11], mat[12], mat[13]};
    std::vector<double> q(3 * ntot, 0.0), F(3 * ntot), T(3 * ntot);
    std::vector<uint> C(ntot);
    std::vector<uint> off(ntot + 1, 0), ln, ooff(ntot + 1, 0), oln;
    std::vector<double> hist, ohist;
    long long P = 0, N = n_active;
    int status = 0, win = 0;
    bool have_old = false;
    for (long long st = 0; st < nsteps; st++) {
        const double time = dt * (double)(st + 1);
        if (N < ntot && time > (double)(float)N * tnewpar / (double)(float)nplayer) {
            const long long nn = std::min(N + nplayer, ntot);
            for (long long i = N + 1; i <= nn; i++) ooff[i] = ooff[N];   /* empty old rows */
            N = nn;
            win = 0;
        }
        OState s{N, pos, pdis, angv, const_cast<double*>(rad), whist, q.data()};
        if (win == 0) {
            ln.assign(cap > 0 ? cap : 1, 0);
            hist.assign(3 * (cap > 0 ? cap : 1), 0.0);
            int mr;
            long long got = orc_build_list(N, pos, rad, world, cs, skin, fp32_list,
                                           have_old ? ooff.data() : nullptr, have_old ? oln.data() : nullptr,
                                           have_old ? ohist.data() : nullptr,
                                           off.data(), ln.data(), hist.data(), cap, &mr);
            if (got < 0) return 3;
            P = got;
            std::fill(q.begin(), q.end(), 0.0);
        }
        engine_forces(s, world, dt, density, pp, pw, P, off.data(), ln.data(), hist.data(),
                      F.data(), T.data(), C.data());
        double mz;
        int viol;
        engine_integrate(s, dt, density, F.data(), T.data(), skin, &mz, &viol);
        if (viol && !status) status = 5;
        ooff = off;
        oln.assign(ln.begin(), ln.begin() + P);
        ohist.assign(hist.begin(), hist.begin() + 3 * P);
        have_old = true;
        win = (win + 1) % interval;
        if (out_nact) out_nact[st] = N;
        if (out_scalars) {
            long long csum = 0;
            for (long long i = 0; i < N; i++) csum += C[i];
            out_scalars[3 * st] = mz;
            out_scalars[3 * st + 1] = (double)(csum / 2);
            out_scalars[3 * st + 2] = (double)P;
        }
    }
    if (out_P) *out_P = P;
    if (out_off) memcpy(out_off, off.data(), (N + 1) * sizeof(uint));
    if (out_ln && P) memcpy(out_ln, ln.data(), P * sizeof(uint));
    if (out_hist && P) memcpy(out_hist, hist.data(), 3 * P * sizeof(double));
    return status;
}

/* One force evaluation (no integration) for a freshly built list: forces,
 * torques and contact counts per particle; wall history and pair history
 * start from zero.  Used for first-step force parity. */
int orc_forces_once(long long n, const double* pos, const double* pdis, const double* angv, const double* rad,
                    const double* world, const double* params, const double* mat, int fp32_list, long long cap,
                    double* force, double* torque, uint* contacts, long long* npairs)
{
    const double dt = params[0], skin = params[1], cs = params[2], density = params[3];
    OContact pp{mat[0], mat[1], mat[2], mat[3], mat[4], mat[5], mat[6]};
    OContact pw{mat[7], mat[8], mat[9], mat[10], mat[11], mat[12], mat[13]};
    std::vector<uint> off(n + 1), ln(cap > 0 ? cap : 1);
    std::vector<double> hist(3 * (cap > 0 ? cap : 1), 0.0), wh(3 * n, 0.0), q(3 * n, 0.0);
    int mr;
    long long P = orc_build_list(n, pos, rad, world, cs, skin, fp32_list, nullptr, nullptr, nullptr,
                                 off.data(), ln.data(), hist.data(), cap, &mr);
    if (P < 0) return 3;
    OState s{n, const_cast<double*>(pos), const_cast<double*>(pdis), const_cast<double*>(angv),
             const_cast<double*>(rad), wh.data(), q.data()};
    engine_forces(s, world, dt, density, pp, pw, P, off.data(), ln.data(), hist.data(), force, torque, contacts);
    if (npairs) *npairs = P;
    return 0;
}

/* Stateful engine handle for step-by-step CPU timing (the CPU baseline):
 * same loop as orc_run, state kept between calls. */
struct OEngine {
    long long n, cap, step;
    int interval, fp32;
    double world[3], params[4];
    OContact pp, pw;
    std::vector<double> pos, pdis, angv, rad, wh, q, F, T;
    std::vector<uint> C, off, ln, ooff, oln;
    std::vector<double> hist, ohist;
    long long P;
    bool have_old;
};

void* orc_engine_new(long long n, const double* pos, const double* pdis, const double* angv, const double* rad,
                     const double* world, const double* params, const double* mat, int fp32_list, int interval,
                     long long cap)
{
    OEngine* e = new OEngine();
    e->n = n; e->cap = cap; e->step = 0; e->interval = interval; e->fp32 = fp32_list;
    for (int c = 0; c < 3; c++) e->world[c] = world[c];
    for (int c = 0; c < 4; c++) e->params[c] = params[c];
    e->pp = OContact{mat[0], mat[1], mat[2], mat[3], mat[4], mat[5], mat[6]};
    e->pw = OContact{mat[7], mat[8], mat[9], mat[10], mat[11], mat[12], mat[13]};
    e->pos.assign(pos, pos + 3 * n);
    e->pdis = pdis ? std::vector<double>(pdis, pdis + 3 * n) : std::vector<double>(3 * n, 0.0);
    e->angv = angv ? std::vector<double>(angv, angv + 3 * n) : std::vector<double>(3 * n, 0.0);
    e->rad.assign(rad, rad + n);
    e->wh.assign(3 * n, 0.0); e->q.assign(3 * n, 0.0); e->F.assign(3 * n, 0.0); e->T.assign(3 * n, 0.0);
    e->C.assign(n, 0); e->off.assign(n + 1, 0); e->ooff.assign(n + 1, 0);
    e->P = 0; e->have_old = false;
    return e;
}

int orc_engine_step(void* h, long long nsteps, double* maxhz_out)
{
    OEngine* e = (OEngine*)h;
    const double dt = e->params[0], skin = e->params[1], cs = e->params[2], density = e->params[3];
    OState s{e->n, e->pos.data(), e->pdis.data(), e->angv.data(), e->rad.data(), e->wh.data(), e->q.data()};
    int status = 0;
    for (long long k = 0; k < nsteps; k++, e->step++) {
        if (e->step % e->interval == 0) {
            e->ln.assign(e->cap, 0);
            e->hist.assign(3 * e->cap, 0.0);
            int mr;
            long long got = orc_build_list(e->n, e->pos.data(), e->rad.data(), e->world, cs, skin, e->fp32,
                                           e->have_old ? e->ooff.data() : nullptr, e->have_old ? e->oln.data() : nullptr,
                                           e->have_old ? e->ohist.data() : nullptr, e->off.data(), e->ln.data(),
                                           e->hist.data(), e->cap, &mr);
            if (got < 0) return 3;
            e->P = got;
            std::fill(e->q.begin(), e->q.end(), 0.0);
        }
        engine_forces(s, e->world, dt, density, e->pp, e->pw, e->P, e->off.data(), e->ln.data(), e->hist.data(),
                      e->F.data(), e->T.data(), e->C.data());
        double mz;
        int viol;
        engine_integrate(s, dt, density, e->F.data(), e->T.data(), skin, &mz, &viol);
        if (viol && !status) status = 5;
        if (maxhz_out) *maxhz_out = mz;
        e->ooff = e->off;
        e->oln.assign(e->ln.begin(), e->ln.begin() + e->P);
        e->ohist.assign(e->hist.begin(), e->hist.begin() + 3 * e->P);
        e->have_old = true;
    }
    return status;
}

void orc_engine_free(void* h) { delete (OEngine*)h; }

} /* extern "C" */
