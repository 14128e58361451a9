/*
 * ref_golden.cu -- TEST INFRASTRUCTURE: runs the reference's own CUDA kernels
 * (compiled in place from the reference's neiglist.cu, never copied) on
 * seeded inputs and dumps inputs and outputs as raw binary golden vectors.
 *
 * The reference cannot be built as a program (its force laws, four kernels and
 * the SDK sort/scan are missing), but neiglist.cu compiles once the two
 * missing device functions have stand-ins.  The stand-ins below report "no
 * contact" / "no wall hit", so the kernels that call them exercise only their
 * own bookkeeping: calculateforcepairD's zeroing and old-list writes
 * (neiglist.cu:211-231) and calculateforceiwD's gravity and history reset
 * (neiglist.cu:263-304).  calcHashD, findCellStartD, addTwoArraysD,
 * updatepositionD, vprojec and vscale run unchanged.
 *
 * Build (oracle/Makefile target ref): nvcc -I stub_include -I <reference dir>.
 * Run:   ref_golden <outdir>   (needs a GPU; writes <outdir>/<name>.bin and
 *        <outdir>/manifest.txt).  tests/golden/make_ref_golden.py packs the
 *        result into tests/golden/ref_kernels.npz.
 */
#include <cuda_runtime.h>
#include <vector_types.h>
#include <vector_functions.h>

/* Stand-ins for the force laws that the reference calls but does not contain
 * (neiglist.cu:208 and :287).  Signatures follow the call sites. */
__device__ void calforceij(double3, double3, double3, double3, double3, double3,
                           double, double, double, double, double3, double, double,
                           double3* olddispti, double* oldfricpi, unsigned int* icontacti,
                           double3* fi, double3* ti, double3* tj)
{
    *olddispti = make_double3(0.0, 0.0, 0.0);
    *oldfricpi = 0.0;
    *icontacti = 0;
    *fi = make_double3(0.0, 0.0, 0.0);
    *ti = make_double3(0.0, 0.0, 0.0);
    *tj = make_double3(0.0, 0.0, 0.0);
}
__device__ void calforceiw(double3, double3, double3, double3, double, double, double3, double, double,
                           double3* dptiw, double* fciw, double3* forceiw, double3* toriw, short* ihit)
{
    *dptiw = make_double3(0.0, 0.0, 0.0);
    *fciw = 0.0;
    *forceiw = make_double3(0.0, 0.0, 0.0);
    *toriw = make_double3(0.0, 0.0, 0.0);
    *ihit = 0;
}

#include "neiglist.cu"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <string>
#include <vector>

static uint64_t g_state = 0x5DEECE66Dull;
static double urand() {           /* SplitMix64 -> [0,1) */
    uint64_t z = (g_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
static double uni(double a, double b) { return a + (b - a) * urand(); }

static std::string g_out;
static FILE* g_manifest;
template <typename T>
static void dump(const char* name, const char* dtype, const std::vector<T>& v) {
    std::string p = g_out + "/" + name + ".bin";
    FILE* f = fopen(p.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", p.c_str()); exit(1); }
    fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
    fprintf(g_manifest, "%s %s %zu\n", name, dtype, v.size());
}
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); exit(2); } } while (0)

template <typename T> static T* dev(const std::vector<T>& h) {
    T* d; CK(cudaMalloc(&d, h.size() * sizeof(T) + 16));
    CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}
template <typename T> static void back(std::vector<T>& h, const T* d) {
    CK(cudaMemcpy(h.data(), d, h.size() * sizeof(T), cudaMemcpyDeviceToHost));
}

__global__ void k_vprojec(int m, const double3* p, const double3* u, double3* r0, double3* r1) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        double3 a, b;
        vprojec(p[i], u[i], &a, 0);
        vprojec(p[i], u[i], &b, 1);
        r0[i] = a; r1[i] = b;
    }
}
__global__ void k_vscale(int m, double3* v, const double* p1, const double* p2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) { double3 t = v[i]; vscale(&t, p1[i], p2[i]); v[i] = t; }
}

int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: ref_golden <outdir>\n"); return 1; }
    g_out = argv[1];
    g_manifest = fopen((g_out + "/manifest.txt").c_str(), "w");
    if (!g_manifest) { fprintf(stderr, "cannot open manifest in %s\n", argv[1]); return 1; }

    /* ---------------------------------------------------------- hashing */
    const int n = 6000;
    const double origin[3] = {-10.0, -10.0, 0.0}, csz[3] = {1.55, 1.55, 1.55}, wsz[3] = {20.0, 20.0, 40.0};
    const unsigned gs[3] = {(unsigned)((int)(wsz[0] / csz[0]) + 1), (unsigned)((int)(wsz[1] / csz[1]) + 1),
                            (unsigned)((int)(wsz[2] / csz[2]) + 1)};
    std::vector<double> pos(3 * n);
    for (int i = 0; i < n; i++) {       /* some particles outside the grid on every side */
        pos[3 * i] = uni(-11.0, 11.0);
        pos[3 * i + 1] = uni(-11.0, 11.0);
        pos[3 * i + 2] = uni(-1.5, 42.0);
    }
    std::vector<unsigned> hash(2 * n);
    double* d_pos = dev(pos);
    unsigned* d_hash; CK(cudaMalloc(&d_hash, 2 * n * sizeof(unsigned)));
    calcHashD<<<(n + 255) / 256, 256>>>(n, (double3*)d_pos, (uint2*)d_hash, make_uint3(gs[0], gs[1], gs[2]),
                                        make_double3(csz[0], csz[1], csz[2]),
                                        make_double3(origin[0], origin[1], origin[2]));
    CK(cudaGetLastError());
    back(hash, d_hash);
    dump("hash_pos", "f8", pos);
    dump("hash_out", "u4", hash);
    std::vector<unsigned> grid = {gs[0], gs[1], gs[2]};
    dump("hash_grid", "u4", grid);

    /* --------------------------------------------------- findCellStart */
    std::vector<std::pair<unsigned, unsigned>> kv(n);
    for (int i = 0; i < n; i++) kv[i] = {hash[2 * i], hash[2 * i + 1]};
    std::stable_sort(kv.begin(), kv.end(), [](const std::pair<unsigned, unsigned>& a,
                                              const std::pair<unsigned, unsigned>& b) { return a.first < b.first; });
    std::vector<unsigned> sorted(2 * n);
    for (int i = 0; i < n; i++) { sorted[2 * i] = kv[i].first; sorted[2 * i + 1] = kv[i].second; }
    const unsigned ncells = gs[0] * gs[1] * gs[2];
    std::vector<unsigned> cstart(ncells);
    unsigned* d_sorted = dev(sorted);
    unsigned* d_cs; CK(cudaMalloc(&d_cs, ncells * sizeof(unsigned)));
    CK(cudaMemset(d_cs, 0xff, ncells * sizeof(unsigned)));
    findCellStartD<<<(n + 255) / 256, 256>>>((uint2*)d_sorted, d_cs, n, ncells);
    CK(cudaGetLastError());
    back(cstart, d_cs);
    dump("cell_sorted", "u4", sorted);
    dump("cell_start", "u4", cstart);

    /* --------------------------------------------------- addTwoArrays */
    const int na = 5000;
    std::vector<unsigned> a(na), b(na);
    for (int i = 0; i < na; i++) { a[i] = (unsigned)(urand() * 1000); b[i] = (unsigned)(urand() * 100000); }
    unsigned* d_a = dev(a); unsigned* d_b = dev(b);
    addTwoArraysD<<<(na + 255) / 256, 256>>>(d_b, d_a, na);
    CK(cudaGetLastError());
    std::vector<unsigned> bo(na);
    back(bo, d_b);
    dump("add_a", "u4", a); dump("add_b", "u4", b); dump("add_out", "u4", bo);

    /* -------------------------------------------------- updatepositionD */
    const int nu = 5000;   /* not a multiple of 256: padding threads in the last block */
    std::vector<double> up(3 * nu), ud(3 * nu), ua(3 * nu), uf(3 * nu), ut(3 * nu), uq(3 * nu), um(nu), ui(nu);
    for (int i = 0; i < nu; i++) {
        double r = uni(0.3, 0.8);
        um[i] = 8.0 * r * r * r;
        ui[i] = 0.4 * um[i] * r * r;
        up[3 * i] = uni(-9.0, 9.0); up[3 * i + 1] = uni(-9.0, 9.0); up[3 * i + 2] = uni(0.5, 30.0);
        for (int c = 0; c < 3; c++) {
            ud[3 * i + c] = uni(-1e-3, 1e-3);
            ua[3 * i + c] = uni(-1e-3, 1e-3);
            uf[3 * i + c] = uni(-50.0, 50.0);
            ut[3 * i + c] = uni(-5.0, 5.0);
            uq[3 * i + c] = uni(-0.2, 0.2);
        }
    }
    const double udt = 1e-3, ucdamp = 0.3;
    const int nb = (nu + 255) / 256;
    double *dp = dev(up), *dd = dev(ud), *da = dev(ua), *df = dev(uf), *dtq = dev(ut), *dq = dev(uq), *dm = dev(um),
           *di = dev(ui);
    unsigned* d_iall; double* d_mz;
    CK(cudaMalloc(&d_iall, nb * sizeof(unsigned))); CK(cudaMalloc(&d_mz, nb * sizeof(double)));
    CK(cudaMemset(d_iall, 0, nb * sizeof(unsigned))); CK(cudaMemset(d_mz, 0, nb * sizeof(double)));
    updatepositionD<<<nb, 256>>>(make_double3(20.0, 20.0, 40.0), nu, (double3*)dp, (double3*)dd, (double3*)da, dm, di,
                                 (double3*)df, (double3*)dtq, (double3*)dq, udt, ucdamp, d_iall, d_mz);
    CK(cudaGetLastError());
    dump("upd_pos_in", "f8", up); dump("upd_pdis_in", "f8", ud); dump("upd_angv_in", "f8", ua);
    dump("upd_force", "f8", uf); dump("upd_torque", "f8", ut); dump("upd_qi_in", "f8", uq);
    dump("upd_rmass", "f8", um); dump("upd_inert", "f8", ui);
    std::vector<double> sc = {udt, ucdamp};
    dump("upd_scalars", "f8", sc);
    back(up, dp); back(ud, dd); back(ua, da); back(uq, dq);
    std::vector<unsigned> piall(nb); std::vector<double> pmz(nb);
    back(piall, d_iall); back(pmz, d_mz);
    dump("upd_pos_out", "f8", up); dump("upd_pdis_out", "f8", ud); dump("upd_angv_out", "f8", ua);
    dump("upd_qi_out", "f8", uq); dump("upd_part_iall", "u4", piall); dump("upd_part_maxhz", "f8", pmz);

    /* ------------------------------------------------- vprojec / vscale */
    const int m = 4096;
    std::vector<double> vp(3 * m), vu(3 * m), vr0(3 * m), vr1(3 * m), s1(m), s2(m), vs(3 * m);
    for (int i = 0; i < m; i++) {
        double u[3] = {uni(-1, 1), uni(-1, 1), uni(-1, 1)};
        double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        double scale = (i % 4 == 0) ? 1e-4 : ((i % 4 == 1) ? 1e-2 : 1.0);
        for (int c = 0; c < 3; c++) { vu[3 * i + c] = u[c] / l; vp[3 * i + c] = scale * uni(-1, 1); }
        if (i % 16 == 3) for (int c = 0; c < 3; c++) vp[3 * i + c] = 0.7 * vu[3 * i + c] + 1e-4 * uni(-1, 1);
        s1[i] = uni(0.1, 2.0); s2[i] = uni(0.1, 2.0);
        for (int c = 0; c < 3; c++) vs[3 * i + c] = uni(-1, 1);
    }
    double *dvp = dev(vp), *dvu = dev(vu), *dr0 = dev(vr0), *dr1 = dev(vr1), *dvs = dev(vs), *ds1 = dev(s1), *ds2 = dev(s2);
    k_vprojec<<<(m + 255) / 256, 256>>>(m, (double3*)dvp, (double3*)dvu, (double3*)dr0, (double3*)dr1);
    k_vscale<<<(m + 255) / 256, 256>>>(m, (double3*)dvs, ds1, ds2);
    CK(cudaGetLastError());
    dump("vp_p", "f8", vp); dump("vp_u", "f8", vu); dump("vs_in", "f8", vs); dump("vs_p1", "f8", s1); dump("vs_p2", "f8", s2);
    back(vr0, dr0); back(vr1, dr1); back(vs, dvs);
    dump("vp_r0", "f8", vr0); dump("vp_r1", "f8", vr1); dump("vs_out", "f8", vs);

    /* ------------------------------- calculateforceiwD (no wall touched) */
    const int nw = 3000;
    std::vector<double> wp(3 * nw), wd(3 * nw), wa(3 * nw), wr(nw), wm(nw), wf(3 * nw), wt(3 * nw), wdw(3 * nw), wfw(nw);
    for (int i = 0; i < nw; i++) {
        wr[i] = uni(0.3, 0.8); wm[i] = 8.0 * wr[i] * wr[i] * wr[i];
        wp[3 * i] = uni(-8.0, 8.0); wp[3 * i + 1] = uni(-8.0, 8.0); wp[3 * i + 2] = uni(1.0, 30.0);
        for (int c = 0; c < 3; c++) {
            wd[3 * i + c] = uni(-1e-3, 1e-3); wa[3 * i + c] = uni(-1e-3, 1e-3);
            wf[3 * i + c] = uni(-5, 5); wt[3 * i + c] = uni(-1, 1); wdw[3 * i + c] = uni(-1e-4, 1e-4);
        }
        wfw[i] = uni(0, 1);
    }
    dump("wall_pos", "f8", wp); dump("wall_pdis", "f8", wd); dump("wall_angv", "f8", wa); dump("wall_rad", "f8", wr);
    dump("wall_rmass", "f8", wm); dump("wall_force_in", "f8", wf); dump("wall_torque_in", "f8", wt);
    dump("wall_disptw_in", "f8", wdw); dump("wall_fricpw_in", "f8", wfw);
    for (int pass = 0; pass < 2; pass++) {
        unsigned total = pass == 0 ? 0u : 7u;
        double *xp = dev(wp), *xd = dev(wd), *xa = dev(wa), *xr = dev(wr), *xm = dev(wm), *xf = dev(wf), *xt = dev(wt),
               *xdw = dev(wdw), *xfw = dev(wfw);
        calculateforceiwD<<<(nw + 255) / 256, 256>>>(nw, make_double3(20.0, 20.0, 40.0), (double3*)xp, (double3*)xd,
                                                     (double3*)xa, xr, xm, 1e-3, total, (double3*)xdw, xfw,
                                                     (double3*)xf, (double3*)xt);
        CK(cudaGetLastError());
        std::vector<double> of(3 * nw), ot(3 * nw), odw(3 * nw), ofw(nw);
        back(of, xf); back(ot, xt); back(odw, xdw); back(ofw, xfw);
        std::string s = pass == 0 ? "_t0" : "_t7";
        dump(("wall_force_out" + s).c_str(), "f8", of); dump(("wall_torque_out" + s).c_str(), "f8", ot);
        dump(("wall_disptw_out" + s).c_str(), "f8", odw); dump(("wall_fricpw_out" + s).c_str(), "f8", ofw);
    }

    /* ---------------------------- calculateforcepairD (no pair touching) */
    const int np = 2000, P = 3000;
    std::vector<double> pp(3 * np), pd(3 * np), pa(3 * np), pr(np), pm(np);
    for (int i = 0; i < np; i++) {
        pr[i] = 0.5; pm[i] = 1.0;
        pp[3 * i] = 2.0 * (i % 10); pp[3 * i + 1] = 2.0 * ((i / 10) % 10); pp[3 * i + 2] = 2.0 * (i / 100) + 1.0;
        for (int c = 0; c < 3; c++) { pd[3 * i + c] = uni(-1e-3, 1e-3); pa[3 * i + c] = uni(-1e-3, 1e-3); }
    }
    std::vector<unsigned> lp(P), ln(P), oln(P, 12345u), cp(P, 7u);
    std::vector<double> dsp(3 * P), frp(P), odsp(3 * P, 9.0), ofrp(P, 9.0), fp(3 * P, 9.0), tpi(3 * P, 9.0), tpj(3 * P, 9.0);
    for (int k = 0; k < P; k++) {
        unsigned i = (unsigned)(urand() * (np - 1)), j = i + 1 + (unsigned)(urand() * (np - 1 - i));
        lp[k] = i; ln[k] = j;
        for (int c = 0; c < 3; c++) dsp[3 * k + c] = uni(-1e-4, 1e-4);
        frp[k] = uni(0, 1);
    }
    dump("pair_lp", "u4", lp); dump("pair_ln", "u4", ln); dump("pair_dispt_in", "f8", dsp); dump("pair_fricp_in", "f8", frp);
    double *qp = dev(pp), *qd = dev(pd), *qa = dev(pa), *qr = dev(pr), *qm = dev(pm), *qds = dev(dsp), *qfr = dev(frp),
           *qods = dev(odsp), *qofr = dev(ofrp), *qfp = dev(fp), *qti = dev(tpi), *qtj = dev(tpj);
    unsigned *qlp = dev(lp), *qln = dev(ln), *qoln = dev(oln), *qcp = dev(cp);
    calculateforcepairD<<<(P + 255) / 256, 256>>>(P, (double3*)qp, (double3*)qd, (double3*)qa, qr, qm, qlp, qln, qoln,
                                                 (double3*)qds, qfr, (double3*)qods, qofr, 1e-3, (double3*)qfp,
                                                 (double3*)qti, (double3*)qtj, qcp);
    CK(cudaGetLastError());
    back(dsp, qds); back(frp, qfr); back(odsp, qods); back(ofrp, qofr); back(fp, qfp); back(tpi, qti); back(tpj, qtj);
    back(oln, qoln); back(cp, qcp);
    dump("pair_pos", "f8", pp);
    dump("pair_dispt_out", "f8", dsp); dump("pair_fricp_out", "f8", frp); dump("pair_olddispt_out", "f8", odsp);
    dump("pair_oldfricp_out", "f8", ofrp); dump("pair_force_out", "f8", fp); dump("pair_tpi_out", "f8", tpi);
    dump("pair_tpj_out", "f8", tpj); dump("pair_oldln_out", "u4", oln); dump("pair_contact_out", "u4", cp);

    CK(cudaDeviceSynchronize());
    fclose(g_manifest);
    printf("ref_golden: wrote golden vectors to %s\n", argv[1]);
    return 0;
}
