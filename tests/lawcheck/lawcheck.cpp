// Host build of the library's contact-law headers, for testing the hand-written
// reverse mode against finite differences on the CPU (test helper only).
#include "dem_law_adj.cuh"

using namespace dem;

static LawParams<double> par(const double* p7) {
    dem_contact c{p7[0], p7[1], p7[2], p7[3], p7[4], p7[5], p7[6]};
    return make_law<double>(c);
}
static V3d v(const double* a) { return mk(a[0], a[1], a[2]); }
static void put(double* o, V3d a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; }

extern "C" {
// in: xi xj di dj ai aj (6x3) ri rj h(3) = 23 ; out: Fi Ti Tj h (12)
int lc_pair_fwd(const double* in, const double* p7, double inv_dt, double density, double* out) {
    PairTape t;
    V3d Fi, Ti, Tj, ho;
    int c = pair_fwd(v(in), v(in + 3), v(in + 6), v(in + 9), v(in + 12), v(in + 15), in[18], in[19], v(in + 20),
                     par(p7), inv_dt, density, t, Fi, Ti, Tj, ho);
    put(out, Fi); put(out + 3, Ti); put(out + 6, Tj); put(out + 9, ho);
    return c;
}
void lc_pair_vjp(const double* in, const double* p7, double inv_dt, double density, const double* ob, double* ib,
                 double* pbar) {
    PairTape t;
    V3d Fi, Ti, Tj, ho;
    LawParams<double> p = par(p7);
    pair_fwd(v(in), v(in + 3), v(in + 6), v(in + 9), v(in + 12), v(in + 15), in[18], in[19], v(in + 20), p, inv_dt,
             density, t, Fi, Ti, Tj, ho);
    V3d xib = zero3<double>(), xjb = xib, dib = xib, djb = xib, aib = xib, ajb = xib, hb = xib;
    double rib = 0, rjb = 0;
    LawBar pb;
    lawbar_zero(pb);
    pair_rev(t, p, inv_dt, density, v(ob), v(ob + 3), v(ob + 6), v(ob + 9), xib, xjb, dib, djb, aib, ajb, rib, rjb, hb,
             pb);
    put(ib, xib); put(ib + 3, xjb); put(ib + 6, dib); put(ib + 9, djb); put(ib + 12, aib); put(ib + 15, ajb);
    ib[18] = rib; ib[19] = rjb; put(ib + 20, hb);
    pbar[0] = pb.estar; pbar[1] = pb.mu; pbar[2] = pb.cn; pbar[3] = pb.ct; pbar[4] = pb.roll; pbar[5] = pb.roll_rel;
}
// in: x d a (3x3) r h(3) = 13 ; out: F T h (9)
int lc_wall_fwd(const double* in, double hx, double hy, const double* p7, double inv_dt, double density, double* out) {
    V3d F, T, ho;
    int c = wall_fwd(hx, hy, v(in), v(in + 3), v(in + 6), in[9], density, v(in + 10), par(p7), inv_dt, F, T, ho);
    put(out, F); put(out + 3, T); put(out + 6, ho);
    return c;
}
void lc_wall_vjp(const double* in, double hx, double hy, const double* p7, double inv_dt, double density,
                 const double* ob, double* ib, double* pbar) {
    LawParams<double> p = par(p7);
    V3d xb = zero3<double>(), db = xb, ab = xb, hb = xb;
    double rb = 0;
    LawBar pb;
    lawbar_zero(pb);
    wall_vjp(hx, hy, v(in), v(in + 3), v(in + 6), in[9], density, v(in + 10), p, inv_dt, v(ob), v(ob + 3), v(ob + 6),
             xb, db, ab, rb, hb, pb);
    put(ib, xb); put(ib + 3, db); put(ib + 6, ab); ib[9] = rb; put(ib + 10, hb);
    pbar[0] = pb.estar; pbar[1] = pb.mu; pbar[2] = pb.cn; pbar[3] = pb.ct; pbar[4] = pb.roll; pbar[5] = pb.roll_rel;
}
// the same law through the float/double template the kernels use (forward only)
int lc_pair_fwd_kernel_law(const double* in, const double* p7, double inv_dt, double density, double* out) {
    return lc_pair_fwd(in, p7, inv_dt, density, out);
}
}
