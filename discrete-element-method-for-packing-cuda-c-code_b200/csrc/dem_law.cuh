// dem_law.cuh -- the sphere contact law (host+device), templated on the
// arithmetic type of the force (F = float or double).  The tangential history
// is always FP64.
//
// The reference calls this law as calforceij / calforceiw (neiglist.cu:208,
// 287) but does not contain it.  It is the published Hertz-Mindlin model with
// viscous damping, Coulomb limit and rolling resistance (Zhou et al. 1999,
// Gan, Zhou & Yu 2016) in the reference's reduced units, with the history
// projection of vprojec (neiglist.cu:133-146, ityp = 0) and the rescale of
// vscale (neiglist.cu:148-153):
//   fn_e = estar sqrt(R*) delta^1.5
//   fn   = fn_e - cn sqrt(6 m* (3/4 estar) sqrt(R* delta)) (U.n)/dt
//   xi   = xi - (xi.n) n + U_t
//   xmax = mu (2-nu)/(2(1-nu)) delta,   s = min(|xi|, xmax)/xmax
//   Ft   = mu fn_e (1-(1-s)^1.5) xi/|xi| + ct sqrt(6 mu m* fn_e sqrt(1-s)/xmax) U_t/dt
//          |Ft| <= mu fn_e,   |xi| <= xmax
//   Mr   = -(roll + roll_rel R*) fn_e Wr/|Wr|
//   Fi   = -fn n + Ft        (force on i; n points from i to j)
// U is the per-step displacement of j's contact point relative to i's and Wr
// the per-step relative rotation a_i - a_j.
#pragma once
#include "dem_common.cuh"

namespace dem {

template <typename F> struct LawParams {
    F estar, mu, nu, cn, ct, roll, roll_rel;
    F xfac;     // mu (2-nu)/(2(1-nu))
    F cnfac;    // 4.5 * estar
};

template <typename F> inline LawParams<F> make_law(const dem_contact& c) {
    LawParams<F> p;
    p.estar = (F)c.estar; p.mu = (F)c.mu; p.nu = (F)c.nu; p.cn = (F)c.damp_n; p.ct = (F)c.damp_t;
    p.roll = (F)c.roll; p.roll_rel = (F)c.roll_rel;
    p.xfac = (F)(c.mu * (2.0 - c.nu) / (2.0 * (1.0 - c.nu)));
    p.cnfac = (F)(4.5 * c.estar);
    return p;
}

// Returns the force on i (Fi), its tangential part (Ft) and the rolling
// torque on i (Mr); xi (FP64) is updated in place.
template <typename F>
DEM_HD void contact_law(F delta, V3<F> n, F rstar, F mstar, V3<F> U, V3<F> Wr, V3<double>& xi,
                        F inv_dt, const LawParams<F>& p, V3<F>& Fi, V3<F>& Ft, V3<F>& Mr)
{
    const F sd = dsqrt(delta);
    const F fn_e = p.estar * dsqrt(rstar) * delta * sd;
    const F Un = dot(U, n);
    const F cn_c = p.cn * dsqrt(p.cnfac * mstar * dsqrt(rstar * delta));
    const F fn = fn_e - cn_c * (Un * inv_dt);
    const V3<F> Ut = U - Un * n;
    // tangential history in FP64: rotate into the current tangent plane, add U_t
    const V3<double> nd = cvt<double>(n);
    const double xn = dot(xi, nd);
    xi = (xi - xn * nd) + cvt<double>(Ut);
    if (p.mu > F(0)) {
        const F xmax = p.xfac * delta;
        // |xi| in the force's precision (FP32 in the mixed form: the history
        // itself stays FP64, its length and the slip rescale are FP32-exact)
        const double xx = dot(xi, xi);
        const double xim_d = sizeof(F) == 4 ? (double)dsqrt((F)xx) : sqrt(xx);
        const F xim = (F)xim_d;
        const F s = (xim < xmax ? xim : xmax) / xmax;
        const F oms = F(1) - s;
        const F so = dsqrt(oms);
        const F ft_e = p.mu * fn_e * (F(1) - oms * so);
        const F ct_c = p.ct * dsqrt(F(6) * p.mu * mstar * fn_e * so / xmax);
        const F el = xim > F(0) ? ft_e / xim : F(0);
        Ft = el * cvt<F>(xi) + ct_c * (Ut * inv_dt);
        const F ftm = dsqrt(dot(Ft, Ft));
        const F cap = p.mu * fn_e;
        if (ftm > cap) Ft = Ft * (cap / ftm);
        if (xim_d > (double)xmax) xi = xi * (sizeof(F) == 4 ? (double)(xmax / xim) : (double)xmax / xim_d);
    } else {
        Ft = zero3<F>();
        xi = zero3<double>();
    }
    const F rl = p.roll + p.roll_rel * rstar;
    const F w = dsqrt(dot(Wr, Wr));
    if (w > F(1e-30) && rl > F(0)) Mr = (-(rl * fn_e / w)) * Wr;
    else Mr = zero3<F>();
    Fi = (-fn) * n + Ft;
}

// Flat walls of the open box: floor z=0, x=-Wx/2, x=+Wx/2, y=-Wy/2, y=+Wy/2
// (world origin (-Wx/2,-Wy/2,0), dempacking.cu:333-339).  One FP64 history
// slot per particle (neiglist.cu:263-264,290-301) belongs to the wall with
// the largest overlap (first on a tie); other touching walls start from a
// zero history each step.  Adds the wall force/torque to F/T; returns 1 when a
// wall is touched (xi then holds the new history), 0 otherwise (xi zeroed).
template <typename F>
DEM_HD int wall_contacts(double hx, double hy, V3<double> x, V3<F> d, V3<F> a, F r, F m,
                         V3<double>& xi, F inv_dt, const LawParams<F>& p, V3<F>& Fsum, V3<F>& Tsum,
                         F* fricpw)
{
    double dl[5];
    dl[0] = (double)r - x.z;
    dl[1] = (double)r - (x.x + hx);
    dl[2] = (double)r - (hx - x.x);
    dl[3] = (double)r - (x.y + hy);
    dl[4] = (double)r - (hy - x.y);
    int prim = -1;
#pragma unroll
    for (int w = 0; w < 5; w++)
        if (dl[w] > 0.0 && (prim < 0 || dl[w] > dl[prim])) prim = w;
    if (prim < 0) {
        xi = zero3<double>();
        if (fricpw) *fricpw = F(0);
        return 0;
    }
    V3<double> newxi = zero3<double>();
    F newfr = F(0);
    // one copy of the law for all five walls (keeps the register footprint of
    // the particle kernel small; touching a wall is the rare path)
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        if (!(dl[w] > 0.0)) continue;
        V3<F> n;
        n.x = (w == 1) ? F(-1) : ((w == 2) ? F(1) : F(0));
        n.y = (w == 3) ? F(-1) : ((w == 4) ? F(1) : F(0));
        n.z = (w == 0) ? F(-1) : F(0);
        const V3<F> U = (-d) - r * cross(a, n);
        V3<double> h = (w == prim) ? xi : zero3<double>();
        V3<F> Fi, Ft, Mr;
        contact_law<F>((F)dl[w], n, r, m, U, a, h, inv_dt, p, Fi, Ft, Mr);
        Fsum += Fi;
        Tsum += r * cross(n, Ft) + Mr;
        if (w == prim) {
            newxi = h;
            newfr = dsqrt(dot(Ft, Ft));
        }
    }
    xi = newxi;
    if (fricpw) *fricpw = newfr;
    return 1;
}

}  // namespace dem
