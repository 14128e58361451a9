// dem_law_adj.cuh -- reverse mode (vector-Jacobian products) of the contact
// law, the pair geometry and the wall geometry of dem_law.cuh, hand-written,
// in FP64, host+device.  Used by the adjoint of the DEM step (dem_adjoint.cu).
//
// Convention: for a primal y = f(x) and an output adjoint yb, the reverse
// functions ADD x's adjoint contributions into the "...b" arguments.
// Non-smooth points (contact on/off, stick/slip, Coulomb limit, primary wall)
// take the branch of the primal at the evaluation point.
#pragma once
#include "dem_law.cuh"

namespace dem {

typedef V3<double> V3d;

// Adjoints of the contact parameters (xfac = mu(2-nu)/(2(1-nu)) and
// cnfac = 4.5 estar are folded back into mu and estar).
struct LawBar {
    double estar, mu, cn, ct, roll, roll_rel;
};

DEM_HD void lawbar_zero(LawBar& b) { b.estar = b.mu = b.cn = b.ct = b.roll = b.roll_rel = 0.0; }


// Intermediates of one evaluation of the law, kept for the reverse sweep.
struct LawTape {
    double delta, rs, ms, sd, srs, fne, Un, q, g, sqg, cnc, fn;
    V3d n, U, Wr, Ut, h_in, h1, Ft0, Ft;
    double xn, xmax, xim, s, oms, so, fte, A, G, sqG, ctc, el, ftm, cap;
    int slip, capped, hclip, tang;
    double rl, w;
    int roll_on;
};

// Primal (FP64) with tape.  Same arithmetic as contact_law<double>.
DEM_HD void law_fwd(double delta, V3d n, double rs, double ms, V3d U, V3d Wr, V3d h_in, double inv_dt,
                    const LawParams<double>& p, LawTape& t, V3d& Fi, V3d& Ft, V3d& Mr, V3d& h_out) {
    t.delta = delta; t.n = n; t.rs = rs; t.ms = ms; t.U = U; t.Wr = Wr; t.h_in = h_in;
    t.sd = sqrt(delta);
    t.srs = sqrt(rs);
    t.fne = p.estar * t.srs * delta * t.sd;
    t.Un = dot(U, n);
    t.q = sqrt(rs * delta);
    t.g = p.cnfac * ms * t.q;
    t.sqg = sqrt(t.g);
    t.cnc = p.cn * t.sqg;
    t.fn = t.fne - t.cnc * (t.Un * inv_dt);
    t.Ut = U - t.Un * n;
    t.xn = dot(h_in, n);
    t.h1 = (h_in - t.xn * n) + t.Ut;
    t.tang = p.mu > 0.0;
    if (t.tang) {
        t.xmax = p.xfac * delta;
        t.xim = sqrt(dot(t.h1, t.h1));
        t.slip = !(t.xim < t.xmax);
        t.s = t.slip ? 1.0 : t.xim / t.xmax;
        t.oms = 1.0 - t.s;
        t.so = sqrt(t.oms);
        t.fte = p.mu * t.fne * (1.0 - t.oms * t.so);
        t.A = 6.0 * p.mu * ms * t.fne * t.so;
        t.G = t.A / t.xmax;
        t.sqG = sqrt(t.G);
        t.ctc = p.ct * t.sqG;
        t.el = t.xim > 0.0 ? t.fte / t.xim : 0.0;
        t.Ft0 = t.el * t.h1 + t.ctc * (t.Ut * inv_dt);
        t.ftm = sqrt(dot(t.Ft0, t.Ft0));
        t.cap = p.mu * t.fne;
        t.capped = t.ftm > t.cap;
        t.Ft = t.capped ? t.Ft0 * (t.cap / t.ftm) : t.Ft0;
        t.hclip = t.xim > t.xmax;
        h_out = t.hclip ? t.h1 * (t.xmax / t.xim) : t.h1;
    } else {
        t.Ft = zero3<double>();
        h_out = zero3<double>();
    }
    Ft = t.Ft;
    t.rl = p.roll + p.roll_rel * rs;
    t.w = sqrt(dot(Wr, Wr));
    t.roll_on = (t.w > 1e-30 && t.rl > 0.0);
    Mr = t.roll_on ? (-(t.rl * t.fne / t.w)) * Wr : zero3<double>();
    Fi = (-t.fn) * n + t.Ft;
}

// Reverse of law_fwd.  Fib/Ftb/Mrb/hb: adjoints of Fi, Ft (as used outside
// the law, e.g. in torques), Mr and h_out.
DEM_HD void law_rev(const LawTape& t, const LawParams<double>& p, double inv_dt, V3d Fib, V3d Ftb, V3d Mrb, V3d hb,
                    double& deltab, V3d& nb, double& rsb, double& msb, V3d& Ub, V3d& Wrb, V3d& hinb, LawBar& pb) {
    const V3d n = t.n;
    // Fi = -fn n + Ft
    const double fnb = -dot(Fib, n);
    nb += (-t.fn) * Fib;
    Ftb += Fib;
    double fneb = 0.0;
    // Mr = -(rl fne / w) Wr
    if (t.roll_on) {
        const double c = t.rl * t.fne / t.w;
        const double cb = -dot(Mrb, t.Wr);
        Wrb += (-c) * Mrb;
        const double rlb = cb * t.fne / t.w;
        fneb += cb * t.rl / t.w;
        const double wb = -cb * t.rl * t.fne / (t.w * t.w);
        Wrb += (wb / t.w) * t.Wr;
        pb.roll += rlb;
        pb.roll_rel += rlb * t.rs;
        rsb += rlb * p.roll_rel;
    }
    V3d Utb = zero3<double>();
    V3d h1b = zero3<double>();
    if (t.tang) {
        double xmaxb = 0.0, ximb = 0.0;
        // h_out
        if (t.hclip) {
            const double k = t.xmax / t.xim;
            h1b += k * hb;
            const double kb = dot(hb, t.h1);
            xmaxb += kb / t.xim;
            ximb += -kb * t.xmax / (t.xim * t.xim);
        } else {
            h1b += hb;
        }
        // Ft = capped(Ft0)
        V3d Ft0b;
        if (t.capped) {
            const double k2 = t.cap / t.ftm;
            Ft0b = k2 * Ftb;
            const double k2b = dot(Ftb, t.Ft0);
            const double capb = k2b / t.ftm;
            const double ftmb = -k2b * t.cap / (t.ftm * t.ftm);
            Ft0b += (ftmb / t.ftm) * t.Ft0;
            pb.mu += capb * t.fne;
            fneb += capb * p.mu;
        } else {
            Ft0b = Ftb;
        }
        // Ft0 = el h1 + ctc inv_dt Ut
        const double elb = dot(Ft0b, t.h1);
        h1b += t.el * Ft0b;
        const double ctcb = inv_dt * dot(Ft0b, t.Ut);
        Utb += (t.ctc * inv_dt) * Ft0b;
        // el = fte / xim
        double fteb = 0.0;
        if (t.xim > 0.0) {
            fteb += elb / t.xim;
            ximb += -elb * t.fte / (t.xim * t.xim);
        }
        double sob = 0.0;
        // ctc = ct sqrt(G), G = A / xmax, A = 6 mu ms fne so (zero at full slip)
        if (t.G > 0.0) {
            pb.ct += ctcb * t.sqG;
            const double Gb = ctcb * p.ct / (2.0 * t.sqG);
            const double Ab = Gb / t.xmax;
            xmaxb += -Gb * t.A / (t.xmax * t.xmax);
            pb.mu += Ab * 6.0 * t.ms * t.fne * t.so;
            msb += Ab * 6.0 * p.mu * t.fne * t.so;
            fneb += Ab * 6.0 * p.mu * t.ms * t.so;
            sob += Ab * 6.0 * p.mu * t.ms * t.fne;
        }
        // fte = mu fne (1 - oms so)
        const double om = 1.0 - t.oms * t.so;
        pb.mu += fteb * t.fne * om;
        fneb += fteb * p.mu * om;
        double omsb = -fteb * p.mu * t.fne * t.so;
        sob += -fteb * p.mu * t.fne * t.oms;
        if (!t.slip) {
            // so = sqrt(oms) (oms > 0 here); s = xim / xmax
            omsb += sob / (2.0 * t.so);
            const double sbar = -omsb;
            ximb += sbar / t.xmax;
            xmaxb += -sbar * t.xim / (t.xmax * t.xmax);
        }
        // xmax = xfac delta, xfac = mu (2-nu)/(2(1-nu))
        deltab += xmaxb * p.xfac;
        pb.mu += xmaxb * t.delta * (2.0 - p.nu) / (2.0 * (1.0 - p.nu));
        // xim = |h1|
        if (t.xim > 0.0) h1b += (ximb / t.xim) * t.h1;
    }
    // h1 = h_in - xn n + Ut, xn = h_in . n
    hinb += h1b;
    const double xnb = -dot(h1b, n);
    nb += (-t.xn) * h1b;
    Utb += h1b;
    hinb += xnb * n;
    nb += xnb * t.h_in;
    // Ut = U - Un n
    Ub += Utb;
    double Unb = -dot(Utb, n);
    nb += (-t.Un) * Utb;
    // fn = fne - cnc Un inv_dt
    fneb += fnb;
    const double cncb = -fnb * t.Un * inv_dt;
    Unb += -fnb * t.cnc * inv_dt;
    // cnc = cn sqrt(g), g = 4.5 estar ms q, q = sqrt(rs delta)
    if (t.g > 0.0) {
        pb.cn += cncb * t.sqg;
        const double gb = cncb * p.cn / (2.0 * t.sqg);
        pb.estar += gb * 4.5 * t.ms * t.q;
        msb += gb * p.cnfac * t.q;
        const double qb = gb * p.cnfac * t.ms;
        if (t.q > 0.0) {
            rsb += qb * t.delta / (2.0 * t.q);
            deltab += qb * t.rs / (2.0 * t.q);
        }
    }
    // Un = U . n
    Ub += Unb * n;
    nb += Unb * t.U;
    // fne = estar srs delta sd
    pb.estar += fneb * t.srs * t.delta * t.sd;
    rsb += fneb * p.estar * t.delta * t.sd / (2.0 * t.srs);
    deltab += fneb * p.estar * t.srs * 1.5 * t.sd;
}

// Pair geometry + law (FP64) with reverse.  Inputs of pair (lo, hi); outputs
// Fi (force on lo), Ti, Tj, h_out; returns 1 when touching.
struct PairTape {
    int on;
    V3d D, n, ra, nxf;
    double dist, ri, rj, mi, mj, sr, rs, ms;
    V3d ai, aj;
    LawTape law;
};

DEM_HD int pair_fwd(V3d xi, V3d xj, V3d di, V3d dj, V3d ai, V3d aj, double ri, double rj, V3d h_in,
                    const LawParams<double>& p, double inv_dt, double density, PairTape& t, V3d& Fi, V3d& Ti,
                    V3d& Tj, V3d& h_out) {
    t.D = xj - xi;
    t.dist = sqrt(dot(t.D, t.D));
    const double delta = (ri + rj) - t.dist;
    t.on = (delta > 0.0 && t.dist > 0.0);
    if (!t.on) {
        Fi = Ti = Tj = h_out = zero3<double>();
        return 0;
    }
    t.ri = ri; t.rj = rj; t.ai = ai; t.aj = aj;
    t.n = t.D * (1.0 / t.dist);
    t.sr = ri + rj;
    t.rs = ri * rj / t.sr;
    t.mi = density * 8.0 * ri * ri * ri;
    t.mj = density * 8.0 * rj * rj * rj;
    t.ms = t.mi * t.mj / (t.mi + t.mj);
    t.ra = ri * ai + rj * aj;
    const V3d U = (dj - di) - cross(t.ra, t.n);
    V3d Ft, Mr;
    law_fwd(delta, t.n, t.rs, t.ms, U, ai - aj, h_in, inv_dt, p, t.law, Fi, Ft, Mr, h_out);
    t.nxf = cross(t.n, Ft);
    Ti = ri * t.nxf + Mr;
    Tj = rj * t.nxf - Mr;
    return 1;
}

DEM_HD void pair_rev(const PairTape& t, const LawParams<double>& p, double inv_dt, double density, V3d Fib, V3d Tib,
                     V3d Tjb, V3d hb, V3d& xib, V3d& xjb, V3d& dib, V3d& djb, V3d& aib, V3d& ajb, double& rib,
                     double& rjb, V3d& hinb, LawBar& pb) {
    if (!t.on) return;
    // Ti = ri nxf + Mr, Tj = rj nxf - Mr
    const V3d nxfb = t.ri * Tib + t.rj * Tjb;
    const V3d Mrb = Tib - Tjb;
    rib += dot(t.nxf, Tib);
    rjb += dot(t.nxf, Tjb);
    // nxf = n x Ft  ->  nb += Ft x nxfb, Ftb += nxfb x n
    const V3d Ft = t.law.Ft;
    V3d nb = cross(Ft, nxfb);
    V3d Ftb = cross(nxfb, t.n);
    double deltab = 0.0, rsb = 0.0, msb = 0.0;
    V3d Ub = zero3<double>(), Wrb = zero3<double>();
    law_rev(t.law, p, inv_dt, Fib, Ftb, Mrb, hb, deltab, nb, rsb, msb, Ub, Wrb, hinb, pb);
    // Wr = ai - aj
    aib += Wrb;
    ajb -= Wrb;
    // U = (dj - di) - ra x n  -> cb = -Ub (c = ra x n): rab += n x cb, nb += cb x ra
    djb += Ub;
    dib -= Ub;
    const V3d cb = -Ub;
    const V3d rab = cross(t.n, cb);
    nb += cross(cb, t.ra);
    // ra = ri ai + rj aj
    rib += dot(rab, t.ai);
    aib += t.ri * rab;
    rjb += dot(rab, t.aj);
    ajb += t.rj * rab;
    // ms = mi mj / (mi + mj), m = density 8 r^3
    const double sm = t.mi + t.mj;
    const double mib = msb * t.mj * t.mj / (sm * sm), mjb = msb * t.mi * t.mi / (sm * sm);
    rib += mib * density * 24.0 * t.ri * t.ri;
    rjb += mjb * density * 24.0 * t.rj * t.rj;
    // rs = ri rj / (ri + rj)
    rib += rsb * t.rj * t.rj / (t.sr * t.sr);
    rjb += rsb * t.ri * t.ri / (t.sr * t.sr);
    // delta = ri + rj - dist
    rib += deltab;
    rjb += deltab;
    double distb = -deltab;
    // n = D / dist
    const double nn = dot(t.n, nb);
    V3d Db = (1.0 / t.dist) * (nb - nn * t.n);
    Db += distb * t.n;
    xjb += Db;
    xib -= Db;
}

// Walls (same order and primary-wall rule as wall_contacts): the forward
// (wall_fwd, totals only) and the reverse (wall_vjp: each touching wall's law
// is re-evaluated with its own tape and reversed at once -- the walls are
// independent given the output adjoints, so no tape array is needed).
DEM_HD V3d wall_normal(int w) {
    V3d n;
    n.x = (w == 1) ? -1.0 : ((w == 2) ? 1.0 : 0.0);
    n.y = (w == 3) ? -1.0 : ((w == 4) ? 1.0 : 0.0);
    n.z = (w == 0) ? -1.0 : 0.0;
    return n;
}

DEM_HD int wall_prim(double hx, double hy, V3d x, double r, double dl[5]) {
    dl[0] = r - x.z;
    dl[1] = r - (x.x + hx);
    dl[2] = r - (hx - x.x);
    dl[3] = r - (x.y + hy);
    dl[4] = r - (hy - x.y);
    int prim = -1;
    for (int w = 0; w < 5; w++)
        if (dl[w] > 0.0 && (prim < 0 || dl[w] > dl[prim])) prim = w;
    return prim;
}

DEM_HD int wall_fwd(double hx, double hy, V3d x, V3d d, V3d a, double r, double density, V3d h_in,
                    const LawParams<double>& p, double inv_dt, V3d& F, V3d& T, V3d& h_out) {
    double dl[5];
    const int prim = wall_prim(hx, hy, x, r, dl);
    F = T = h_out = zero3<double>();
    if (prim < 0) return 0;
    const double m = density * 8.0 * r * r * r;
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        if (!(dl[w] > 0.0)) continue;
        const V3d n = wall_normal(w);
        const V3d U = (-d) - r * cross(a, n);
        const V3d h = (w == prim) ? h_in : zero3<double>();
        LawTape t;
        V3d Fi, Ft, Mr, ho;
        law_fwd(dl[w], n, r, m, U, a, h, inv_dt, p, t, Fi, Ft, Mr, ho);
        F += Fi;
        T += r * cross(n, Ft) + Mr;
        if (w == prim) h_out = ho;
    }
    return 1;
}

// Adds the input adjoints of the wall contacts of one particle given the
// adjoints of its wall force/torque (Fb, Tb) and of its output history (hb).
// Returns 1 if a wall was touched.
DEM_HD int wall_vjp(double hx, double hy, V3d x, V3d d, V3d a, double r, double density, V3d h_in,
                    const LawParams<double>& p, double inv_dt, V3d Fb, V3d Tb, V3d hb, V3d& xb, V3d& db, V3d& ab,
                    double& rb, V3d& hinb, LawBar& pb) {
    double dl[5];
    const int prim = wall_prim(hx, hy, x, r, dl);
    if (prim < 0) return 0;
    const double m = density * 8.0 * r * r * r;
    // one copy of the law's forward and reverse for all five walls (touching
    // a wall is the rare path; unrolled, the copies would crowd out the
    // registers of the rest of the reverse step)
#pragma unroll 1
    for (int w = 0; w < 5; w++) {
        if (!(dl[w] > 0.0)) continue;
        const V3d n = wall_normal(w);
        const V3d axn = cross(a, n);
        const V3d U = (-d) - r * axn;
        const V3d h = (w == prim) ? h_in : zero3<double>();
        LawTape t;
        V3d Fi, Ft, Mr, ho;
        law_fwd(dl[w], n, r, m, U, a, h, inv_dt, p, t, Fi, Ft, Mr, ho);
        // T += r (n x Ft) + Mr
        const V3d nxf = cross(n, Ft);
        rb += dot(nxf, Tb);
        const V3d nxfb = r * Tb;
        V3d Ftb = cross(nxfb, n);
        double deltab = 0.0, rsb = 0.0, msb = 0.0;
        V3d nb = zero3<double>(), Ub = zero3<double>(), Wrb = zero3<double>(), hib = zero3<double>();
        law_rev(t, p, inv_dt, Fb, Ftb, Tb, (w == prim) ? hb : zero3<double>(), deltab, nb, rsb, msb, Ub, Wrb, hib,
                pb);
        if (w == prim) hinb += hib;
        ab += Wrb;                                  // Wr = a
        db -= Ub;                                   // U = -d - r (a x n)
        ab += cross(n, (-r) * Ub);
        rb += -dot(axn, Ub);
        rb += rsb + msb * density * 24.0 * r * r;   // R* = r, m* = density 8 r^3
        rb += deltab;                               // delta = r + x.n - c
        xb += deltab * n;
    }
    return 1;
}

}  // namespace dem
