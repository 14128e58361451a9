"""CPU check of the hand-written reverse mode of the contact law (the code the
adjoint kernels run, dem_law_adj.cuh) against central finite differences of
its own primal: every input adjoint (positions, per-step displacements and
rotations, radii, tangential history) and every parameter adjoint (estar,
mu, damping, rolling) of a pair contact and of wall contacts, in stick, slip
and Coulomb-capped states.  The headers are compiled for the host with g++."""
import ctypes
import pathlib
import subprocess

import numpy as np
import pytest

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE.parent / "discrete-element-method-for-packing-cuda-c-code_b200" / "csrc"

ESTAR = 566830.28
NU = 0.29


@pytest.fixture(scope="module")
def lc():
    out = HERE / "lawcheck" / "_build" / "liblawcheck.so"
    out.parent.mkdir(exist_ok=True)
    src = HERE / "lawcheck" / "lawcheck.cpp"
    deps = [src, CSRC / "dem_law.cuh", CSRC / "dem_law_adj.cuh", CSRC / "dem_common.cuh"]
    if not out.exists() or any(d.stat().st_mtime > out.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", f"-I{CSRC}",
                        f"-I{HERE.parent / 'include'}", "-I/usr/local/cuda/include", "-o", str(out), str(src)],
                       check=True)
    L = ctypes.CDLL(str(out))
    vp, d = ctypes.c_void_p, ctypes.c_double
    L.lc_pair_fwd.argtypes = [vp, vp, d, d, vp]
    L.lc_pair_fwd.restype = ctypes.c_int
    L.lc_pair_vjp.argtypes = [vp, vp, d, d, vp, vp, vp]
    L.lc_wall_fwd.argtypes = [vp, d, d, vp, d, d, vp]
    L.lc_wall_fwd.restype = ctypes.c_int
    L.lc_wall_vjp.argtypes = [vp, d, d, vp, d, d, vp, vp, vp]
    return L


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def pair_case(rng, hist_scale, vt_scale):
    ri, rj = rng.uniform(0.3, 0.8, 2)
    n = rng.normal(size=3)
    n /= np.linalg.norm(n)
    xi = rng.normal(size=3)
    delta = rng.uniform(2e-5, 5e-4)
    xj = xi + n * (ri + rj - delta)
    di = rng.normal(0, 1e-5, 3)
    dj = di + rng.normal(0, vt_scale, 3)
    ai, aj = rng.normal(0, 2e-5, 3), rng.normal(0, 2e-5, 3)
    h = rng.normal(0, hist_scale, 3)
    return np.concatenate([xi, xj, di, dj, ai, aj, [ri, rj], h])


def fd_check(fwd, vjp, x0, par, nout, rng, rel=2e-5, geometric=()):
    """geometric: indices of positions/radii, which move the overlap (1e-5 to
    1e-3 here) directly: they get an absolute step well below it."""
    ob = rng.normal(size=nout)
    ib, pb = vjp(x0, par, ob)
    big = np.abs(ib).max()
    # inputs: three step sizes (truncation vs rounding), the best must agree
    for k in range(x0.size):
        errs = []
        for f in (10.0, 1.0, 0.1):
            h = 2e-9 * f if k in geometric else 1e-5 * f * max(abs(x0[k]), 1e-7)
            xp, xm = x0.copy(), x0.copy()
            xp[k] += h
            xm[k] -= h
            fd = (ob @ (fwd(xp, par) - fwd(xm, par))) / (2 * h)
            errs.append(abs(fd - ib[k]) - rel * max(abs(fd), abs(ib[k])) - 1e-7 * big)
        assert min(errs) <= 0.0, (k, ib[k], errs)
    # parameters: estar, mu, cn, ct, roll, roll_rel  (par indices 0,1,3,4,5,6)
    for pk, pi in enumerate((0, 1, 3, 4, 5, 6)):
        if par[pi] == 0.0 and pi in (5,):
            continue
        # parameters enter smoothly (damping and rolling linearly): a larger
        # step keeps the difference above the FP64 noise of O(1) outputs
        h = 1e-4 * max(abs(par[pi]), 1e-4)
        pp, pm = par.copy(), par.copy()
        pp[pi] += h
        pm[pi] -= h
        fd = (ob @ (fwd(x0, pp) - fwd(x0, pm))) / (2 * h)
        scale = max(abs(fd), abs(pb[pk]), 1e-300)
        assert abs(fd - pb[pk]) <= 1e-4 * scale + 1e-10 * max(abs(pb).max(), 1.0), (pk, fd, pb[pk])


@pytest.mark.parametrize("state", ["stick", "slip", "capped", "fresh"])
def test_pair_vjp_matches_finite_differences(lc, state):
    rng = np.random.default_rng({"stick": 1, "slip": 2, "capped": 3, "fresh": 4}[state])
    dt = 5e-5
    inv_dt = 1.0 / dt
    par = np.array([ESTAR, 0.3, NU, 0.23, 0.23, 0.001, 0.002])
    hs, vs = {"stick": (1e-6, 1e-8), "slip": (3e-4, 1e-6), "capped": (1e-6, 3e-5), "fresh": (0.0, 1e-7)}[state]

    def fwd(x, p):
        out = np.zeros(12)
        lc.lc_pair_fwd(P(x), P(p), inv_dt, 1.0, P(out))
        return out

    def vjp(x, p, ob):
        ib = np.zeros(23)
        pb = np.zeros(6)
        lc.lc_pair_vjp(P(x), P(p), inv_dt, 1.0, P(ob), P(ib), P(pb))
        return ib, pb

    checked = 0
    for _ in range(40):
        x0 = pair_case(rng, hs, vs)
        if state == "fresh":
            x0[20:23] = 0.0
        out = fwd(x0, par)
        assert np.all(np.isfinite(out))
        # stay away from the non-smooth switches of the law for the FD check
        h1 = out[9:12]
        if state in ("stick", "fresh") and np.linalg.norm(h1) == 0.0 and state != "fresh":
            continue
        fd_check(fwd, vjp, x0, par, 12, rng, geometric=tuple(range(6)) + (18, 19))
        checked += 1
    assert checked >= 20


@pytest.mark.parametrize("where", ["floor", "corner"])
def test_wall_vjp_matches_finite_differences(lc, where):
    rng = np.random.default_rng(7 if where == "floor" else 8)
    dt = 5e-5
    inv_dt = 1.0 / dt
    par = np.array([ESTAR, 0.3, NU, 0.23, 0.23, 0.0, 0.002])
    hx = hy = 5.0

    def fwd(x, p):
        out = np.zeros(9)
        lc.lc_wall_fwd(P(x), hx, hy, P(p), inv_dt, 1.0, P(out))
        return out

    def vjp(x, p, ob):
        ib = np.zeros(13)
        pb = np.zeros(6)
        lc.lc_wall_vjp(P(x), hx, hy, P(p), inv_dt, 1.0, P(ob), P(ib), P(pb))
        return ib, pb

    for _ in range(30):
        r = rng.uniform(0.3, 0.8)
        x = np.array([rng.uniform(-2, 2), rng.uniform(-2, 2), r - rng.uniform(2e-5, 4e-4)])
        if where == "corner":
            x[0] = hx - r + rng.uniform(2e-5, 3e-4)
            x[1] = -hy + r - rng.uniform(2e-5, 3e-4)
        d = rng.normal(0, 1e-6, 3)
        a = rng.normal(0, 2e-5, 3)
        h = rng.normal(0, 2e-6, 3)
        x0 = np.concatenate([x, d, a, [r], h])
        fd_check(fwd, vjp, x0, par, 9, rng, geometric=(0, 1, 2, 9))
