"""TEST INFRASTRUCTURE ONLY: ctypes binding of liboracle.so, the FP64
C++/OpenMP restatement of the reference's DEM step (oracle/dem_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (libdem_b200.so and its binding) never does.
"""
import ctypes
import pathlib
import subprocess

import numpy as np

ORACLE_DIR = pathlib.Path(__file__).resolve().parent
LIB = ORACLE_DIR / "liboracle.so"
_L = None

_d = ctypes.c_double
_u = ctypes.c_uint
_ll = ctypes.c_longlong
_vp = ctypes.c_void_p
_i = ctypes.c_int


def build():
    subprocess.run(["make", "-C", str(ORACLE_DIR), "liboracle.so"], check=True, capture_output=True)


def lib():
    global _L
    if _L is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        sigs = {
            "orc_num_threads": (_i, []),
            "orc_set_threads": (None, [_i]),
            "ref_length": (_d, [_vp]),
            "ref_vprojec": (None, [_vp, _vp, _vp, _u]),
            "ref_vscale": (None, [_vp, _d, _d]),
            "orc_pair_force": (_i, [_vp] * 6 + [_d] * 4 + [_vp, _d, _vp, _vp, _vp, _vp]),
            "orc_wall_force": (_i, [_vp, _vp, _vp, _vp, _d, _d, _vp, _d, _vp, _vp, _vp]),
            "ref_set_material": (None, [_vp, _vp]),
            "ref_set_cutoff": (None, [_d, _d]),
            "ref_calcHash": (None, [_vp, _vp, _vp, _vp, _vp, _i]),
            "ref_radix_sort": (None, [_vp, _u, _u]),
            "ref_findCellStart": (None, [_vp, _vp, _i, _u]),
            "ref_neighborarray": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp]),
            "ref_prefixsum": (_u, [_u, _vp, _vp, _vp]),
            "ref_pairlist": (None, [_vp] * 8 + [_i, _i, _u] + [_vp] * 5),
            "ref_calculateforcepair": (None, [_vp] * 12 + [_d] + [_vp] * 4 + [_u]),
            "ref_sumallforcei": (None, [_i, _i] + [_vp] * 10),
            "ref_calculateforceiw": (None, [_vp] * 6 + [_d, _u, _i] + [_vp] * 4),
            "ref_updateposition": (_u, [_vp, _i] + [_vp] * 8 + [_d, _vp]),
            "ref_outputporositycn": (_u, [_u, _vp]),
            "orc_grid_size": (_i, [_vp, _d, _vp]),
            "orc_hash": (None, [_ll, _vp, _vp, _d, _i, _vp]),
            "orc_sort_cells": (None, [_ll, _vp, _u, _vp, _vp, _vp, _vp]),
            "orc_build_list": (_ll, [_ll, _vp, _vp, _vp, _d, _d, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _vp]),
            "orc_run": (_i, [_ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _ll, _i, _ll, _vp, _vp, _vp, _vp]),
            "orc_run_list": (_i, [_ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _ll, _i, _ll, _vp, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp]),
            "orc_run_pour": (_i, [_ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _ll, _i, _ll, _ll, _d, _ll, _vp,
                                  _vp, _vp, _vp, _vp, _vp]),
            "orc_forces_once": (_i, [_ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _ll, _vp, _vp, _vp, _vp]),
            "orc_engine_new": (_vp, [_ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _ll]),
            "orc_engine_step": (_i, [_vp, _ll, _vp]),
            "orc_engine_free": (None, [_vp]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def P(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "need a C-contiguous numpy array"
    # data_as keeps a reference to the array, so temporaries stay alive for the call
    return a.ctypes.data_as(ctypes.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_threads(n):
    lib().orc_set_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


# ----------------------------------------------------------- engine oracle
def grid(world, cell):
    g = np.zeros(3, dtype=np.uint32)
    lib().orc_grid_size(P(f64(world)), float(cell), P(g))
    return g


def hash_keys(pos, world, cell, fp32):
    pos = f64(pos)
    n = pos.size // 3
    keys = np.empty(n, dtype=np.uint32)
    lib().orc_hash(n, P(pos), P(f64(world)), float(cell), int(fp32), P(keys))
    return keys


def sort_cells(keys, ncells):
    keys = u32(keys)
    n = keys.size
    sk = np.empty(n, dtype=np.uint32)
    si = np.empty(n, dtype=np.uint32)
    cs = np.empty(ncells, dtype=np.uint32)
    ce = np.empty(ncells, dtype=np.uint32)
    lib().orc_sort_cells(n, P(keys), int(ncells), P(sk), P(si), P(cs), P(ce))
    return sk, si, cs, ce


def build_list(pos, rad, world, cell, skin, fp32, cap=None, old=None):
    """Returns (off[n+1], ln[P], hist[3P], max_row).  old = (off, ln, hist)."""
    pos, rad = f64(pos), f64(rad)
    n = rad.size
    cap = cap or 16 * n + 16
    off = np.zeros(n + 1, dtype=np.uint32)
    ln = np.zeros(cap, dtype=np.uint32)
    hist = np.zeros(3 * cap)
    mr = ctypes.c_int(0)
    oo = ol = oh = None
    if old is not None:
        oo, ol, oh = u32(old[0]), u32(old[1]), f64(old[2])
    got = lib().orc_build_list(n, P(pos), P(rad), P(f64(world)), float(cell), float(skin), int(fp32), P(oo), P(ol),
                               P(oh), P(off), P(ln), P(hist), cap, ctypes.byref(mr))
    if got < 0:
        raise RuntimeError(f"oracle list capacity {cap} < {-got}")
    return off, ln[:got].copy(), hist[:3 * got].copy(), mr.value


def run(pos, rad, world, dt, skin, cell, density, mat14, fp32_list, nsteps, interval, pdis=None, angv=None,
        cap=None, scalars=True):
    """Engine loop restated.  Returns dict with final pos/pdis/angv, wall
    history, per-step scalars (maxhz, contacts, pairs), last forces."""
    pos = f64(pos).copy()
    rad = f64(rad)
    n = rad.size
    pdis = np.zeros(3 * n) if pdis is None else f64(pdis).copy()
    angv = np.zeros(3 * n) if angv is None else f64(angv).copy()
    wh = np.zeros(3 * n)
    cap = cap or 16 * n + 16
    params = np.array([dt, skin, cell, density], dtype=np.float64)
    sc = np.zeros(3 * nsteps) if scalars else None
    F = np.zeros(3 * n)
    T = np.zeros(3 * n)
    C = np.zeros(n, dtype=np.uint32)
    off = np.zeros(n + 1, dtype=np.uint32)
    ln = np.zeros(cap, dtype=np.uint32)
    hist = np.zeros(3 * cap)
    npairs = ctypes.c_longlong(0)
    st = lib().orc_run_list(n, P(pos), P(pdis), P(angv), P(rad), P(wh), P(f64(world)), P(params), P(f64(mat14)),
                            int(fp32_list), int(nsteps), int(interval), int(cap), P(sc), P(F), P(T), P(C), P(off),
                            P(ln), P(hist), ctypes.byref(npairs))
    Pn = npairs.value
    out = dict(status=st, pos=pos, pdis=pdis, angv=angv, whist=wh, force=F, torque=T, contacts=C,
               list_off=off, list_ln=ln[:Pn].copy(), list_hist=hist[:3 * Pn].copy())
    if scalars:
        s = sc.reshape(-1, 3)
        out.update(maxhz=s[:, 0].copy(), ncontacts=s[:, 1].copy(), npairs=s[:, 2].copy())
    return out


def run_pour(pos, rad, world, dt, skin, cell, density, mat14, fp32_list, nsteps, interval, nplayer, tnewpar,
             n_active=0, pdis=None, angv=None, cap=None):
    """Poured packing (orc_run_pour): pos/pdis/angv/rad hold all ntot
    particles, entries from the active count on being injection states.
    Returns the final state, the active count and scalars of every step, and
    the final list."""
    pos = f64(pos).copy()
    rad = f64(rad)
    n = rad.size
    pdis = np.zeros(3 * n) if pdis is None else f64(pdis).copy()
    angv = np.zeros(3 * n) if angv is None else f64(angv).copy()
    wh = np.zeros(3 * n)
    cap = cap or 16 * n + 16
    params = np.array([dt, skin, cell, density], dtype=np.float64)
    sc = np.zeros(3 * nsteps)
    nact = np.zeros(nsteps, dtype=np.int64)
    off = np.zeros(n + 1, dtype=np.uint32)
    ln = np.zeros(cap, dtype=np.uint32)
    hist = np.zeros(3 * cap)
    npairs = ctypes.c_longlong(0)
    st = lib().orc_run_pour(n, P(pos), P(pdis), P(angv), P(rad), P(wh), P(f64(world)), P(params), P(f64(mat14)),
                            int(fp32_list), int(nsteps), int(interval), int(cap), int(nplayer), float(tnewpar),
                            int(n_active), P(nact), P(sc), P(off), P(ln), P(hist), ctypes.byref(npairs))
    Pn = npairs.value
    s = sc.reshape(-1, 3)
    na = int(nact[-1]) if nsteps else int(n_active)
    return dict(status=st, pos=pos, pdis=pdis, angv=angv, whist=wh, nact=nact, maxhz=s[:, 0].copy(),
                ncontacts=s[:, 1].copy(), npairs=s[:, 2].copy(), list_off=off[:na + 1].copy(),
                list_ln=ln[:Pn].copy(), list_hist=hist[:3 * Pn].copy())


def forces_once(pos, rad, world, dt, skin, cell, density, mat14, fp32_list, pdis=None, angv=None, cap=None):
    pos, rad = f64(pos), f64(rad)
    n = rad.size
    pdis = np.zeros(3 * n) if pdis is None else f64(pdis)
    angv = np.zeros(3 * n) if angv is None else f64(angv)
    cap = cap or 16 * n + 16
    params = np.array([dt, skin, cell, density], dtype=np.float64)
    F = np.zeros(3 * n)
    T = np.zeros(3 * n)
    C = np.zeros(n, dtype=np.uint32)
    npairs = ctypes.c_longlong(0)
    st = lib().orc_forces_once(n, P(pos), P(pdis), P(angv), P(rad), P(f64(world)), P(params), P(f64(mat14)),
                               int(fp32_list), cap, P(F), P(T), P(C), ctypes.byref(npairs))
    if st:
        raise RuntimeError(f"oracle forces_once status {st}")
    return F, T, C, npairs.value


def pair_force(xi, xj, di, dj, ai, aj, ri, rj, mi, mj, hist, dt, par7):
    Fi = np.zeros(3)
    Ti = np.zeros(3)
    Tj = np.zeros(3)
    h = f64(hist).copy()
    c = lib().orc_pair_force(P(f64(xi)), P(f64(xj)), P(f64(di)), P(f64(dj)), P(f64(ai)), P(f64(aj)), float(ri),
                             float(rj), float(mi), float(mj), P(h), float(dt), P(f64(par7)), P(Fi), P(Ti), P(Tj))
    return c, Fi, Ti, Tj, h


def wall_force(world, x, d, a, r, m, hist, dt, par7):
    F = np.zeros(3)
    T = np.zeros(3)
    h = f64(hist).copy()
    c = lib().orc_wall_force(P(f64(world)), P(f64(x)), P(f64(d)), P(f64(a)), float(r), float(m), P(h), float(dt),
                             P(f64(par7)), P(F), P(T))
    return c, F, T, h


def par7(c: dict):
    return np.array([c["estar"], c["mu"], c["nu"], c["damp_n"], c["damp_t"], c["roll"], c["roll_rel"]])


class Stepper:
    """Stateful oracle engine (one call advances nsteps, re-list cadence kept)."""

    def __init__(self, pos, rad, world, dt, skin, cell, density, mat14, fp32_list, interval, cap=None):
        pos, rad = f64(pos), f64(rad)
        self.n = rad.size
        cap = cap or 16 * self.n + 16
        params = np.array([dt, skin, cell, density], dtype=np.float64)
        self._h = lib().orc_engine_new(self.n, P(pos), None, None, P(rad), P(f64(world)), P(params), P(f64(mat14)),
                                       int(fp32_list), int(interval), int(cap))

    def step(self, nsteps=1):
        mz = ctypes.c_double(0.0)
        st = lib().orc_engine_step(self._h, int(nsteps), ctypes.byref(mz))
        if st == 3:
            raise RuntimeError("oracle pair capacity exceeded")
        return mz.value

    def close(self):
        if self._h:
            lib().orc_engine_free(self._h)
            self._h = None

    def __del__(self):
        self.close()
