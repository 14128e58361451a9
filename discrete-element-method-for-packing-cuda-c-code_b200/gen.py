"""Initial states and material helpers from libdem_gen.so: the same C++
source (csrc/dem_gen.cpp) as the generators of libdem_b200.so, built host
only.  The workloads use it, so that CPU-only runs (the oracle's runs in the
tests, the CPU timing of the reference step) generate their inputs without
loading the GPU library, bit for bit as the GPU runs do.
"""
import ctypes
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libdem_gen.so"
_L = None
_vp = ctypes.c_void_p
_d = ctypes.c_double


def lib():
    global _L
    if _L is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               f"(make -C {LIB_PATH.parent / 'csrc'})")
        L = ctypes.CDLL(str(LIB_PATH))
        sigs = {
            "dem_gen_last_error": (ctypes.c_char_p, []),
            "dem_reduced_modulus": (_d, [_d, _d, _d]),
            "dem_estar": (_d, [_d, _d, _d, _d]),
            "dem_damp_from_restitution": (_d, [_d]),
            "dem_gen_lattice": (ctypes.c_int, [ctypes.c_longlong, _d, ctypes.c_int, ctypes.c_int, _d, _d, _d,
                                               ctypes.c_ulonglong, _vp, _vp]),
            "dem_gen_radii": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, _d, _d, _d, _d, ctypes.c_ulonglong,
                                             _vp]),
            "dem_gen_rsa": (ctypes.c_int, [ctypes.c_longlong, ctypes.POINTER(_d), _vp, ctypes.c_ulonglong, _vp]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().dem_gen_last_error().decode(errors='replace')}")


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def gen_lattice(n, spacing, nx, ny, z0, jitter, radius, seed):
    pos = np.empty(3 * n)
    rad = np.empty(n)
    _check(lib().dem_gen_lattice(int(n), float(spacing), int(nx), int(ny), float(z0), float(jitter), float(radius),
                                 int(seed), _p(pos), _p(rad)), "dem_gen_lattice")
    return pos, rad


def gen_radii(n, kind, a, b=0.0, c=0.0, d=0.0, seed=0):
    rad = np.empty(n)
    _check(lib().dem_gen_radii(int(n), int(kind), float(a), float(b), float(c), float(d), int(seed), _p(rad)),
           "dem_gen_radii")
    return rad


def gen_rsa(world, rad, seed):
    rad = np.ascontiguousarray(rad, dtype=np.float64)
    pos = np.empty(3 * rad.size)
    w = (ctypes.c_double * 3)(*[float(x) for x in world])
    _check(lib().dem_gen_rsa(int(rad.size), w, _p(rad), int(seed), _p(pos)), "dem_gen_rsa")
    return pos


def estar(E, nu, rho, dref):
    return lib().dem_estar(float(E), float(nu), float(rho), float(dref))


def damp_from_restitution(e):
    return lib().dem_damp_from_restitution(float(e))


def reduced_modulus(E, rho, dref):
    return lib().dem_reduced_modulus(float(E), float(rho), float(dref))
