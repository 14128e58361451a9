"""dem_b200 -- Python binding of libdem_b200.so (the sm_100a DEM packing step).

The library's C ABI is declared in include/dem_b200.h.  This module binds it
with ctypes; there is no Python or CPU implementation of any kernel here, and
every entry point fails loudly when the shared library is missing.

Two layers, as in the C ABI:

* ``compat``: the reference-compatible entry points (calcHash, RadixSort,
  findCellStart, neighborarray, prefixsum, pairlist, calculateforcepair,
  sumallforcei, calculateforceiw, updateposition, outputporositycn --
  particleSystem.cu:13-424 and dempacking.cu:553) taking device pointers.
  Helpers accept torch CUDA tensors and pass their data pointers.
* ``Engine``: the context API (structure-of-arrays state, CSR pair list,
  CUDA-graph windows) with FP64 or mixed precision.
"""
import ctypes
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libdem_b200.so"

DEM_OK, DEM_ERR_ARG, DEM_ERR_CUDA, DEM_ERR_CAPACITY = 0, 1, 2, 3
DEM_ERR_NONFINITE, DEM_ERR_SKIN, DEM_ERR_IO, DEM_ERR_STATE, DEM_ERR_TIMEOUT = 4, 5, 6, 7, 8
PREC_FP64, PREC_MIXED = 0, 1
OBJ_PACKING, OBJ_POTENTIAL = 0, 1
FORCE_PCCP, FORCE_PP = 0, 1
RADII_MONO, RADII_LOGNORMAL, RADII_BIDISPERSE = 0, 1, 2

_c_uint_p = ctypes.POINTER(ctypes.c_uint)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class DemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dem_b200 error {code}: {msg}")
        self.code = code


class KeyValuePair(ctypes.Structure):
    _fields_ = [("key", ctypes.c_uint), ("value", ctypes.c_uint)]


class Matproperties(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("estarp", "ufricp", "vpois", "dampnp", "damptp", "upp")]


class Wallproperties(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("estarw", "ufricw", "vpoisw", "dampnw", "damptw", "upw")]


class Contact(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("estar", "mu", "nu", "damp_n", "damp_t", "roll", "roll_rel")]


class Material(ctypes.Structure):
    _fields_ = [("pp", Contact), ("pw", Contact)]


class Config(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_longlong),
        ("precision", ctypes.c_int),
        ("relist_interval", ctypes.c_int),
        ("world", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("skin", ctypes.c_double),
        ("cell", ctypes.c_double),
        ("density", ctypes.c_double),
        ("pair_capacity", ctypes.c_longlong),
        ("force_mode", ctypes.c_int),
    ]


class Scalars(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_longlong),
        ("pairs", ctypes.c_longlong),
        ("contacts", ctypes.c_longlong),
        ("maxhz", ctypes.c_double),
        ("packing_fraction", ctypes.c_double),
        ("mean_cn", ctypes.c_double),
        ("relists", ctypes.c_longlong),
        ("status", ctypes.c_int),
        ("max_row", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AdjointResult(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("d_pp", Contact), ("d_pw", Contact), ("forward_ms", ctypes.c_double),
                ("adjoint_ms", ctypes.c_double)]


class Deck(ctypes.Structure):
    _fields_ = [
        ("iforcemode", ctypes.c_int), ("ntot", ctypes.c_int),
        ("emod", ctypes.c_double), ("vpois", ctypes.c_double), ("denp", ctypes.c_double), ("diam", ctypes.c_double),
        ("dt", ctypes.c_double), ("tstop", ctypes.c_uint),
        ("dmt1", ctypes.c_double), ("dmt2", ctypes.c_double), ("thick", ctypes.c_double),
        ("zht1", ctypes.c_double), ("zht2", ctypes.c_double),
        ("vel0", ctypes.c_double), ("nrings", ctypes.c_int),
        ("ufricp", ctypes.c_double), ("ufricw", ctypes.c_double),
        ("dampnp", ctypes.c_double), ("damptp", ctypes.c_double), ("dampnw", ctypes.c_double),
        ("damptw", ctypes.c_double), ("cdamp", ctypes.c_double),
        ("stiffness", ctypes.c_double), ("dampcoeffn", ctypes.c_double), ("dampcoefft", ctypes.c_double),
        ("upp", ctypes.c_double), ("upw", ctypes.c_double),
        ("emod_red", ctypes.c_double), ("estarp", ctypes.c_double), ("estarw", ctypes.c_double),
        ("world", ctypes.c_double * 3),
        ("upp_red", ctypes.c_double), ("upw_red", ctypes.c_double),
    ]


# --------------------------------------------------------------------- loader
_LIB = None

# (name, restype, argtypes)
_SIGS = [
    ("dem_last_error_string", ctypes.c_char_p, []),
    ("dem_version", ctypes.c_char_p, []),
    ("setMaterialProperties", ctypes.c_int, [ctypes.POINTER(Matproperties), ctypes.POINTER(Wallproperties)]),
    ("setListCutoff", ctypes.c_int, [ctypes.c_double, ctypes.c_double]),
    ("dem_compat_set_stream", ctypes.c_int, [_vp]),
    ("RadixSort", ctypes.c_int, [_vp, _vp, ctypes.c_uint, ctypes.c_uint]),
    ("RadixSortNoAlloc", ctypes.c_int, [_vp, _vp, ctypes.c_uint, ctypes.c_uint]),
    ("calcHash", ctypes.c_int, [_vp, _vp, _c_uint_p, _c_double_p, _c_double_p, ctypes.c_int]),
    ("findCellStart", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint]),
    ("neighborarray", ctypes.c_int, [_vp, _vp, _vp, _c_uint_p, _c_double_p, _c_double_p, ctypes.c_int, ctypes.c_int,
                                     _vp, _vp, _vp]),
    ("prefixsum", ctypes.c_int, [ctypes.c_uint, _vp, _vp, _vp, _c_uint_p]),
    ("pairlist", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                _vp, _vp, _vp, _vp, _vp]),
    ("calculateforcepair", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double,
                                          _vp, _vp, _vp, _vp, ctypes.c_uint]),
    ("sumallforcei", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("calculateforceiw", ctypes.c_int, [_c_double_p, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_uint,
                                        ctypes.c_int, _vp, _vp, _vp, _vp]),
    ("updateposition", ctypes.c_int, [_c_double_p, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                      ctypes.c_double, ctypes.c_double, _c_uint_p, _c_double_p]),
    ("outputporositycn", ctypes.c_int, [ctypes.c_uint, _vp, ctypes.c_double, _c_double_p, _c_uint_p]),
    ("dem_create", ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(_vp)]),
    ("dem_destroy", ctypes.c_int, [_vp]),
    ("dem_set_stream", ctypes.c_int, [_vp, _vp]),
    ("dem_set_material", ctypes.c_int, [_vp, ctypes.POINTER(Material)]),
    ("dem_upload_state", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("dem_upload_state_device", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("dem_download_state", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("dem_download_state_device", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("dem_step_n", ctypes.c_int, [_vp, ctypes.c_longlong]),
    ("dem_get_scalars", ctypes.c_int, [_vp, ctypes.POINTER(Scalars)]),
    ("dem_scalars_raw_bytes", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    ("dem_scalars_enqueue", ctypes.c_int, [_vp, _vp]),
    ("dem_scalars_from_raw", ctypes.c_int, [_vp, _vp, ctypes.POINTER(Scalars)]),
    ("dem_synchronize", ctypes.c_int, [_vp]),
    ("dem_record_forces", ctypes.c_int, [_vp, ctypes.c_int]),
    ("dem_download_forces", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("dem_download_pairs", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    ("dem_download_cells", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_longlong]),
    ("dem_grid_info", ctypes.c_int, [_vp, _c_uint_p, _c_double_p, ctypes.POINTER(ctypes.c_longlong)]),
    ("dem_set_profiling", ctypes.c_int, [_vp, ctypes.c_int]),
    ("dem_kernel_times", ctypes.c_int, [_vp, _c_double_p]),
    ("dem_set_window_timing", ctypes.c_int, [_vp, ctypes.c_int]),
    ("dem_window_kernel_times", ctypes.c_int, [_vp, _c_double_p]),
    ("dem_window_work", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]),
    ("dem_adjoint_window", ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(AdjointResult), _vp]),
    ("dem_adjoint_release", ctypes.c_int, [_vp]),
    ("dem_read_deck", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Deck)]),
    ("dem_deck_material", ctypes.c_int, [ctypes.POINTER(Deck), ctypes.POINTER(Material)]),
    ("dem_reduced_modulus", ctypes.c_double, [ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ("dem_estar", ctypes.c_double, [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ("dem_damp_from_restitution", ctypes.c_double, [ctypes.c_double]),
    ("dem_gen_lattice", ctypes.c_int, [ctypes.c_longlong, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong,
                                       _vp, _vp]),
    ("dem_gen_radii", ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, _vp]),
    ("dem_gen_rsa", ctypes.c_int, [ctypes.c_longlong, _c_double_p, _vp, ctypes.c_ulonglong, _vp]),
    ("dem_write_view", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Deck)]),
    ("dem_write_ppor", ctypes.c_int, [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ("dem_write_particles", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_longlong, _vp, _vp,
                                           ctypes.c_double]),
    ("dem_write_preflow", ctypes.c_int, [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                                         _vp, _vp, _vp]),
    ("dem_write_timesteps", ctypes.c_int, [ctypes.c_char_p, ctypes.c_double, ctypes.c_longlong]),
    ("dem_read_preflow", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), _vp, _vp,
                                        _vp, ctypes.c_longlong]),
    ("dem_save_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("dem_load_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("dem_set_pour", ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_double, ctypes.c_longlong]),
    ("dem_check_barrier_timeout", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
    ("dem_active_count", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    ("dem_write_finish", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p]),
]


def lib():
    """The loaded libdem_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               f"(make -C {PKG_DIR / 'csrc'})")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def symbols():
    return [s[0] for s in _SIGS]


def check(rc, what=""):
    if rc != DEM_OK:
        msg = lib().dem_last_error_string().decode(errors="replace")
        raise DemError(rc, f"{what}: {msg}" if what else msg)
    return rc


def _ptr(a):
    """Data pointer of a torch tensor or numpy array (None -> NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data_as(ctypes.c_void_p)   # keeps the array alive during the call
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    raise TypeError(f"cannot take a pointer of {type(a)}")


def _u3(v):
    return (ctypes.c_uint * 3)(*[int(x) for x in v])


def _d3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


# ------------------------------------------------------- compat entry points
class compat:
    """Reference-compatible entry points.  Arguments are device buffers (torch
    CUDA tensors or raw device pointers as int), in the reference layout."""

    @staticmethod
    def set_material(par: dict, parw: dict):
        m = Matproperties(**par)
        w = Wallproperties(**parw)
        check(lib().setMaterialProperties(ctypes.byref(m), ctypes.byref(w)), "setMaterialProperties")

    @staticmethod
    def set_cutoff(cua, cub):
        check(lib().setListCutoff(float(cua), float(cub)), "setListCutoff")

    @staticmethod
    def set_stream(stream_handle):
        check(lib().dem_compat_set_stream(ctypes.c_void_p(stream_handle)), "dem_compat_set_stream")

    @staticmethod
    def RadixSort(d0, d1, n, bits=32):
        return check(lib().RadixSort(_ptr(d0), _ptr(d1), int(n), int(bits)), "RadixSort")

    @staticmethod
    def RadixSortNoAlloc(d0, d1, n, bits=32):
        return check(lib().RadixSortNoAlloc(_ptr(d0), _ptr(d1), int(n), int(bits)), "RadixSortNoAlloc")

    @staticmethod
    def calcHash(pos, phash, grid, cell, origin, n):
        return check(lib().calcHash(_ptr(pos), _ptr(phash), _u3(grid), _d3(cell), _d3(origin), int(n)), "calcHash")

    @staticmethod
    def findCellStart(phash, cstart, n, ncells):
        return check(lib().findCellStart(_ptr(phash), _ptr(cstart), int(n), int(ncells)), "findCellStart")

    @staticmethod
    def neighborarray(pos, phash, cstart, grid, cell, origin, maxppc, n, anei, njgi, njli):
        return check(lib().neighborarray(_ptr(pos), _ptr(phash), _ptr(cstart), _u3(grid), _d3(cell), _d3(origin),
                                         int(maxppc), int(n), _ptr(anei), _ptr(njgi), _ptr(njli)), "neighborarray")

    @staticmethod
    def prefixsum(n, njgi, sjgi, oldsjgi):
        tot = ctypes.c_uint(0)
        check(lib().prefixsum(int(n), _ptr(njgi), _ptr(sjgi), _ptr(oldsjgi), ctypes.byref(tot)), "prefixsum")
        return tot.value

    @staticmethod
    def pairlist(sjgi, oldsjgi, oldln, anei, njgi, njli, olddispt, oldfricp, maxppc, maxcn, n, aref, lp, ln,
                 dispt, fricp):
        return check(lib().pairlist(_ptr(sjgi), _ptr(oldsjgi), _ptr(oldln), _ptr(anei), _ptr(njgi), _ptr(njli),
                                    _ptr(olddispt), _ptr(oldfricp), int(maxppc), int(maxcn), int(n), _ptr(aref),
                                    _ptr(lp), _ptr(ln), _ptr(dispt), _ptr(fricp)), "pairlist")

    @staticmethod
    def calculateforcepair(pos, pdis, angv, rad, rmass, lp, ln, oldln, dispt, fricp, olddispt, oldfricp, dt,
                           forcepair, torqpairi, torqpairj, contactpair, total):
        return check(lib().calculateforcepair(_ptr(pos), _ptr(pdis), _ptr(angv), _ptr(rad), _ptr(rmass), _ptr(lp),
                                              _ptr(ln), _ptr(oldln), _ptr(dispt), _ptr(fricp), _ptr(olddispt),
                                              _ptr(oldfricp), float(dt), _ptr(forcepair), _ptr(torqpairi),
                                              _ptr(torqpairj), _ptr(contactpair), int(total)), "calculateforcepair")

    @staticmethod
    def sumallforcei(maxppc, n, njgi, njli, forcepair, torqpairi, torqpairj, contactpair, aref, forcei, torquei,
                     contacti):
        return check(lib().sumallforcei(int(maxppc), int(n), _ptr(njgi), _ptr(njli), _ptr(forcepair),
                                        _ptr(torqpairi), _ptr(torqpairj), _ptr(contactpair), _ptr(aref),
                                        _ptr(forcei), _ptr(torquei), _ptr(contacti)), "sumallforcei")

    @staticmethod
    def calculateforceiw(world, pos, pdis, angv, rad, rmass, dt, total, n, disptw, fricpw, forcei, torquei):
        return check(lib().calculateforceiw(_d3(world), _ptr(pos), _ptr(pdis), _ptr(angv), _ptr(rad), _ptr(rmass),
                                            float(dt), int(total), int(n), _ptr(disptw), _ptr(fricpw),
                                            _ptr(forcei), _ptr(torquei)), "calculateforceiw")

    @staticmethod
    def updateposition(world, n, pos, pdis, angv, rmass, inert, forcei, torquei, qi, dt, cdamp=0.0):
        iall = ctypes.c_uint(0)
        mz = ctypes.c_double(0.0)
        check(lib().updateposition(_d3(world), int(n), _ptr(pos), _ptr(pdis), _ptr(angv), _ptr(rmass), _ptr(inert),
                                   _ptr(forcei), _ptr(torquei), _ptr(qi), float(dt), float(cdamp),
                                   ctypes.byref(iall), ctypes.byref(mz)), "updateposition")
        return iall.value, mz.value

    @staticmethod
    def outputporositycn(n, contacti, maxhz, world):
        pc = ctypes.c_uint(0)
        check(lib().outputporositycn(int(n), _ptr(contacti), float(maxhz), _d3(world), ctypes.byref(pc)),
              "outputporositycn")
        return pc.value


# ------------------------------------------------------------------ engine
def contact(estar, mu, nu, damp_n, damp_t, roll=0.0, roll_rel=0.0):
    return dict(estar=estar, mu=mu, nu=nu, damp_n=damp_n, damp_t=damp_t, roll=roll, roll_rel=roll_rel)


def material_array(pp: dict, pw: dict):
    """14 doubles (pp then pw) in Contact field order (the oracle's layout)."""
    keys = [k for k, _ in Contact._fields_]
    return np.array([pp[k] for k in keys] + [pw[k] for k in keys], dtype=np.float64)


class Engine:
    """Owns a dem_ctx.  Host arrays are numpy float64 (AoS xyz-interleaved)."""

    def __init__(self, n, world, dt, skin, precision=PREC_MIXED, relist_interval=20, cell=0.0, density=1.0,
                 pair_capacity=0, force_mode=FORCE_PCCP):
        L = lib()
        cfg = Config()
        cfg.n = int(n)
        cfg.precision = int(precision)
        cfg.relist_interval = int(relist_interval)
        cfg.world = (ctypes.c_double * 3)(*world)
        cfg.dt = float(dt)
        cfg.skin = float(skin)
        cfg.cell = float(cell)
        cfg.density = float(density)
        cfg.pair_capacity = int(pair_capacity)
        cfg.force_mode = int(force_mode)
        self.n = int(n)
        self.cfg = cfg
        h = ctypes.c_void_p()
        check(L.dem_create(ctypes.byref(cfg), ctypes.byref(h)), "dem_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().dem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_handle):
        check(lib().dem_set_stream(self._h, ctypes.c_void_p(stream_handle)), "dem_set_stream")

    def set_material(self, pp: dict, pw: dict):
        m = Material(Contact(**pp), Contact(**pw))
        check(lib().dem_set_material(self._h, ctypes.byref(m)), "dem_set_material")

    def upload(self, pos, rad, pdis=None, angv=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        rad = np.ascontiguousarray(rad, dtype=np.float64).reshape(-1)
        pdis = None if pdis is None else np.ascontiguousarray(pdis, dtype=np.float64).reshape(-1)
        angv = None if angv is None else np.ascontiguousarray(angv, dtype=np.float64).reshape(-1)
        assert pos.size == 3 * self.n and rad.size == self.n
        check(lib().dem_upload_state(self._h, _ptr(pos), _ptr(pdis), _ptr(angv), _ptr(rad)), "dem_upload_state")

    def upload_device(self, pos, rad, pdis=None, angv=None):
        check(lib().dem_upload_state_device(self._h, _ptr(pos), _ptr(pdis), _ptr(angv), _ptr(rad)),
              "dem_upload_state_device")

    def step(self, nsteps):
        check(lib().dem_step_n(self._h, int(nsteps)), "dem_step_n")

    def scalars(self, raise_on_status=True):
        s = Scalars()
        rc = lib().dem_get_scalars(self._h, ctypes.byref(s))
        if raise_on_status:
            check(rc, "dem_get_scalars")
        return s.as_dict()

    def scalars_raw_bytes(self):
        v = ctypes.c_longlong(0)
        check(lib().dem_scalars_raw_bytes(self._h, ctypes.byref(v)), "dem_scalars_raw_bytes")
        return v.value

    def scalars_enqueue(self, raw_addr):
        """Queue the observables' copy into host memory at raw_addr (pinned
        for an asynchronous copy; scalars_raw_bytes() bytes); no wait."""
        check(lib().dem_scalars_enqueue(self._h, ctypes.c_void_p(raw_addr)), "dem_scalars_enqueue")

    def scalars_from_raw(self, raw_addr, raise_on_status=True):
        """Observables from a buffer filled by scalars_enqueue (after a sync)."""
        s = Scalars()
        rc = lib().dem_scalars_from_raw(self._h, ctypes.c_void_p(raw_addr), ctypes.byref(s))
        if raise_on_status:
            check(rc, "dem_scalars_from_raw")
        return s.as_dict()

    def synchronize(self):
        check(lib().dem_synchronize(self._h), "dem_synchronize")

    def download(self):
        pos = np.empty(3 * self.n)
        pdis = np.empty(3 * self.n)
        angv = np.empty(3 * self.n)
        check(lib().dem_download_state(self._h, _ptr(pos), _ptr(pdis), _ptr(angv)), "dem_download_state")
        return pos, pdis, angv

    def download_device(self, pos=None, pdis=None, angv=None):
        check(lib().dem_download_state_device(self._h, _ptr(pos), _ptr(pdis), _ptr(angv)),
              "dem_download_state_device")

    def record_forces(self, on=True):
        check(lib().dem_record_forces(self._h, 1 if on else 0), "dem_record_forces")

    def forces(self):
        f = np.empty(3 * self.n)
        t = np.empty(3 * self.n)
        c = np.empty(self.n, dtype=np.uint32)
        check(lib().dem_download_forces(self._h, _ptr(f), _ptr(t), _ptr(c)), "dem_download_forces")
        return f, t, c

    def pairs(self):
        npairs = ctypes.c_longlong(0)
        check(lib().dem_download_pairs(self._h, None, None, None, 0, ctypes.byref(npairs)), "dem_download_pairs")
        P = npairs.value
        lp = np.empty(max(P, 1), dtype=np.uint32)
        ln = np.empty(max(P, 1), dtype=np.uint32)
        hist = np.empty(3 * max(P, 1))
        if P:
            check(lib().dem_download_pairs(self._h, _ptr(lp), _ptr(ln), _ptr(hist), P, ctypes.byref(npairs)),
                  "dem_download_pairs")
        return lp[:P], ln[:P], hist[:3 * P]

    def grid_info(self):
        g = (ctypes.c_uint * 3)()
        cs = ctypes.c_double(0)
        nc = ctypes.c_longlong(0)
        check(lib().dem_grid_info(self._h, g, ctypes.byref(cs), ctypes.byref(nc)), "dem_grid_info")
        return tuple(g), cs.value, nc.value

    def cells(self):
        g, cs, nc = self.grid_info()
        keys = np.empty(self.n, dtype=np.uint32)
        ids = np.empty(self.n, dtype=np.uint32)
        st = np.empty(nc, dtype=np.uint32)
        en = np.empty(nc, dtype=np.uint32)
        check(lib().dem_download_cells(self._h, _ptr(keys), _ptr(ids), _ptr(st), _ptr(en), nc), "dem_download_cells")
        return keys, ids, st, en

    def adjoint(self, nsteps, checkpoint_every, objective=OBJ_PACKING, radii=True):
        """Reverse mode over a window: returns the objective, its gradients
        with respect to the contact parameters (pp, pw) and every radius, and
        the device times of the forward and of the reverse sweep."""
        r = AdjointResult()
        dr = np.zeros(self.n) if radii else None
        check(lib().dem_adjoint_window(self._h, int(nsteps), int(checkpoint_every), int(objective), ctypes.byref(r),
                                       _ptr(dr)), "dem_adjoint_window")
        keys = [k for k, _ in Contact._fields_]
        return {"value": r.value, "d_pp": {k: getattr(r.d_pp, k) for k in keys},
                "d_pw": {k: getattr(r.d_pw, k) for k in keys}, "d_radii": dr, "forward_ms": r.forward_ms,
                "adjoint_ms": r.adjoint_ms}

    def adjoint_release(self):
        check(lib().dem_adjoint_release(self._h), "dem_adjoint_release")

    def set_profiling(self, on=True):
        check(lib().dem_set_profiling(self._h, 1 if on else 0), "dem_set_profiling")

    def kernel_times(self):
        out = (ctypes.c_double * 3)()
        check(lib().dem_kernel_times(self._h, out), "dem_kernel_times")
        return {"relist_ms": out[0], "pair_ms": out[1], "particle_ms": out[2]}

    def save_state(self, path):
        check(lib().dem_save_state(self._h, str(path).encode()), "dem_save_state")

    def load_state(self, path):
        check(lib().dem_load_state(self._h, str(path).encode()), "dem_load_state")

    def set_pour(self, nplayer, tnewpar, n_active=0):
        """Poured packing (dem_set_pour): the uploaded states are injection
        states; n_active particles are in the system, and nplayer more join
        before every step whose time dt*it passes N*tnewpar/nplayer."""
        check(lib().dem_set_pour(self._h, int(nplayer), float(tnewpar), int(n_active)), "dem_set_pour")

    def check_barrier_timeout(self):
        """Run one grid-barrier wait that cannot complete (dem_check_barrier_timeout):
        it must give up and report DEM_ERR_TIMEOUT; returns the ms waited."""
        ms = ctypes.c_double(0.0)
        check(lib().dem_check_barrier_timeout(self._h, ctypes.byref(ms)), "dem_check_barrier_timeout")
        return ms.value

    def active_count(self):
        v = ctypes.c_longlong(0)
        check(lib().dem_active_count(self._h, ctypes.byref(v)), "dem_active_count")
        return v.value

    def set_window_timing(self, on=True):
        check(lib().dem_set_window_timing(self._h, 1 if on else 0), "dem_set_window_timing")

    def window_work(self):
        """Bound particles, wall candidates and listed pairs of the current
        list's window, and whether its bound particles were stepped as cluster
        batches (dem_window_work)."""
        b, w, p, bt = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_int(0)
        check(lib().dem_window_work(self._h, ctypes.byref(b), ctypes.byref(w), ctypes.byref(p), ctypes.byref(bt)),
              "dem_window_work")
        return {"bound": b.value, "wall_candidates": w.value, "pairs": p.value, "batched": bt.value}

    def window_kernel_times(self):
        out = (ctypes.c_double * 5)()
        check(lib().dem_window_kernel_times(self._h, out), "dem_window_kernel_times")
        return {"relist_ms": out[0], "pair_ms": out[1], "particle_ms": out[2], "free_window_ms": out[3],
                "window_kernel_ms": out[4]}


# ------------------------------------------------------------ host helpers
def read_deck(path):
    d = Deck()
    check(lib().dem_read_deck(str(path).encode(), ctypes.byref(d)), "dem_read_deck")
    return d


def deck_material(deck):
    m = Material()
    check(lib().dem_deck_material(ctypes.byref(deck), ctypes.byref(m)), "dem_deck_material")
    keys = [k for k, _ in Contact._fields_]
    return {k: getattr(m.pp, k) for k in keys}, {k: getattr(m.pw, k) for k in keys}


def gen_lattice(n, spacing, nx, ny, z0, jitter, radius, seed):
    pos = np.empty(3 * n)
    rad = np.empty(n)
    check(lib().dem_gen_lattice(int(n), float(spacing), int(nx), int(ny), float(z0), float(jitter), float(radius),
                                int(seed), _ptr(pos), _ptr(rad)), "dem_gen_lattice")
    return pos, rad


def gen_radii(n, kind, a, b=0.0, c=0.0, d=0.0, seed=0):
    rad = np.empty(n)
    check(lib().dem_gen_radii(int(n), int(kind), float(a), float(b), float(c), float(d), int(seed), _ptr(rad)),
          "dem_gen_radii")
    return rad


def gen_rsa(world, rad, seed):
    rad = np.ascontiguousarray(rad, dtype=np.float64)
    pos = np.empty(3 * rad.size)
    check(lib().dem_gen_rsa(int(rad.size), _d3(world), _ptr(rad), int(seed), _ptr(pos)), "dem_gen_rsa")
    return pos


def read_preflow(path):
    it, n, itime = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    check(lib().dem_read_preflow(str(path).encode(), ctypes.byref(it), ctypes.byref(n), ctypes.byref(itime), None,
                                 None, None, 0), "dem_read_preflow")
    pos, pdis, angv = np.empty(3 * n.value), np.empty(3 * n.value), np.empty(3 * n.value)
    check(lib().dem_read_preflow(str(path).encode(), ctypes.byref(it), ctypes.byref(n), ctypes.byref(itime),
                                 _ptr(pos), _ptr(pdis), _ptr(angv), n.value), "dem_read_preflow")
    return it.value, itime.value, pos, pdis, angv


def estar(E, nu, rho, dref):
    return lib().dem_estar(float(E), float(nu), float(rho), float(dref))


def damp_from_restitution(e):
    return lib().dem_damp_from_restitution(float(e))


def reduced_modulus(E, rho, dref):
    return lib().dem_reduced_modulus(float(E), float(rho), float(dref))
