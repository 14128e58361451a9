"""Workloads of the DEM packing step, in the reference's reduced units.

Length unit d_ref = 1 mm (the median diameter), time unit tau = sqrt(d_ref/g)
= 0.010096 s, mass unit rho*pi*d_ref^3/6 (dempacking.cu:146-149,213-225,311).
All share E = 1e7 Pa, nu = 0.29, rho = 2500 kg/m^3, restitution 0.5 (viscous
damping, normal and tangential), flat frictional walls, gravity -z, skin
0.1*R with R the median radius (0.05 d), re-list every 20 steps.

  lattice_2k     2,000 monodisperse r = 0.5 mm, 20x20x100 mm box, cubic lattice
                 a = 1.1 mm (18x18 per layer), jitter +-0.04 mm, dt = 1e-6 s,
                 20,000 steps, mu = 0.3, mu_r = 0.002 R*.  FP64.
  rsa_500k       500,000 lognormal radii (median 0.5 mm, sigma 0.2, [0.3, 0.8] mm)
                 placed by random sequential addition in 100x100x400 mm,
                 dt = 5e-7 s, 10,000 steps, mu = 0.3, mu_r = 0.002 R*.
                 FP64 (plain form) or mixed precision.
  bidisperse_4m  4,000,000 radii 0.4/0.6 mm 1:1, 200x200x600 mm, dt = 4e-7 s,
                 5,000 steps, mu = 0.5, mu_r = 0.005 R*.  Mixed precision.
  settle_50k     50,000 lognormal (as rsa_500k) in 40x40x150 mm, dt = 5e-7 s,
                 pre-settled 20,000 steps, then a 2,000-step window.
  bed_500k       the rsa_500k spheres as a settled bed (every sphere in
                 contact): RSA largest first at solid fraction 0.32 in a
                 100x100 mm base, compacted by a downward velocity
                 proportional to height and gravity with restitution 0.1,
                 then quenched (velocities zeroed) ten times 500 steps apart
                 (dense_bed()); then stepped as rsa_500k.
  pour_box       a poured packing (the reference's layer injection) at test
                 size: 108 spheres r = 0.5 mm in 8x8 mm, 3 layers of 36 on a
                 6x6 injection lattice 3 mm above the floor, initial speed 1.5
                 (reduced) in the reference's random downward directions, a
                 layer every 1507 steps (each layer has left the injection
                 height before the next arrives), dt = 5e-4 (reduced), skin
                 0.55 (the reference's cub - cua).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import PREC_FP64, PREC_MIXED, RADII_BIDISPERSE, RADII_LOGNORMAL, contact
# host-only generators (libdem_gen.so): a workload never loads the GPU library
from .gen import damp_from_restitution, estar, gen_lattice, gen_radii, gen_rsa

D_REF = 1e-3                       # m
G = 9.81
TAU = math.sqrt(D_REF / G)         # s
SEED = 20261203


def reduced_dt(dt_seconds):
    return dt_seconds / TAU


def material(E=1e7, nu=0.29, rho=2500.0, mu=0.3, mu_w=None, roll_rel=0.002, e=0.5):
    """pp and pw contact dicts (reduced units).  Rolling length roll_rel * R*."""
    es = estar(E, nu, rho, D_REF)
    c = damp_from_restitution(e)
    pp = contact(es, mu, nu, c, c, 0.0, roll_rel)
    pw = contact(es, mu if mu_w is None else mu_w, nu, c, c, 0.0, roll_rel)
    return pp, pw


@dataclass
class Workload:
    name: str
    n: int
    pos: np.ndarray
    rad: np.ndarray
    world: tuple
    dt: float
    steps: int
    relist_interval: int
    skin: float
    precision: int
    pp: dict
    pw: dict
    density: float = 1.0
    pair_capacity: int = 0
    meta: dict = field(default_factory=dict)

    def cell(self):
        return 2.0 * float(self.rad.max()) + self.skin + 1e-4

    def engine_kwargs(self):
        return dict(n=self.n, world=self.world, dt=self.dt, skin=self.skin, precision=self.precision,
                    relist_interval=self.relist_interval, density=self.density, pair_capacity=self.pair_capacity)


def lattice_2k(seed=SEED, n=2000):
    a = 1.1
    pos, rad = gen_lattice(n, a, 18, 18, 0.55, 0.04, 0.5, seed)
    pp, pw = material(mu=0.3, roll_rel=0.002)
    return Workload("lattice_2k", n, pos, rad, (20.0, 20.0, 100.0), reduced_dt(1e-6), 20000, 20, 0.05, PREC_FP64,
                    pp, pw, meta={"init": "cubic lattice a=1.1 mm, jitter 0.04 mm"})


def rsa_500k(seed=SEED, precision=PREC_MIXED, n=500_000, box=(100.0, 100.0, 400.0)):
    rad = gen_radii(n, RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed)
    pos = gen_rsa(box, rad, seed + 1)
    pp, pw = material(mu=0.3, roll_rel=0.002)
    name = "rsa_500k" if n == 500_000 else f"rsa_{n}"
    return Workload(name, n, pos, rad, tuple(box), reduced_dt(5e-7), 10000, 20, 0.05, precision, pp, pw,
                    meta={"init": "RSA, lognormal radii median 0.5 mm sigma 0.2 in [0.3,0.8] mm"})


def bidisperse_4m(seed=SEED, n=4_000_000, box=(200.0, 200.0, 600.0)):
    rad = gen_radii(n, RADII_BIDISPERSE, 0.4, 0.6, 0.0, 0.0, seed)
    pos = gen_rsa(box, rad, seed + 1)
    pp, pw = material(mu=0.5, roll_rel=0.005)
    return Workload("bidisperse_4m", n, pos, rad, tuple(box), reduced_dt(4e-7), 5000, 20, 0.05, PREC_MIXED, pp, pw,
                    meta={"init": "RSA, radii 0.4/0.6 mm 1:1"})


def settle_50k(seed=SEED, n=50_000, box=(40.0, 40.0, 150.0)):
    rad = gen_radii(n, RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed)
    pos = gen_rsa(box, rad, seed + 1)
    pp, pw = material(mu=0.3, roll_rel=0.002)
    return Workload("settle_50k", n, pos, rad, tuple(box), reduced_dt(5e-7), 2000, 20, 0.05, PREC_MIXED, pp, pw,
                    meta={"init": "RSA then 20,000 settling steps", "presettle_steps": 20000})


def small_box(n=3000, box=(16.0, 16.0, 40.0), seed=SEED, precision=PREC_FP64, compress=1.0):
    """A small polydisperse case for parity tests: RSA (solid fraction about
    0.16), optionally compressed towards the floor and the box axis by the
    factor `compress` (< 1 creates overlapping contacts)."""
    rad = gen_radii(n, RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed)
    pos = gen_rsa(box, rad, seed + 1)
    if compress != 1.0:
        p = pos.reshape(-1, 3)
        p[:, 0] *= compress
        p[:, 1] *= compress
        p[:, 2] = rad + (p[:, 2] - rad) * compress
        pos = p.reshape(-1).copy()
    pp, pw = material(mu=0.3, roll_rel=0.002)
    return Workload("small_box", n, pos, rad, tuple(box), reduced_dt(5e-7), 200, 20, 0.05, precision, pp, pw)


def pour_box(seed=SEED, nx=6, ny=6, layers=3, box=(8.0, 8.0, 12.0), z_inject=3.0, vel0=1.5, dt=5e-4,
             layer_steps=1507.0, precision=PREC_FP64):
    """Poured packing at test size.  Injection states of all particles:
    nx*ny lattice sites per layer (dempacking.cu:253-279), every layer at the
    same height, speed vel0 at elevation pi*(u/3 + 1/3) below the horizontal
    and a uniform azimuth (:302-309, seeded).  meta: pdis (displacement per
    step), nplayer, tnewpar (one layer per layer_steps steps)."""
    rng = np.random.default_rng(seed)
    n = nx * ny * layers
    W, T = box[0], box[1]
    xs = ((np.arange(nx) + 0.5) / nx - 0.5) * W
    ys = ((np.arange(ny) + 0.5) / ny - 0.5) * T
    site = np.array([(x, y) for x in xs for y in ys])
    pos = np.zeros((n, 3))
    pos[:, :2] = np.tile(site, (layers, 1))
    pos[:, 2] = z_inject
    ang = np.pi * (rng.random(n) / 3.0 + 1.0 / 3.0)
    az = 2.0 * np.pi * rng.random(n)
    pdis = np.zeros((n, 3))
    pdis[:, 2] = -vel0 * np.sin(ang) * dt
    dxy = -vel0 * np.cos(ang) * dt
    pdis[:, 0] = dxy * np.cos(az)
    pdis[:, 1] = dxy * np.sin(az)
    rad = np.full(n, 0.5)
    pp, pw = material(mu=0.3, roll_rel=0.002)
    w = Workload("pour_box", n, pos.reshape(-1), rad, tuple(box), dt, int(layer_steps * layers), 20, 0.55,
                 precision, pp, pw,
                 meta={"pdis": pdis.reshape(-1), "nplayer": nx * ny, "tnewpar": layer_steps * dt,
                       "init": f"poured: {nx}x{ny} injection lattice, a layer every {layer_steps:g} steps"})
    return w


def bed_500k_initial(seed=SEED, precision=PREC_MIXED, n=500_000, base=(100.0, 100.0), phi0=0.32, phi_bed=0.55,
                     compact_s=0.0125):
    """Initial state of the settled 500,000-sphere bed: the rsa_500k radii
    placed by random sequential addition largest first (which reaches solid
    fraction phi0 = 0.32; in random order RSA stops near 0.25) in a
    base[0] x base[1] box of height V / (phi0 A), with a downward velocity
    proportional to height, z (1 - phi0/phi_bed) / compact_s, so that the
    column closes to about phi_bed in compact_s seconds with gentle
    neighbour impacts (relative speeds ~ gap x 46/s).  meta["pdis"]: the
    per-step displacement (velocity x dt) of that motion at dt = 5e-7 s."""
    rad = gen_radii(n, RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed)
    V = float(np.sum(4.0 / 3.0 * np.pi * rad ** 3))
    H = V / (phi0 * base[0] * base[1])
    order = np.argsort(-rad, kind="stable")
    ps = gen_rsa((base[0], base[1], H), rad[order], seed + 1).reshape(-1, 3)
    pos = np.empty_like(ps)
    pos[order] = ps
    dt = reduced_dt(5e-7)
    vz = -pos[:, 2] * (1.0 - phi0 / phi_bed) / (compact_s / TAU)     # reduced velocity
    pdis = np.zeros_like(pos)
    pdis[:, 2] = vz * dt
    pp, pw = material(mu=0.3, roll_rel=0.002)
    world = (base[0], base[1], float(np.ceil(H + 5.0)))
    return Workload("bed_500k", n, pos.reshape(-1).copy(), rad, world, dt, 10000, 20, 0.05, precision, pp, pw,
                    meta={"init": f"RSA largest first at phi {phi0} in {base[0]:g}x{base[1]:g}x{H:.1f} mm, "
                                  f"compacted in {compact_s * 1e3:g} ms then settled",
                          "pdis": pdis.reshape(-1).copy(), "compact_steps": int(round(compact_s / 5e-7))})


def dense_bed(dem, w, settle_steps, relist=10, stream=None, e_settle=0.1, quench_cycles=10, quench_every=500,
              log=None):
    """Settles bed_500k_initial's column on the GPU and returns the bed as a
    Workload at the production cadence (re-list every 20 steps) with its
    state: pos, and pdis/angv in meta.  Mixed precision, re-list every
    `relist` steps (the compaction's fastest spheres stay inside the skin
    guard), restitution e_settle (the returned workload keeps its own
    material): `settle_steps` of compaction, then `quench_cycles` times the
    velocities set to zero (an upload of the positions alone) and
    `quench_every` steps, which drains the kinetic and elastic energy the
    compaction left, so that the bed rests under gravity instead of
    rebounding.  log(stage, scalars) is called after each stage."""
    e = dem.Engine(**{**w.engine_kwargs(), "precision": PREC_MIXED, "relist_interval": relist})
    if stream is not None:
        e.set_stream(stream)
    e.set_material(*material(mu=0.3, roll_rel=0.002, e=e_settle))
    e.upload(w.pos, w.rad, w.meta["pdis"], None)
    e.step(settle_steps)
    if log:
        log("compaction", e.scalars(raise_on_status=False))
    for q in range(quench_cycles):
        pos, _, _ = e.download()
        e.upload(pos, w.rad)
        e.step(quench_every)
        if log:
            log(f"quench {q + 1}", e.scalars(raise_on_status=False))
    s = e.scalars()
    pos, pdis, angv = e.download()
    e.close()
    meta = dict(w.meta)
    meta.update(pdis=pdis, angv=angv, settle_steps=settle_steps + quench_cycles * quench_every, settled=s)
    return Workload(w.name, w.n, pos, w.rad, w.world, w.dt, w.steps, 20, w.skin, w.precision, w.pp, w.pw,
                    meta=meta)
