"""Parity at the configurations' own sizes and lengths against the FP64
oracle (the CPU restatement of the reference step), with the errors stated.

* 500,000 lognormal spheres (RSA, 100x100x400 mm, dt 5e-7 s), the full
  10,000 steps (500 re-lists) from the initial state, one FP64 oracle run
  compared with the FP64 plain engine and with the mixed engine (FP32
  list/forces/accumulation, FP64 positions, velocities and history).
  Observables of dempacking.cu:766-776: packing fraction (tolerance 1e-3),
  mean coordination number (0.02), and the per-particle position RMS
  (FP64 1e-10 d, mixed 1e-5 d).
* 4,000,000 bidisperse spheres (200x200x600 mm, dt 4e-7 s, mu 0.5), a
  200-step sub-window (10 re-lists), mixed engine against the oracle.
* 50,000 lognormal spheres pre-settled 20,000 steps, then the 2,000-step
  mixed window with checkpoints every 100: gradients of the potential energy
  with respect to sliding and rolling friction against central differences
  of the GPU forward and of the FP64 oracle.

The packing-fraction objective has zero friction gradients on that window:
it is sum (4/3) pi r^3 / (Wx Wy max z), and the highest sphere is in free
fall for the whole window (20,000 + 2,000 steps of 5e-7 s = 11 ms, a fall of
0.6 mm), touching nothing, so max z does not depend on any contact
parameter.  The potential energy sum m g z + elastic energy does: spheres
that hit the floor bounce into the spheres falling above them, and those
oblique impacts load the tangential springs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_engine(dem, w, precision, steps, pdis=None, angv=None, pos=None, mat=None):
    e = dem.Engine(**{**w.engine_kwargs(), "precision": precision})
    e.set_material(*(mat or (w.pp, w.pw)))
    e.upload(w.pos if pos is None else pos, w.rad, pdis, angv)
    e.step(steps)
    s = e.scalars()
    out = e.download()
    cell = e.grid_info()[1]
    e.close()
    return s, out, cell


def packing_fraction(rad, world, maxhz):
    return np.sum(4.0 / 3.0 * np.pi * rad ** 3) / (world[0] * world[1] * maxhz)


@pytest.fixture(scope="module")
def config3(dem, orc, wl):
    w = wl.rsa_500k(precision=dem.PREC_FP64)
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, w.cell(), w.density, dem.material_array(w.pp, w.pw), False,
                w.steps, w.relist_interval, cap=2 * w.n, scalars=True)
    assert o["status"] == 0
    return w, o


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_config3_full_run_against_oracle(dem, wl, cuda, config3, prec):
    """500,000 spheres, all 10,000 steps: final packing fraction, mean
    coordination number and per-particle position RMS against the FP64
    oracle."""
    w, o = config3
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    s, (pos, pdis, angv), cell = run_engine(dem, w, p, w.steps)
    assert abs(cell - w.cell()) < 1e-15
    assert s["status"] == 0 and s["relists"] == w.steps // w.relist_interval
    rms = float(np.sqrt(np.mean((pos - o["pos"]) ** 2)))
    vrms = float(np.sqrt(np.mean((pdis - o["pdis"]) ** 2))) / w.dt
    phi_o = packing_fraction(w.rad, w.world, o["maxhz"][-1])
    cn_o = 2.0 * float(o["ncontacts"][-1]) / w.n
    dphi = abs(s["packing_fraction"] - phi_o)
    dcn = abs(s["mean_cn"] - cn_o)
    contacts_seen = int(np.max(o["ncontacts"]))
    print(f"\nconfig3 {prec}: |dphi| {dphi:.3e} (phi {phi_o:.7f}) |dCN| {dcn:.3e} (CN {cn_o:.4f}) "
          f"pos RMS {rms:.3e} d  vel RMS {vrms:.3e}  max contacts {contacts_seen}  pairs {s['pairs']}")
    assert contacts_seen > 0                       # collisions happen in the run
    assert dphi <= 1e-3 and dcn <= 0.02
    if prec == "fp64":
        assert rms <= 1e-10, rms
        assert s["contacts"] == int(o["ncontacts"][-1])
        assert s["pairs"] == int(o["npairs"][-1])    # the same FP64 list
    else:
        assert rms <= 1e-5, rms


def test_config4_subwindow_against_oracle(dem, orc, wl, cuda):
    """4,000,000 bidisperse spheres, 200 steps (10 re-lists): the mixed engine
    against the FP64 oracle (FP32 candidate test, so the lists agree)."""
    w = wl.bidisperse_4m()
    steps = 10 * w.relist_interval
    s, (pos, pdis, _), cell = run_engine(dem, w, dem.PREC_MIXED, steps)
    assert s["status"] == 0 and s["relists"] == 10
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(w.pp, w.pw), True, steps,
                w.relist_interval, cap=2 * w.n)
    assert o["status"] == 0
    rms = float(np.sqrt(np.mean((pos - o["pos"]) ** 2)))
    dphi = abs(s["packing_fraction"] - packing_fraction(w.rad, w.world, o["maxhz"][-1]))
    print(f"\nconfig4 mixed 200 steps: pos RMS {rms:.3e} d  |dphi| {dphi:.3e}  pairs {s['pairs']} / "
          f"{int(o['npairs'][-1])}  contacts {s['contacts']} / {int(o['ncontacts'][-1])}")
    assert rms <= 1e-6, rms
    assert dphi <= 1e-3
    assert abs(s["pairs"] - int(o["npairs"][-1])) <= max(2, s["pairs"] // 10000)
    assert abs(s["contacts"] - int(o["ncontacts"][-1])) <= max(2, s["contacts"] // 1000)


def energy_parts(pos, rad, lp, ln, world, density, pp, pw):
    """The potential-energy objective sum m z + (2/5) E* sqrt(R*) delta^2.5
    (touching listed pairs and walls; reduced units) as the per-particle
    m z terms and the elastic sum, so that central differences can subtract
    the large gravity term particle by particle instead of as two totals."""
    p = pos.reshape(-1, 3)
    mz = density * 8.0 * rad ** 3 * p[:, 2]
    lp = lp.astype(np.int64)
    ln = ln.astype(np.int64)
    D = p[ln] - p[lp]
    dist = np.sqrt((D ** 2).sum(1))
    d = rad[lp] + rad[ln] - dist
    t = d > 0
    Rs = rad[lp] * rad[ln] / (rad[lp] + rad[ln])
    el = float(np.sum(0.4 * pp["estar"] * np.sqrt(Rs[t]) * d[t] ** 2.5))
    hx, hy = world[0] / 2, world[1] / 2
    for dl in (rad - p[:, 2], rad - (p[:, 0] + hx), rad - (hx - p[:, 0]), rad - (p[:, 1] + hy), rad - (hy - p[:, 1])):
        t = dl > 0
        el += float(np.sum(0.4 * pw["estar"] * np.sqrt(rad[t]) * dl[t] ** 2.5))
    return mz, el


def central_difference(plus, minus, h):
    (mzp, elp), (mzm, elm) = plus, minus
    return (float(np.sum(mzp - mzm)) + (elp - elm)) / (2 * h)


def scaled(c, key, f):
    c = dict(c)
    c[key] = c[key] * f
    return c


def test_config5_friction_gradients(dem, orc, wl, cuda):
    """50,000 spheres pre-settled 20,000 steps, 2,000-step mixed window with
    checkpoints every 100: d(potential energy)/d(log mu) and d/d(log mu_r)
    (particle-particle and particle-wall together) from the adjoint against
    central differences with step 1e-4 relative, of the GPU forward (same
    precision) and of the FP64 oracle (from the same pre-settled state).  The
    differences subtract the two runs' energies particle by particle (the
    gravity term is ~1e6 times the gradient).  Tolerance 1e-3 relative for
    the sliding friction.  The rolling-friction gradient is 5e-4 of the
    sliding one here (only the few spheres that bounced off the floor roll):
    against the FP64 oracle's differences (step 1e-4) it is held to 1e-2
    relative; the mixed forward's differences at step 1e-4 are dominated by
    the FP32 torques' rounding (the energy change is ~1e-8 of a 4e6
    objective), so the GPU differences for it take the step 1e-2 and the
    tolerance 5e-2."""
    w = wl.settle_50k()
    s0, (pos, pdis, angv), cell = run_engine(dem, w, dem.PREC_MIXED, w.meta["presettle_steps"])
    assert s0["status"] == 0
    cellw = w.cell() + 0.01

    def adjoint(pp, pw):
        x = dem.Engine(**{**w.engine_kwargs(), "cell": cellw})
        x.set_material(pp, pw)
        x.upload(pos, w.rad, pdis, angv)
        r = x.adjoint(w.steps, 100, dem.OBJ_POTENTIAL, radii=False)
        assert x.scalars()["status"] == 0
        x.close()
        return r

    def gpu_parts(pp, pw):
        x = dem.Engine(**{**w.engine_kwargs(), "cell": cellw})
        x.set_material(pp, pw)
        x.upload(pos, w.rad, pdis, angv)
        x.step(w.steps)
        assert x.scalars()["status"] == 0
        p, _, _ = x.download()
        lp, ln, _ = x.pairs()
        x.close()
        return energy_parts(p, w.rad, lp, ln, w.world, w.density, pp, pw)

    def oracle_parts(pp, pw):
        o = orc.run(pos, w.rad, w.world, w.dt, w.skin, cellw, w.density, dem.material_array(pp, pw), False,
                    w.steps, w.relist_interval, pdis=pdis, angv=angv, cap=4 * w.n, scalars=False)
        assert o["status"] == 0
        lp = np.repeat(np.arange(w.n), np.diff(o["list_off"].astype(np.int64)))
        return energy_parts(o["pos"], w.rad, lp, o["list_ln"], w.world, w.density, pp, pw)

    base = adjoint(w.pp, w.pw)
    assert base["value"] > 0
    h_or = 1e-4
    h_gpu = {"mu": 1e-4, "roll_rel": 1e-2}
    rows = []
    for key in ("mu", "roll_rel"):
        g_ad = (base["d_pp"][key] * w.pp[key] + base["d_pw"][key] * w.pw[key])   # d/d(log parameter)
        h = h_gpu[key]
        g_fd = central_difference(gpu_parts(scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h)),
                                  gpu_parts(scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h)), h)
        h = h_or
        g_or = central_difference(oracle_parts(scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h)),
                                  oracle_parts(scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h)), h)
        print(f"\nconfig5 d U / d log {key}: adjoint {g_ad:.6e}  GPU FD {g_fd:.6e}  oracle FD {g_or:.6e}  "
              f"(U {base['value']:.6e})")
        rows.append((key, g_ad, g_fd, g_or))
    tol = {"mu": (1e-3, 1e-3), "roll_rel": (5e-2, 1e-2)}
    for key, g_ad, g_fd, g_or in rows:
        assert g_ad != 0.0, key                    # the friction gradients of the energy are not zero
        t_fd, t_or = tol[key]
        assert abs(g_ad - g_fd) <= t_fd * abs(g_fd), (key, g_ad, g_fd)
        assert abs(g_ad - g_or) <= t_or * abs(g_or), (key, g_ad, g_or)
