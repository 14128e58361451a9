"""GPU adjoint of the DEM step over a window (dem_adjoint_window) against
central finite differences, on the GPU forward and on the FP64 CPU oracle.

Case: a polydisperse bed with ~3 persistent contacts per sphere and random
initial motion (sliding, rolling), 100 steps (5 re-lists with history carry),
checkpoints every 20 steps.  Derivatives of the packing fraction and of the
potential energy with respect to the sliding friction, the rolling friction,
the contact stiffness (Young's modulus), the damping (restitution) -- each
shared by particle-particle and particle-wall contacts -- and a random
direction in the space of all radii.  Tolerance: 1e-3 relative, plus an
absolute floor of 1e-8 of the objective for derivatives at the FD noise level
(FD step 1e-5 relative in FP64 for parameters, 1e-9 absolute for radii).

The bed is pressed 5e-4 d into the floor.  Left at exactly zero floor overlap,
every bottom sphere starts at the onset of its floor contact, where the
damping term (proportional to sqrt(overlap)) is not differentiable: central
differences in the radii then fail to converge as the step shrinks.
"""
import numpy as np
import pytest

from _cases import dense_lattice

pytestmark = pytest.mark.gpu

STEPS, EVERY = 100, 20
KEYS = {"mu": ("mu",), "roll_rel": ("roll_rel",), "estar": ("estar",), "damp": ("damp_n", "damp_t")}


def case(dem):
    w = dense_lattice(dem, nx=6, ny=6, nz=5, seed=3)
    pos = w.pos.reshape(-1, 3).copy()
    pos[:, 2] -= 5e-4
    w.pos = pos.reshape(-1)
    rng = np.random.default_rng(12)
    pdis = rng.normal(0, 3e-6, 3 * w.n)
    angv = rng.normal(0, 3e-5, 3 * w.n)
    return w, pdis, angv


def scaled(c: dict, key, f):
    c = dict(c)
    for k in KEYS[key]:
        c[k] = c[k] * f
    return c


def run_adjoint(dem, w, pdis, angv, pp, pw, rad, objective):
    e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64, "cell": w.cell() + 0.01})
    e.set_material(pp, pw)
    e.upload(w.pos, rad, pdis, angv)
    r = e.adjoint(STEPS, EVERY, objective)
    s = e.scalars()
    assert s["status"] == 0
    e.close()
    return r


def grad_from_adjoint(r, key):
    return sum(r["d_pp"][k] for k in KEYS[key]) * 1.0, sum(r["d_pw"][k] for k in KEYS[key])


def oracle_objective(orc, dem, w, pdis, angv, pp, pw, rad, objective, cell):
    o = orc.run(w.pos, rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(pp, pw), False, STEPS,
                w.relist_interval, pdis=pdis, angv=angv)
    p = o["pos"].reshape(-1, 3)
    area = w.world[0] * w.world[1]
    if objective == dem.OBJ_PACKING:
        return np.sum(4.0 / 3.0 * np.pi * rad ** 3) / (area * max(p[:, 2].max(), 0.0))
    m = w.density * 8.0 * rad ** 3
    U = np.sum(m * p[:, 2])
    d = p[:, None, :] - p[None, :, :]
    dist = np.sqrt((d ** 2).sum(-1))
    ov = rad[:, None] + rad[None, :] - dist
    iu = np.triu_indices(w.n, 1)
    ov = ov[iu]
    Rs = (rad[:, None] * rad[None, :] / (rad[:, None] + rad[None, :]))[iu]
    touch = ov > 0
    U += np.sum(0.4 * pp["estar"] * np.sqrt(Rs[touch]) * ov[touch] ** 2.5)
    hx, hy = w.world[0] / 2, w.world[1] / 2
    for dl in (rad - p[:, 2], rad - (p[:, 0] + hx), rad - (hx - p[:, 0]), rad - (p[:, 1] + hy), rad - (hy - p[:, 1])):
        t = dl > 0
        U += np.sum(0.4 * pw["estar"] * np.sqrt(rad[t]) * dl[t] ** 2.5)
    return U


@pytest.mark.parametrize("objective", [0, 1])
def test_adjoint_matches_finite_differences(dem, orc, cuda, objective):
    w, pdis, angv = case(dem)
    base = run_adjoint(dem, w, pdis, angv, w.pp, w.pw, w.rad, objective)
    assert np.isfinite(base["value"]) and base["value"] > 0
    cell = w.cell() + 0.01
    h = 1e-5
    floor = 1e-8 * abs(base["value"])   # FD noise floor of the objective
    for key in KEYS:
        g_ad = sum(grad_from_adjoint(base, key)) * w.pp[KEYS[key][0]]   # d/d(log parameter)
        vp = run_adjoint(dem, w, pdis, angv, scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h), w.rad, objective)
        vm = run_adjoint(dem, w, pdis, angv, scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h), w.rad, objective)
        g_fd = (vp["value"] - vm["value"]) / (2 * h)
        op = oracle_objective(orc, dem, w, pdis, angv, scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h), w.rad,
                              objective, cell)
        om = oracle_objective(orc, dem, w, pdis, angv, scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h), w.rad,
                              objective, cell)
        g_or = (op - om) / (2 * h)
        assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd) + floor, (key, g_ad, g_fd)
        assert abs(g_ad - g_or) <= 1e-3 * abs(g_or) + floor, (key, g_ad, g_or)
    # radii: directional derivative along a random direction
    rng = np.random.default_rng(5)
    v = rng.normal(size=w.n)
    g_ad = float(base["d_radii"] @ v)
    hr = 1e-9
    vp = run_adjoint(dem, w, pdis, angv, w.pp, w.pw, w.rad + hr * v, objective)
    vm = run_adjoint(dem, w, pdis, angv, w.pp, w.pw, w.rad - hr * v, objective)
    g_fd = (vp["value"] - vm["value"]) / (2 * hr)
    assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd), (g_ad, g_fd)


def sparse_case(dem):
    """Spheres pressed into the floor (wall contacts and no pair contact, one
    with a listed non-touching neighbour), a pair overlapping mid-air and
    approaching (a pair contact through the whole window), and a falling
    sphere listed with both of the pair but touching neither: the reverse
    step's paths for spheres with and without pair contacts side by side."""
    import dem_b200.workloads as wm
    pos = [1.2, 1.2, 0.4995, -1.2, 1.2, 0.4995, 1.2, -1.2, 0.4995, -1.2, -1.2, 0.4995, 2.24, 1.2, 0.4995,
           -0.4999, 0.0, 8.0, 0.4999, 0.0, 8.0, 0.0, 0.9, 8.0]
    rad = np.full(8, 0.5)
    pp, pw = wm.material(mu=0.3, roll_rel=0.002)
    w = wm.Workload("sparse", 8, np.array(pos), rad, (6.0, 6.0, 20.0), wm.reduced_dt(5e-7), 0, 20, 0.05,
                    dem.PREC_FP64, pp, pw)
    rng = np.random.default_rng(8)
    pdis = rng.normal(0, 2e-6, 24)
    pdis[15], pdis[18] = 0.05 * w.dt, -0.05 * w.dt
    angv = rng.normal(0, 2e-5, 24)
    return w, pdis, angv


def test_adjoint_spheres_with_and_without_pair_contacts(dem, cuda):
    """Bound spheres without pair contacts (wall contacts only; the forward's
    taped contact count lets their reverse step skip the pair loops) beside a
    pair in contact, against central differences of the potential energy in
    every contact parameter."""
    w, pdis, angv = sparse_case(dem)
    base = run_adjoint(dem, w, pdis, angv, w.pp, w.pw, w.rad, dem.OBJ_POTENTIAL)
    assert base["value"] > 0
    h = 1e-5
    floor = 1e-8 * abs(base["value"])
    for key in KEYS:
        g_ad = sum(grad_from_adjoint(base, key)) * w.pp[KEYS[key][0]]
        vp = run_adjoint(dem, w, pdis, angv, scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h), w.rad,
                         dem.OBJ_POTENTIAL)
        vm = run_adjoint(dem, w, pdis, angv, scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h), w.rad,
                         dem.OBJ_POTENTIAL)
        g_fd = (vp["value"] - vm["value"]) / (2 * h)
        assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd) + floor, (key, g_ad, g_fd)


def test_adjoint_leaves_forward_state(dem, cuda):
    """After dem_adjoint_window the context holds the state of a plain
    forward run of the same window, and its observables."""
    w, pdis, angv = case(dem)
    kw = {**w.engine_kwargs(), "precision": dem.PREC_FP64}
    a = dem.Engine(**kw)
    a.set_material(w.pp, w.pw)
    a.upload(w.pos, w.rad, pdis, angv)
    a.adjoint(STEPS, EVERY, dem.OBJ_POTENTIAL)
    b = dem.Engine(**kw)
    b.set_material(w.pp, w.pw)
    b.upload(w.pos, w.rad, pdis, angv)
    b.step(STEPS)
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)
    sa, sb = a.scalars(), b.scalars()
    assert sa["maxhz"] == sb["maxhz"] and sa["contacts"] == sb["contacts"] and sa["step"] == sb["step"]
    a.step(20)   # and it can continue
    assert a.scalars()["status"] == 0


def test_repeated_calls_and_material_change(dem, cuda):
    """One context, several calls: the adjoint's graphs are kept across calls
    of the same segment length, so a second call from the same state gives
    the same bits; after a material change (the graphs hold the contact
    parameters) it gives the new material's gradients, bit for bit those of
    a fresh context; another checkpoint interval recaptures."""
    w, pdis, angv = case(dem)
    kw = {**w.engine_kwargs(), "precision": dem.PREC_FP64, "cell": w.cell() + 0.01}
    e = dem.Engine(**kw)
    e.set_material(w.pp, w.pw)

    def call(every=EVERY):
        e.upload(w.pos, w.rad, pdis, angv)
        r = e.adjoint(STEPS, every, dem.OBJ_POTENTIAL)
        assert e.scalars()["status"] == 0
        return r

    r1, r2 = call(), call()
    assert r1["value"] == r2["value"] and r1["d_pp"] == r2["d_pp"] and r1["d_pw"] == r2["d_pw"]
    np.testing.assert_array_equal(r1["d_radii"], r2["d_radii"])
    pp2, pw2 = scaled(w.pp, "mu", 1.5), scaled(w.pw, "mu", 1.5)
    e.set_material(pp2, pw2)
    r3 = call()
    fresh = run_adjoint(dem, w, pdis, angv, pp2, pw2, w.rad, dem.OBJ_POTENTIAL)
    assert r3["d_pp"] == fresh["d_pp"] and r3["d_pw"] == fresh["d_pw"] and r3["value"] == fresh["value"]
    assert r3["d_pp"] != r1["d_pp"]
    r4 = call(every=2 * EVERY if STEPS % (2 * EVERY) == 0 else STEPS)
    assert abs(r4["value"] - r3["value"]) <= 1e-12 * abs(r3["value"])
    e.close()


def test_plain_and_programmatic_reverse_sweeps_agree(dem, cuda, monkeypatch):
    """The reverse steps launched programmatically (the default: each loads
    its tape before waiting for its predecessor) and plainly (DEM_B200_PDL=0)
    give the same objective and gradients bit for bit."""
    w, pdis, angv = case(dem)
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("DEM_B200_PDL", flag)
        out.append(run_adjoint(dem, w, pdis, angv, w.pp, w.pw, w.rad, dem.OBJ_POTENTIAL))
    a, b = out
    assert a["value"] == b["value"]
    assert a["d_pp"] == b["d_pp"] and a["d_pw"] == b["d_pw"]
    np.testing.assert_array_equal(a["d_radii"], b["d_radii"])


@pytest.mark.parametrize("which", ["dense", "sparse"])
def test_recompute_paths_agree(dem, cuda, monkeypatch, which):
    """The reverse sweep's recompute through the per-step kernels (window
    kernel off: tape from the force record, contact counts included) and
    through the window path (cluster batches where the components fit a
    block, else the grid-barrier window kernel, writing the tape) give the
    same objective and gradients bit for bit; the particle-parallel force
    mode (its own per-step kernel, whose forward agrees with the pair-parallel
    one to rounding) agrees within the gradient tolerance, 1e-3."""
    w, pdis, angv = case(dem) if which == "dense" else sparse_case(dem)

    def run(**env):
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64, "cell": w.cell() + 0.01,
                          "force_mode": dem.FORCE_PP if env.get("PP") else dem.FORCE_PCCP})
        e.set_material(w.pp, w.pw)
        e.upload(w.pos, w.rad, pdis, angv)
        r = e.adjoint(STEPS, EVERY, dem.OBJ_POTENTIAL)
        assert e.scalars()["status"] == 0
        e.close()
        return r

    a = run(DEM_B200_WINDOW="1")
    b = run(DEM_B200_WINDOW="0")
    assert a["value"] == b["value"]
    assert a["d_pp"] == b["d_pp"] and a["d_pw"] == b["d_pw"]
    np.testing.assert_array_equal(a["d_radii"], b["d_radii"])
    monkeypatch.setenv("DEM_B200_WINDOW", "1")
    c = run(PP="1")
    assert c["value"] == pytest.approx(a["value"], rel=1e-9)
    floor = 1e-8 * abs(a["value"])
    for key in KEYS:
        x, y = sum(grad_from_adjoint(a, key)), sum(grad_from_adjoint(c, key))
        assert abs(x - y) <= 1e-3 * abs(x) + floor, (key, x, y)
    v = np.random.default_rng(4).normal(size=w.n)
    x, y = float(a["d_radii"] @ v), float(c["d_radii"] @ v)
    assert abs(x - y) <= 1e-3 * abs(x), (x, y)


def test_adjoint_settle_50k_window(dem, wl, cuda):
    """The 50,000-sphere configuration: pre-settled 20,000 steps, then a
    2,000-step mixed-precision window with checkpoints every 100; gradients of
    the potential energy against central differences of the GPU forward."""
    w = wl.settle_50k()
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    e.step(w.meta["presettle_steps"])
    pos, pdis, angv = e.download()
    e.close()

    def value(pp, pw, rad, grads=False):
        x = dem.Engine(**{**w.engine_kwargs(), "cell": w.cell() + 0.01})
        x.set_material(pp, pw)
        x.upload(pos, rad, pdis, angv)
        r = x.adjoint(w.steps, 100, dem.OBJ_POTENTIAL, radii=grads)
        assert x.scalars()["status"] == 0
        x.close()
        return r

    base = value(w.pp, w.pw, w.rad, grads=True)
    floor = 1e-8 * abs(base["value"])
    h = 1e-4
    for key in ("estar", "damp"):
        g_ad = sum(grad_from_adjoint(base, key)) * w.pp[KEYS[key][0]]
        vp = value(scaled(w.pp, key, 1 + h), scaled(w.pw, key, 1 + h), w.rad)["value"]
        vm = value(scaled(w.pp, key, 1 - h), scaled(w.pw, key, 1 - h), w.rad)["value"]
        g_fd = (vp - vm) / (2 * h)
        assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd) + floor, (key, g_ad, g_fd)
    # radii are FP32 in the mixed form: a direction on the FP32 grid, scaled
    rng = np.random.default_rng(2)
    v = np.sign(rng.normal(size=w.n)) * 2.0 ** -16
    g_ad = float(base["d_radii"] @ v)
    vp = value(w.pp, w.pw, w.rad + v)["value"]
    vm = value(w.pp, w.pw, w.rad - v)["value"]
    g_fd = (vp - vm) / 2.0
    assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd), (g_ad, g_fd)


def test_autograd_function_matches_finite_differences(dem, wl, cuda):
    """The adjoint through a torch.autograd.Function of the physical
    parameters (tests/_adjoint_torch.py): torch.autograd.grad of the
    potential energy after the window with respect to Young's modulus,
    restitution, sliding and rolling friction and the radii, against central
    differences of the same window.  Tolerance 1e-3 relative plus the FD noise
    floor (1e-8 of the objective)."""
    import torch
    from _adjoint_torch import DemWindow, WindowSetup, window_value
    w, pdis, angv = case(dem)
    s = WindowSetup(dem, wl, w, w.pos, pdis, angv, STEPS, EVERY, dem.OBJ_POTENTIAL, dem.PREC_FP64, w.cell() + 0.01)
    p0 = {"E": 1e7, "e": 0.5, "mu": 0.3, "mu_r": 0.002}
    xs = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in p0.items()}
    rad = torch.tensor(w.rad, dtype=torch.float64, requires_grad=True)
    val = DemWindow.apply(xs["E"], xs["e"], xs["mu"], xs["mu_r"], rad, s)
    g = torch.autograd.grad(val, [xs["E"], xs["e"], xs["mu"], xs["mu_r"], rad])
    base = float(val.detach())
    assert np.isfinite(base) and base > 0
    floor = 1e-8 * abs(base)
    for idx, k in enumerate(("E", "e", "mu", "mu_r")):
        h = 1e-5 * p0[k] if k != "e" else 1e-5
        vp = window_value(s, **{**p0, k: p0[k] + h}, rad=w.rad)
        vm = window_value(s, **{**p0, k: p0[k] - h}, rad=w.rad)
        g_fd = (vp - vm) / (2 * h) * (p0[k] if k != "e" else 1.0)
        g_ad = float(g[idx]) * (p0[k] if k != "e" else 1.0)
        assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd) + floor, (k, g_ad, g_fd)
    rng = np.random.default_rng(7)
    v = rng.normal(size=w.n)
    hr = 1e-9
    g_fd = (window_value(s, **p0, rad=w.rad + hr * v) - window_value(s, **p0, rad=w.rad - hr * v)) / (2 * hr)
    g_ad = float(g[4].numpy() @ v)
    assert abs(g_ad - g_fd) <= 1e-3 * abs(g_fd), (g_ad, g_fd)


@pytest.mark.parametrize("which", ["dense", "sparse"])
def test_pair_parallel_and_particle_parallel_reverse_agree(dem, cuda, monkeypatch, which):
    """The reverse step in its two pair-parallel phases (the default: one
    thread per pair's law, then one per bound sphere gathering the shares)
    and in its particle-parallel form (DEM_B200_ADJ=pp: each sphere reverses
    all its pairs) compute the same adjoint with the additions in another
    order: objective equal, gradients within 1e-9 relative (plus 1e-12 of
    the objective for gradients near zero)."""
    w, pdis, angv = case(dem) if which == "dense" else sparse_case(dem)
    out = []
    for flag in ("pairs", "pp"):
        monkeypatch.setenv("DEM_B200_ADJ", flag)
        e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64, "cell": w.cell() + 0.01})
        e.set_material(w.pp, w.pw)
        e.upload(w.pos, w.rad, pdis, angv)
        out.append(e.adjoint(STEPS, EVERY, dem.OBJ_POTENTIAL))
        assert e.scalars()["status"] == 0
        e.close()
    a, b = out
    assert a["value"] == b["value"]
    floor = 1e-12 * abs(a["value"])
    for side in ("d_pp", "d_pw"):
        for k, x in a[side].items():
            assert abs(x - b[side][k]) <= 1e-9 * abs(x) + floor, (side, k, x, b[side][k])
    np.testing.assert_allclose(a["d_radii"], b["d_radii"], rtol=1e-9, atol=1e-12 * np.abs(a["d_radii"]).max())
