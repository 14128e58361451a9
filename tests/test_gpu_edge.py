"""Edge cases of the context API against the oracle: one and two spheres
(the smallest systems the engine takes), a sphere driven into a corner (two
walls at once: the wall-history slot goes to the deeper contact), an oblique
spinning collision of unequal spheres (tangential history, Coulomb limit,
rolling resistance), and spheres above the top of the box (open top: their
cell keys clamp into the top layer).  Each runs through contact and out of
it, across re-lists (every 20 steps), in both precisions; tolerances as in
the engine tests: FP64 positions RMS <= 1e-10 d, mixed <= 1e-6 d."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SKIN = 0.05


def _workload(wl, pos, rad, world, prec):
    pp, pw = wl.material(mu=0.3, roll_rel=0.002)
    rad = np.asarray(rad, dtype=np.float64)
    return wl.Workload("edge", rad.size, np.asarray(pos, dtype=np.float64), rad, world, wl.reduced_dt(5e-7), 0, 20,
                       SKIN, prec, pp, pw)


def _run_both(dem, orc, w, pdis, angv, steps, prec):
    e = dem.Engine(**{**w.engine_kwargs(), "precision": prec})
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad, pdis, angv)
    e.step(steps)
    s = e.scalars()
    pos, pd, av = e.download()
    cell = e.grid_info()[1]
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(w.pp, w.pw),
                prec == dem.PREC_MIXED, steps, w.relist_interval, pdis=pdis, angv=angv)
    e.close()
    assert s["status"] == 0 and o["status"] == 0
    tol = 1e-10 if prec == dem.PREC_FP64 else 1e-6
    assert np.sqrt(np.mean((pos - o["pos"]) ** 2)) <= tol
    # velocities (per-step displacement / dt) to the same relative tolerance
    assert np.max(np.abs(pd - o["pdis"])) / w.dt <= 1e3 * tol
    assert np.max(np.abs(av - o["angv"])) / w.dt <= 1e4 * tol
    return s, pos, pd / w.dt, av / w.dt, o


PRECS = [("fp64", 0), ("mixed", 1)]


@pytest.mark.parametrize("name,mixed", PRECS)
def test_single_sphere_bounces_off_the_floor(dem, orc, wl, cuda, name, mixed):
    """n = 1: falls 0.03 d onto the floor with spin, bounces (e = 0.5 map)
    and leaves the floor with friction-changed horizontal velocity."""
    prec = dem.PREC_MIXED if mixed else dem.PREC_FP64
    w = _workload(wl, [-0.9, 0.95, 0.53], [0.5], (3.0, 3.0, 10.0), prec)
    pdis = np.array([-0.3, 0.2, -1.0]) * w.dt
    angv = np.array([2.0, -1.0, 5.0]) * w.dt
    s, pos, v, _, _ = _run_both(dem, orc, w, pdis, angv, 1500, prec)
    assert pos[2] > 0.5 and 0.4 < v[2] < 0.55         # off the floor, rising at ~e x the impact speed
    assert abs(v[1] - 0.2) > 0.1                      # friction acted
    assert s["pairs"] == 0 and s["contacts"] == 0


@pytest.mark.parametrize("name,mixed", PRECS)
def test_sphere_into_a_corner_two_walls(dem, orc, wl, cuda, name, mixed):
    """Side wall and floor touched in the same steps (one history slot, owned
    by the deeper contact)."""
    prec = dem.PREC_MIXED if mixed else dem.PREC_FP64
    w = _workload(wl, [-0.98, 0.0, 0.52], [0.5], (3.0, 3.0, 10.0), prec)
    pdis = np.array([-1.0, 0.3, -1.0]) * w.dt
    angv = np.array([0.0, 3.0, 0.0]) * w.dt
    _, pos, v, av, _ = _run_both(dem, orc, w, pdis, angv, 1000, prec)
    assert v[0] > 0.2 and v[2] > 0.2                  # rebounded from both walls
    assert abs(av[1] - 3.0) > 1.0                     # the walls' friction changed the spin


@pytest.mark.parametrize("name,mixed", PRECS)
def test_head_on_pair_restitution(dem, orc, wl, cuda, name, mixed):
    """n = 2 in free fall, head on along x: one listed pair, one contact, and
    the rebound speed is e = 0.5 of the approach speed."""
    prec = dem.PREC_MIXED if mixed else dem.PREC_FP64
    w = _workload(wl, [-0.52, 0.0, 8.0, 0.52, 0.0, 8.0], [0.5, 0.5], (6.0, 6.0, 20.0), prec)
    pdis = np.array([1.0, 0.0, 0.0, -1.0, 0.0, 0.0]) * w.dt
    s, _, v, _, o = _run_both(dem, orc, w, pdis, np.zeros(6), 1500, prec)
    assert s["pairs"] == 1 and o["ncontacts"].max() == 1
    assert -v[0] / 1.0 == pytest.approx(0.5, abs=0.02) and v[3] == pytest.approx(-v[0], abs=1e-9)
    assert v[2] == pytest.approx(v[5])                # both still falling alike


@pytest.mark.parametrize("name,mixed", PRECS)
def test_oblique_spinning_pair_of_unequal_spheres(dem, orc, wl, cuda, name, mixed):
    """Unequal radii, an offset impact and spin about all axes: tangential
    history, the Coulomb limit and rolling resistance act in one contact."""
    prec = dem.PREC_MIXED if mixed else dem.PREC_FP64
    w = _workload(wl, [-0.47, 0.15, 8.0, 0.42, -0.1, 8.02], [0.5, 0.375], (6.0, 6.0, 20.0), prec)
    pdis = np.array([1.0, 0.0, 0.1, -0.8, 0.2, 0.0]) * w.dt
    angv = np.array([0.0, 0.0, 20.0, 5.0, -3.0, 0.0]) * w.dt
    _, _, v, av, o = _run_both(dem, orc, w, pdis, angv, 1500, prec)
    assert o["ncontacts"].max() == 1
    assert abs(av[2] - 20.0) > 0.5 and abs(av[5]) > 1.0   # torques from the contact
    assert v[0] < 0.5 and v[3] > 0.5                      # the pair separated


@pytest.mark.parametrize("name,mixed", PRECS)
def test_spheres_above_the_top_of_the_box(dem, orc, wl, cuda, name, mixed):
    """The box is open at the top: spheres above it hash into the top cell
    layer.  Cells and the pair set stay bit-exact, the pairs across the top
    and far above it are found, and the fall through the top matches."""
    prec = dem.PREC_MIXED if mixed else dem.PREC_FP64
    world = (6.0, 6.0, 5.0)
    pos = [0.0, 0.0, 4.8,    0.0, 0.0, 5.83,     # straddling the top: one pair
           1.0, 1.0, 9.0,    1.0, 1.0, 10.02,    # above the top: one pair
           1.0, 1.0, 30.0,                       # far above, same clamped cell
           -2.0, -2.0, 0.5]                      # on the floor
    w = _workload(wl, pos, [0.5] * 6, world, prec)
    e = dem.Engine(**{**w.engine_kwargs(), "precision": prec})
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    e.step(1)
    grid, cell, _ = e.grid_info()
    keys, ids, st, en = e.cells()
    fp32 = prec == dem.PREC_MIXED
    g = orc.grid(w.world, cell)
    sk, si, cs, ce = orc.sort_cells(orc.hash_keys(w.pos, w.world, cell, fp32), int(g.prod()))
    assert tuple(g) == tuple(grid)
    np.testing.assert_array_equal(keys, sk)
    np.testing.assert_array_equal(ids, si)
    np.testing.assert_array_equal(st, cs)
    np.testing.assert_array_equal(en, ce)
    top = (int(g[2]) - 1) * int(g[0]) * int(g[1])
    assert (keys[np.isin(ids, [1, 2, 3, 4])] >= top).all()
    lp, ln, _ = e.pairs()
    assert list(zip(lp.tolist(), ln.tolist())) == [(0, 1), (2, 3)]
    e.close()
    _run_both(dem, orc, w, None, None, 600, prec)
