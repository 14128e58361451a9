"""The oracle's poured loop (orc_run_pour) on the CPU: the reference's layer
injection rule (dempacking.cu:379-381,459-461) and its edge cases."""
import numpy as np


def _case(dem, wl, **kw):
    w = wl.pour_box(**kw)
    cell = 2.0 * float(w.rad.max()) + w.skin + 1e-4
    return w, cell, dem.material_array(w.pp, w.pw)


def test_all_in_from_the_start_is_the_plain_loop(dem, orc, wl):
    w = wl.small_box(n=300)
    cell = w.cell()
    mat = dem.material_array(w.pp, w.pw)
    a = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, False, 120, w.relist_interval)
    b = orc.run_pour(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, False, 120, w.relist_interval,
                     nplayer=50, tnewpar=1e-9, n_active=w.n)
    np.testing.assert_array_equal(a["pos"], b["pos"])
    np.testing.assert_array_equal(a["list_ln"], b["list_ln"])
    assert (b["nact"] == w.n).all()


def test_insertion_steps_follow_the_rule(dem, orc, wl):
    w, cell, mat = _case(dem, wl)
    npl, tn = w.meta["nplayer"], w.meta["tnewpar"]
    o = orc.run_pour(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, False, 3100, w.relist_interval,
                     npl, tn, 0, pdis=w.meta["pdis"])
    assert o["status"] == 0
    # before step it (1-based) while dt*it > N*tnewpar/nplayer: N += nplayer
    expect, N = [], 0
    for s in range(3100):
        if N < w.n and w.dt * (s + 1) > float(np.float32(N)) * tn / float(np.float32(npl)):
            N = min(N + npl, w.n)
        expect.append(N)
    np.testing.assert_array_equal(o["nact"], expect)
    assert expect[0] == npl and expect[-1] == 3 * npl


def test_ragged_last_layer_and_waiting_particles(dem, orc, wl):
    w, cell, mat = _case(dem, wl, layers=2)
    npl = w.meta["nplayer"]
    ntot = npl + 10                         # the second layer is 10 particles
    pos, rad, pdis = w.pos[:3 * ntot], w.rad[:ntot], w.meta["pdis"][:3 * ntot]
    o = orc.run_pour(pos, rad, w.world, w.dt, w.skin, cell, w.density, mat, False, 1600, w.relist_interval,
                     npl, w.meta["tnewpar"], 0, pdis=pdis)
    assert o["status"] == 0
    assert o["nact"][1506] == npl and o["nact"][1507] == ntot
    o2 = orc.run_pour(pos, rad, w.world, w.dt, w.skin, cell, w.density, mat, False, 1000, w.relist_interval,
                      npl, w.meta["tnewpar"], 0, pdis=pdis)
    np.testing.assert_array_equal(o2["pos"][3 * npl:], pos[3 * npl:])      # not yet in: untouched
    np.testing.assert_array_equal(o2["pdis"][3 * npl:], pdis[3 * npl:])
