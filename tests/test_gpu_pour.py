"""Poured packing on the device (dem_set_pour): layers of particles join the
system at the reference's injection times (dempacking.cu:375-461) inside
buffers sized once, checked against the oracle's poured loop, across the
windows an insertion cuts short, in both force modes and precisions, and
through a checkpoint taken in the middle of the pour."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 3600          # pour_box: layers join at steps 0, 1507 and 3014


def _engine(dem, w, prec, mode):
    e = dem.Engine(**{**w.engine_kwargs(), "precision": prec, "force_mode": mode})
    e.set_material(w.pp, w.pw)
    return e


def _poured(dem, w, prec, mode):
    e = _engine(dem, w, prec, mode)
    e.upload(w.pos, w.rad, w.meta["pdis"], None)
    e.set_pour(w.meta["nplayer"], w.meta["tnewpar"], 0)
    return e


def _relists_expected(nact, interval):
    """Re-lists of a run whose active count per step is nact: a window starts
    at step 0, after every interval steps, and at every insertion."""
    count, win = 0, 0
    for s in range(len(nact)):
        if s > 0 and nact[s] != nact[s - 1]:
            win = 0
        if win == 0:
            count += 1
        win = (win + 1) % interval
    return count


@pytest.mark.parametrize("prec,mode", [("fp64", "pccp"), ("fp64", "pp"), ("mixed", "pccp"), ("mixed", "pp")])
def test_pour_matches_oracle(dem, orc, wl, cuda, prec, mode):
    w = wl.pour_box()
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    m = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    e = _poured(dem, w, p, m)
    assert e.active_count() == 0
    e.step(STEPS)
    s = e.scalars()
    pos, pd, _ = e.download()
    cell = e.grid_info()[1]
    mat = dem.material_array(w.pp, w.pw)
    o = orc.run_pour(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, prec == "mixed", STEPS,
                     w.relist_interval, w.meta["nplayer"], w.meta["tnewpar"], 0, pdis=w.meta["pdis"])
    assert o["status"] == 0 and s["status"] == 0
    assert [0] + (np.nonzero(np.diff(o["nact"]))[0] + 1).tolist() == [0, 1507, 3014]
    assert e.active_count() == int(o["nact"][-1]) == w.n
    assert s["relists"] == _relists_expected(o["nact"], w.relist_interval)
    rms = np.sqrt(np.mean((pos - o["pos"]) ** 2))
    assert rms <= (1e-10 if prec == "fp64" else 1e-6), rms
    assert s["pairs"] == int(o["npairs"][-1])
    if prec == "fp64":
        assert s["contacts"] == int(o["ncontacts"][-1])
        np.testing.assert_array_equal(e.pairs()[1], o["list_ln"])
    assert o["ncontacts"].max() >= 5                # the layers met
    assert abs(s["maxhz"] - o["maxhz"][-1]) < 1e-6
    vol = np.sum(4.0 / 3.0 * np.pi * w.rad ** 3)
    assert s["packing_fraction"] == pytest.approx(vol / (w.world[0] * w.world[1] * s["maxhz"]), rel=1e-6)


def test_pour_state_before_and_between_layers(dem, wl, cuda):
    w = wl.pour_box()
    npl = w.meta["nplayer"]
    e = _poured(dem, w, dem.PREC_FP64, dem.FORCE_PCCP)
    pos, pd, _ = e.download()                    # not yet in: the injection states
    np.testing.assert_array_equal(pos, w.pos)
    np.testing.assert_array_equal(pd, w.meta["pdis"])
    e.step(1)
    assert e.active_count() == npl
    e.step(1506)
    assert e.active_count() == npl
    pos, pd, _ = e.download()
    np.testing.assert_array_equal(pos[3 * npl:], w.pos[3 * npl:])            # still waiting
    np.testing.assert_array_equal(pd[3 * npl:], w.meta["pdis"][3 * npl:])
    assert np.all(pos[2:3 * npl:3] < w.pos[2])                                 # the first layer fell
    s = e.scalars()
    vol = np.sum(4.0 / 3.0 * np.pi * w.rad[:npl] ** 3)
    assert s["packing_fraction"] == pytest.approx(vol / (w.world[0] * w.world[1] * s["maxhz"]), rel=1e-12)
    assert s["mean_cn"] == pytest.approx(2.0 * s["contacts"] / npl)
    lp, ln, _ = e.pairs()
    assert lp.size == 0 or ln.max() < npl
    e.step(1)                                    # step 1507: the second layer
    assert e.active_count() == 2 * npl
    pos, _, _ = e.download()
    np.testing.assert_array_equal(pos[3 * 2 * npl:], w.pos[3 * 2 * npl:])
    assert np.all(pos[3 * npl + 2:3 * 2 * npl:3] < w.pos[2])                  # moved one step


@pytest.mark.parametrize("mode", ["pccp", "pp"])
def test_pour_resume_is_bit_exact(dem, wl, cuda, tmp_path, mode):
    w = wl.pour_box()
    m = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    a = _poured(dem, w, dem.PREC_MIXED, m)
    a.step(1527)                                 # layers at 0 and 1507; window 1507..1526 complete
    assert a.active_count() == 2 * w.meta["nplayer"]
    a.save_state(tmp_path / "pour.bin")
    a.step(1600)                                 # the third layer at 3014
    b = _engine(dem, w, dem.PREC_MIXED, m)
    b.load_state(tmp_path / "pour.bin")
    assert b.active_count() == 2 * w.meta["nplayer"] and b.scalars()["step"] == 1527
    b.step(1600)
    sa, sb = a.scalars(), b.scalars()
    assert sa["status"] == sb["status"] == 0
    assert a.active_count() == b.active_count() == w.n
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)
    for k in ("step", "relists", "pairs", "contacts", "maxhz", "packing_fraction"):
        assert sa[k] == sb[k], k


@pytest.mark.parametrize("mode", ["pccp", "pp"])
def test_pour_window_kernel_equals_per_step_kernels(dem, wl, cuda, monkeypatch, mode):
    w = wl.pour_box()
    m = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("DEM_B200_WINDOW", flag)
        e = _poured(dem, w, dem.PREC_MIXED, m)
        e.step(1700)
        out.append((e.download(), e.scalars()))
    for x, y in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(x, y)
    assert out[0][1]["pairs"] == out[1][1]["pairs"]


def test_full_pour_equals_plain_run(dem, wl, cuda):
    """Every particle in from the start: no insertion ever, the same run."""
    w = wl.small_box(n=2000)
    a = _engine(dem, w, dem.PREC_MIXED, dem.FORCE_PCCP)
    a.upload(w.pos, w.rad)
    a.step(87)
    b = _engine(dem, w, dem.PREC_MIXED, dem.FORCE_PCCP)
    b.upload(w.pos, w.rad)
    b.set_pour(100, 1e-9, w.n)
    b.step(87)
    assert b.active_count() == w.n
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)


def test_pour_errors(dem, wl, cuda):
    w = wl.pour_box()
    npl, tn = w.meta["nplayer"], w.meta["tnewpar"]
    e = _engine(dem, w, dem.PREC_MIXED, dem.FORCE_PCCP)
    with pytest.raises(dem.DemError) as x:                 # nothing uploaded
        e.set_pour(npl, tn, 0)
    assert x.value.code == dem.DEM_ERR_STATE
    e.upload(w.pos, w.rad, w.meta["pdis"], None)
    for args in ((0, tn, 0), (npl, 0.0, 0), (npl, tn, -1), (npl, tn, w.n + 1)):
        with pytest.raises(dem.DemError) as x:
            e.set_pour(*args)
        assert x.value.code == dem.DEM_ERR_ARG
    e.set_pour(npl, tn, 0)
    with pytest.raises(dem.DemError) as x:                 # already pouring
        e.set_pour(npl, tn, 0)
    assert x.value.code == dem.DEM_ERR_STATE
    e.step(w.relist_interval)
    with pytest.raises(dem.DemError) as x:                 # layers still to come
        e.adjoint(w.relist_interval, w.relist_interval, dem.OBJ_PACKING)
    assert x.value.code == dem.DEM_ERR_STATE
    e.upload(w.pos, w.rad, w.meta["pdis"], None)          # an upload ends the pour
    assert e.active_count() == w.n


DECK = """1
10000000 0.29 2500.0
0.01
500
0.001 3000
0.1 0.1 0.1
0.0 0.2
4.0 9
0.40 0.40
0.3 0.3 0.3 0.3 0.30
10000.0 100.0 100.0
0.000 0.000
"""


def test_deck_driver_pours_layers(dem, cuda, tmp_path):
    """The deck driver pours as the reference does: a 10x10 (reduced) box
    gives 7x7 injection sites, layers join at it = 1, 501, 1001, ... (time >
    N*0.5/49), so ppor.dat reports 98, 196 and 294 particles at steps 1000,
    2000 and 3000."""
    import pathlib
    import subprocess
    exe = pathlib.Path(dem.__file__).resolve().parent / "dempacking"
    (tmp_path / "hopp3d.inp").write_text(DECK)
    r = subprocess.run([str(exe), "hopp3d.inp"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [line.split() for line in (tmp_path / "ppor.dat").read_text().splitlines() if line.strip()]
    assert [(int(a[0]), int(a[1])) for a in rows] == [(1000, 98), (2000, 196), (3000, 294)]
    assert all(0.0 <= float(a[4]) < 1.0 for a in rows)
    assert (tmp_path / "particle.dat").exists() and (tmp_path / "jobfinished").exists()


def _driver_injection(deck, seed=20261203):
    """The deck driver's injection states (driver/dempacking.cpp, after
    dempacking.cu:243-309): ntot spheres of radius 0.5 on the deck's
    (W-3) x (T-3) injection lattice at hopzt - 5, speed vel0 at elevation
    pi (u/3 + 1/3) below the horizontal and a uniform azimuth, u from
    SplitMix64 seeded with `seed`; the same libm sin/cos as the driver."""
    import math
    n = deck.ntot
    W, T, H = deck.world[0], deck.world[1], deck.world[2]
    nx, ny = int(W) - 3, int(T) - 3
    if not (0.5 * W > 1.99) or nx < 1 or ny < 1:
        nx = ny = 1
    ax, ay = W / nx, T / ny
    mask = (1 << 64) - 1
    state = [seed]

    def urand():
        state[0] = (state[0] + 0x9E3779B97F4A7C15) & mask
        z = state[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        return float(z >> 11) * (1.0 / 9007199254740992.0)

    pi = 4.0 * math.atan(1.0)
    pos = np.zeros((n, 3))
    pdis = np.zeros((n, 3))
    nplayer = nx * ny
    for i in range(n):
        site = i % nplayer
        ix, iy = site // ny, site % ny
        pos[i, 0] = (ix + 0.5) * ax - 0.5 * W if nx > 1 else 0.0
        pos[i, 1] = (iy + 0.5) * ay - 0.5 * T if ny > 1 else 0.0
        pos[i, 2] = H - 5.0
        ang = pi * (urand() * .33333 + .33333)
        pdis[i, 2] = -deck.vel0 * math.sin(ang) * deck.dt
        dxy = -deck.vel0 * math.cos(ang) * deck.dt
        ang = 2.0 * pi * urand()
        pdis[i, 0] = dxy * math.cos(ang)
        pdis[i, 1] = dxy * math.sin(ang)
    return pos.reshape(-1), pdis.reshape(-1), nplayer, (W, T, H)


def _ppor_rows(path):
    return [[float(x) for x in line.split()] for line in path.read_text().splitlines() if line.strip()]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_shipped_deck_through_the_driver_against_the_oracle(dem, orc, cuda, tmp_path, prec):
    """The reference's own deck (hopp3d.inp: 10,000 spheres of 1 cm poured
    in layers of 2,209 into a 50 x 50 (reduced) box from 55 diameters up,
    40,000 steps) through the deck driver, its ppor.dat rows (particles in
    the system, contacts, packing fraction, mean coordination number, max
    height, every 1,000 steps) against the oracle's poured loop from the same
    injection states.  The particle counts agree on every row.  While the
    layers fall and first land the rows agree exactly: FP64 through step
    8,000 (contacts equal, the written values to their 6 decimals), mixed
    through step 6,000 (contacts equal); then the pile's formation is chaotic
    and the two runs part particle by particle, so the settled bed is
    compared by its statistics: final mean coordination number within 1 % of
    the oracle's, final packing fraction (the reference's max-height form)
    within 6 %."""
    import pathlib
    import shutil
    import subprocess
    src = pathlib.Path(__file__).resolve().parent / "golden" / "hopp3d.inp"
    shutil.copy(src, tmp_path / "hopp3d.inp")
    deck = dem.read_deck(str(src))
    exe = pathlib.Path(dem.__file__).resolve().parent / "dempacking"
    r = subprocess.run([str(exe), "hopp3d.inp", "--precision", prec], cwd=tmp_path, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = _ppor_rows(tmp_path / "ppor.dat")
    assert [int(a[0]) for a in rows] == list(range(1000, deck.tstop + 1, 1000))
    pos, pdis, nplayer, world = _driver_injection(deck)
    rad = np.full(deck.ntot, 0.5)
    pp, pw = dem.deck_material(deck)
    o = orc.run_pour(pos, rad, world, deck.dt, 0.55, 1.55, 1.0, dem.material_array(pp, pw), prec == "mixed",
                     deck.tstop, 20, nplayer, 0.5, 0, pdis=pdis)
    assert o["status"] == 0
    exact_until = 8000 if prec == "fp64" else 6000
    for a in rows:
        it = int(a[0])
        na = int(o["nact"][it - 1])
        contacts = int(o["ncontacts"][it - 1])
        mz = float(o["maxhz"][it - 1])
        phi = na * (np.pi / 6.0) / (world[0] * world[1] * mz)
        cn = 2.0 * contacts / na
        assert int(a[1]) == na, (it, a[1], na)
        if it <= exact_until:
            assert int(a[2]) == contacts, (it, a[2], contacts)
            if prec == "fp64":
                assert abs(a[4] - phi) <= 2e-6 and abs(a[5] - cn) <= 2e-6 and abs(a[6] - mz) <= 2e-6, (it, a, phi)
    last = rows[-1]
    na = int(o["nact"][-1])
    phi_end = na * (np.pi / 6.0) / (world[0] * world[1] * float(o["maxhz"][-1]))
    cn_end = 2.0 * float(o["ncontacts"][-1]) / na
    print(f"\nshipped deck {prec}: final phi {last[4]:.6f} (oracle {phi_end:.6f}), CN {last[5]:.4f} "
          f"(oracle {cn_end:.4f}), max height {last[6]:.4f} (oracle {o['maxhz'][-1]:.4f})")
    assert int(last[1]) == deck.ntot
    assert abs(last[5] - cn_end) <= 0.01 * cn_end
    assert abs(last[4] - phi_end) <= 0.06 * phi_end
