"""Host utilities of the library, on the CPU: the deck reader and its
reduced-unit constants (dempacking.cu:107-149,213-225), the material it
yields, the restitution map, the seeded initial-state generators and the
reference output files (dempacking.cu:227-234,772-776,785-791,802,812-820,
904-913).  No GPU is touched."""
import ctypes
import math

import numpy as np
import pytest

# An input deck in the positional layout the reference reads (twelve numeric
# lines): force mode; E, nu, rho; diameter; total particles; dt, steps;
# dmt1, dmt2, thickness; two bed heights; injection velocity, rings;
# sliding friction p/w; four damping coefficients and global damping; three
# spring/damping constants; rolling friction p/w.  Values are this test's own.
DECK = """1
2.0e7 0.25 2600.0
0.002
12345
2.0e-6 50000
0.03 0.04 0.05
0.06 0.01
0.5 3
0.4 0.35
0.2 0.25 0.22 0.21 0.0
1.0 0.0 0.0
0.00004 0.00006
"""


@pytest.fixture()
def deck(dem, tmp_path):
    p = tmp_path / "deck.inp"
    p.write_text(DECK)
    return dem.read_deck(p)


def test_deck_fields_and_reduced_units(dem, deck):
    assert deck.iforcemode == 1 and deck.ntot == 12345 and deck.tstop == 50000 and deck.nrings == 3
    assert deck.emod == 2.0e7 and deck.vpois == 0.25 and deck.denp == 2600.0 and deck.diam == 0.002
    assert (deck.dt, deck.dmt1, deck.dmt2, deck.thick) == (2.0e-6, 0.03, 0.04, 0.05)
    assert (deck.ufricp, deck.ufricw, deck.upp, deck.upw) == (0.4, 0.35, 0.00004, 0.00006)
    # constants as the reference writes them (3.14159265, 1.33333333)
    emod = 6.0 * 2.0e7 / (3.14159265 * 2600.0 * 9.81 * 0.002)
    assert deck.emod_red == pytest.approx(emod, rel=1e-15)
    assert deck.estarp == pytest.approx(1.33333333 * emod / (2.0 * (1.0 - 0.25 ** 2)), rel=1e-15)
    assert deck.estarw == pytest.approx(1.33333333 / (2.0 * (1.0 - 0.25 ** 2) / emod), rel=1e-15)
    assert list(deck.world) == pytest.approx([0.04 / 0.002, 0.05 / 0.002, (0.06 + 0.01) / 0.002])
    assert deck.upp_red == pytest.approx(0.02) and deck.upw_red == pytest.approx(0.03)


def test_deck_material_blocks(dem, deck):
    pp, pw = dem.deck_material(deck)
    assert pp["estar"] == deck.estarp and pw["estar"] == deck.estarw
    assert (pp["mu"], pw["mu"]) == (0.4, 0.35)
    assert (pp["damp_n"], pp["damp_t"], pw["damp_n"], pw["damp_t"]) == (0.2, 0.25, 0.22, 0.21)
    assert (pp["roll"], pw["roll"]) == (deck.upp_red, deck.upw_red)
    assert pp["nu"] == pw["nu"] == 0.25


def test_deck_errors(dem, tmp_path):
    with pytest.raises(dem.DemError) as e:
        dem.read_deck(tmp_path / "missing.inp")
    assert e.value.code == dem.DEM_ERR_IO
    bad = tmp_path / "bad.inp"
    bad.write_text("1\n2.0e7 0.25\n")
    with pytest.raises(dem.DemError) as e:
        dem.read_deck(bad)
    assert e.value.code == dem.DEM_ERR_IO
    neg = tmp_path / "neg.inp"
    neg.write_text(DECK.replace("0.002\n", "-0.002\n", 1))
    with pytest.raises(dem.DemError) as e:
        dem.read_deck(neg)
    assert e.value.code == dem.DEM_ERR_IO


def test_reduced_modulus_and_restitution_map(dem):
    E, nu, rho, d = 1e7, 0.3, 2500.0, 1e-3
    er = 6 * E / (math.pi * rho * 9.81 * d)
    assert dem.reduced_modulus(E, rho, d) == pytest.approx(er, rel=1e-15)
    assert dem.estar(E, nu, rho, d) == pytest.approx(4 / 3 * er / (2 * (1 - nu * nu)), rel=1e-15)
    # c = -2 sqrt(5/18) ln e / sqrt(ln^2 e + pi^2); e = 0.5 -> 0.2271
    c = dem.damp_from_restitution(0.5)
    le = math.log(0.5)
    assert c == pytest.approx(-2 * math.sqrt(5 / 18) * le / math.sqrt(le * le + math.pi ** 2), rel=1e-15)
    assert c == pytest.approx(0.2271, abs=1e-4)
    assert dem.damp_from_restitution(1.0) == 0.0 and dem.damp_from_restitution(0.0) == 0.0
    assert dem.damp_from_restitution(0.1) > dem.damp_from_restitution(0.9) > 0.0


def test_radius_generators(dem):
    n = 20000
    mono = dem.gen_radii(n, 0, 0.5, seed=1)
    assert np.all(mono == 0.5)
    ln = dem.gen_radii(n, 1, 0.5, 0.1, 0.4, 0.65, seed=2)
    assert ln.min() >= 0.4 and ln.max() <= 0.65
    assert np.median(ln) == pytest.approx(0.5, rel=0.02)
    np.testing.assert_array_equal(ln, dem.gen_radii(n, 1, 0.5, 0.1, 0.4, 0.65, seed=2))   # seeded
    assert not np.array_equal(ln, dem.gen_radii(n, 1, 0.5, 0.1, 0.4, 0.65, seed=3))
    # radii are FP32-representable (the mixed form then sees the same radii)
    assert np.all(ln == ln.astype(np.float32).astype(np.float64))
    bi = dem.gen_radii(n, 2, 0.3, 0.6, seed=4)
    a, b = float(np.float32(0.3)), float(np.float32(0.6))
    assert set(np.unique(bi).tolist()) == {a, b}
    assert np.count_nonzero(bi == a) == n // 2
    assert not np.all(bi[: n // 2] == a)   # shuffled


def test_lattice_generator(dem):
    n, a, nx, ny, z0, jit, r = 2000, 1.0, 20, 20, 0.6, 0.05, 0.5
    pos, rad = dem.gen_lattice(n, a, nx, ny, z0, jit, r, 7)
    p = pos.reshape(-1, 3)
    assert np.all(rad == r)
    layer = np.arange(n) // (nx * ny)
    # layers a apart from z0, positions within +-jitter of the lattice sites
    assert np.all(np.abs(p[:, 2] - (z0 + layer * a)) <= jit + 1e-12)
    gx = (np.arange(n) % nx - 0.5 * (nx - 1)) * a
    gy = ((np.arange(n) // nx) % ny - 0.5 * (ny - 1)) * a
    assert np.all(np.abs(p[:, 0] - gx) <= jit + 1e-12) and np.all(np.abs(p[:, 1] - gy) <= jit + 1e-12)
    p2, _ = dem.gen_lattice(n, a, nx, ny, z0, jit, r, 7)
    np.testing.assert_array_equal(pos, p2)


def test_rsa_generator_places_without_overlap(dem):
    world = (12.0, 12.0, 30.0)
    rad = dem.gen_radii(1500, 1, 0.5, 0.1, 0.4, 0.65, seed=5)
    pos = dem.gen_rsa(world, rad, 11)
    p = pos.reshape(-1, 3)
    d = np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1))
    s = rad[:, None] + rad[None, :]
    iu = np.triu_indices(rad.size, 1)
    assert np.all(d[iu] >= s[iu])
    hx, hy = world[0] / 2, world[1] / 2
    assert np.all(p[:, 0] - rad >= -hx) and np.all(p[:, 0] + rad <= hx)
    assert np.all(p[:, 1] - rad >= -hy) and np.all(p[:, 1] + rad <= hy)
    assert np.all(p[:, 2] - rad >= 0.0) and np.all(p[:, 2] + rad <= world[2])
    np.testing.assert_array_equal(pos, dem.gen_rsa(world, rad, 11))
    with pytest.raises(dem.DemError) as e:   # far more volume than the box holds
        dem.gen_rsa((4.0, 4.0, 4.0), np.full(500, 0.5), 1)
    assert e.value.code == dem.DEM_ERR_ARG


def test_output_files(dem, deck, tmp_path):
    L = dem.lib()
    v = tmp_path / "view.dat"
    assert L.dem_write_view(str(v).encode(), ctypes.byref(deck)) == 0
    lines = v.read_text().splitlines()
    assert lines[0] == "number of particles=12345" and lines[1] == "diameters = 0.002"
    assert "time step=0.000002" in lines[2] and "bed width=15.000" in lines[2]
    ppor = tmp_path / "ppor.dat"
    for it in (1000, 2000):
        assert L.dem_write_ppor(str(ppor).encode(), it, 500, 900, 0.42, 0.58, 1.8, 12.5) == 0
    rows = [r.split() for r in ppor.read_text().splitlines()]
    assert rows == [[str(it), "500", "450", "0.420000", "0.580000", "1.800000", "12.500000"] for it in (1000, 2000)]
    pos = np.array([0.1, 0.2, 0.3, 1.0, 2.0, 3.0])
    rad = np.array([0.5, 0.25])
    pt = tmp_path / "particle.dat"
    assert L.dem_write_particles(str(pt).encode(), 7, 2, dem._ptr(pos), dem._ptr(rad), 0.002) == 0
    lines = pt.read_text().splitlines()
    assert lines[0] == 'ZONE T="ZONE007"'
    np.testing.assert_allclose([float(x) for x in lines[2].split()], [0.002, 0.004, 0.006, 0.0005, 1])
    pre = tmp_path / "preflow.dat"
    pdis = np.array([1e-6, 2e-6, 3e-6, 4e-6, 5e-6, 6e-6])
    angv = np.zeros(6)
    assert L.dem_write_preflow(str(pre).encode(), 3000, 2, 42, dem._ptr(pos), dem._ptr(pdis), dem._ptr(angv)) == 0
    lines = pre.read_text().splitlines()
    assert [int(x) for x in lines[0].split(",")] == [3000, 2, 42]
    assert [float(x) for x in lines[2].split()][:3] == [1.0, 2.0, 3.0]
    ts = tmp_path / "timesteps.dat"
    assert L.dem_write_timesteps(str(ts).encode(), 0.25, 1000) == 0
    assert ts.read_text().split() == ["0.250000", "1000.000000"]
    jf, rs = tmp_path / "jobfinished", tmp_path / "restart.dat"
    assert L.dem_write_finish(str(jf).encode(), str(rs).encode()) == 0
    assert jf.read_text() == "job finished\n"
    assert rs.read_text().splitlines() == ["program comes to end!", "       1        1"]
    assert L.dem_write_ppor(str(tmp_path / "no" / "dir" / "x.dat").encode(), 1, 1, 0, 0.0, 0.0, 0.0, 0.0) \
        == dem.DEM_ERR_IO


def test_preflow_reader_round_trip(dem, tmp_path):
    rng = np.random.default_rng(4)
    n = 50
    pos, pdis, angv = rng.uniform(-5, 5, 3 * n), rng.normal(0, 1e-3, 3 * n), rng.normal(0, 1e-3, 3 * n)
    pre = tmp_path / "preflow.dat"
    assert dem.lib().dem_write_preflow(str(pre).encode(), 7000, n, 5, dem._ptr(pos), dem._ptr(pdis),
                                       dem._ptr(angv)) == 0
    it, itime, p2, d2, a2 = dem.read_preflow(pre)
    assert (it, itime, p2.size) == (7000, 5, 3 * n)
    # the file keeps 6 decimals
    np.testing.assert_allclose(p2, pos, rtol=0, atol=5e-7)
    np.testing.assert_allclose(d2, pdis, rtol=0, atol=5e-7)
    np.testing.assert_allclose(a2, angv, rtol=0, atol=5e-7)
    small = np.empty(3)
    c = ctypes.c_longlong
    rc = dem.lib().dem_read_preflow(str(pre).encode(), ctypes.byref(c()), ctypes.byref(c()), ctypes.byref(c()),
                                    dem._ptr(small), dem._ptr(small), dem._ptr(small), 1)
    assert rc == dem.DEM_ERR_ARG
    bad = tmp_path / "bad.dat"
    bad.write_text("7000, 2, 5\n1 2 3 4 5 6 7 8 9\n1 2 3\n")
    with pytest.raises(dem.DemError) as e:
        dem.read_preflow(bad)
    assert e.value.code == dem.DEM_ERR_IO


def test_host_only_generators_match_and_leave_the_gpu_library_unloaded(dem, tmp_path):
    """The workloads generate their initial states with libdem_gen.so (the
    generators' source built host only): bit for bit the library's own
    generators, and a process that only generates a workload (the CPU timing
    of the reference step) never maps libdem_b200.so."""
    import subprocess
    import sys
    from dem_b200 import gen
    rad_g = gen.gen_radii(5000, dem.RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed=11)
    np.testing.assert_array_equal(rad_g, dem.gen_radii(5000, dem.RADII_LOGNORMAL, 0.5, 0.2, 0.3, 0.8, seed=11))
    np.testing.assert_array_equal(gen.gen_rsa((30.0, 30.0, 30.0), rad_g, 12),
                                  dem.gen_rsa((30.0, 30.0, 30.0), rad_g, 12))
    assert gen.estar(1e7, 0.29, 2500.0, 1e-3) == dem.estar(1e7, 0.29, 2500.0, 1e-3)
    code = ("import sys, pathlib; sys.path.insert(0, 'tests'); from _load import load_pkg; dem = load_pkg(); "
            "import dem_b200.workloads as wl; w = wl.rsa_500k(n=3000, box=(30.0, 30.0, 60.0)); "
            "maps = pathlib.Path('/proc/self/maps').read_text(); "
            "print('gpu-lib' if 'libdem_b200.so' in maps else 'host-only', dem._LIB is None)")
    root = __import__("pathlib").Path(__file__).resolve().parents[1]
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, check=True).stdout
    assert out.split() == ["host-only", "True"], out
