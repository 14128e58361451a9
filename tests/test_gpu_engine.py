"""GPU parity of the context API (SoA engine) against the CPU oracle.

Bit-exact: sorted cell keys / ids, cell ranges and the canonical candidate
pair set, for the FP64 list and the FP32 (mixed) list.
Tolerances (stated per result):
  FP64 engine vs FP64 oracle   forces rel-L2 <= 1e-9, positions RMS <= 1e-9 d
  mixed engine vs FP64 oracle  forces rel-L2 <= 2e-4 (max-abs <= 2e-3 of the
                               largest), positions RMS <= 1e-5 d after the run,
                               packing fraction |delta| <= 1e-3 (the target),
                               mean coordination number |delta| <= 0.02
"""
import numpy as np
import pytest

from _cases import dense_lattice

pytestmark = pytest.mark.gpu


def make_engine(dem, w, precision=None, **over):
    kw = w.engine_kwargs()
    if precision is not None:
        kw["precision"] = precision
    kw.update(over)
    e = dem.Engine(**kw)
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    return e


def oracle_cells(orc, w, cell, fp32):
    g = orc.grid(w.world, cell)
    keys = orc.hash_keys(w.pos, w.world, cell, fp32)
    sk, si, cs, ce = orc.sort_cells(keys, int(g.prod()))
    return g, sk, si, cs, ce


def case_workload(dem, wl, case):
    if case == "lattice":
        return wl.lattice_2k()
    if case == "small":
        return wl.small_box(n=4000, compress=0.62)
    return dense_lattice(dem)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["lattice", "small", "dense"])
def test_cells_and_pairs_bit_exact(dem, orc, wl, cuda, prec, case):
    w = case_workload(dem, wl, case)
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    fp32 = prec == "mixed"
    e = make_engine(dem, w, p)
    e.step(1)
    grid, cell, nc = e.grid_info()
    assert abs(cell - w.cell()) < 1e-15
    keys, ids, st, en = e.cells()
    g, sk, si, cs, ce = oracle_cells(orc, w, cell, fp32)
    assert tuple(g) == tuple(grid)
    np.testing.assert_array_equal(keys, sk)
    np.testing.assert_array_equal(ids, si)
    np.testing.assert_array_equal(st, cs)
    np.testing.assert_array_equal(en, ce)
    lp, ln, hist = e.pairs()
    off, oln, ohist, _ = orc.build_list(w.pos, w.rad, w.world, cell, w.skin, fp32)
    olp = np.repeat(np.arange(w.n, dtype=np.uint32), np.diff(off))
    np.testing.assert_array_equal(lp, olp)
    np.testing.assert_array_equal(ln, oln)
    assert lp.size > 0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_lists_from_the_outer_list_equal_fresh_lists(dem, orc, wl, cuda, prec):
    """The re-list filters an outer candidate list (built at skin + ext,
    ext = min(skin, r_max / 10), and rebuilt once a particle has moved 0.4
    ext): after hundreds of
    windows of falling, colliding spheres -- many rebuilds and many windows
    between them -- each window's list equals the oracle's fresh cell-walk
    list at the positions of its re-list, bit for bit."""
    w = wl.lattice_2k()
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    e = make_engine(dem, w, p)
    cell = e.grid_info()[1]
    K = w.relist_interval
    for m, windows in enumerate((1, 60, 200, 37, 400)):
        e.step(windows * K)
        pos = e.download()[0]
        e.step(1)   # the re-list at these positions
        lp, ln, _ = e.pairs()
        off, oln, _, _ = orc.build_list(pos, w.rad, w.world, cell, w.skin, prec == "mixed")
        olp = np.repeat(np.arange(w.n, dtype=np.uint32), np.diff(off))
        np.testing.assert_array_equal(lp, olp)
        np.testing.assert_array_equal(ln, oln)
        assert e.scalars()["status"] == 0
        e.step(K - 1)
    assert lp.size > 1000   # a bed with contacts by the end
    e.close()


@pytest.mark.parametrize("mode", ["pccp", "pp"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_relist_deterministic_and_bound_count(dem, wl, cuda, prec, mode):
    """The re-list's single-pass scans (tiles that start in any order add up
    the totals their predecessors publish), the fill and the component pass
    over the bound list, and the lock-free unions give the same lists,
    batches and states in two contexts, bit for bit, on a sparse bed
    (cluster batches) and a dense lattice; the bound count (the bound scan's
    total) equals the particles that have a listed pair or lie within
    r + skin/2 of a wall at the re-list's positions."""
    from _cases import dense_lattice
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    fm = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    for w in (wl.small_box(n=3000), dense_lattice(dem, nx=10, ny=10, nz=8)):
        rng = np.random.default_rng(11)
        pdis = rng.normal(0, 2e-6, 3 * w.n)
        a = make_engine(dem, w, p, force_mode=fm)
        a.upload(w.pos, w.rad, pdis, None)
        b = make_engine(dem, w, p, force_mode=fm)
        b.upload(w.pos, w.rad, pdis, None)
        for steps in (4 * w.relist_interval, 3):
            a.step(steps)
            b.step(steps)
            assert a.window_work() == b.window_work()
            for x, y in zip(a.download(), b.download()):
                np.testing.assert_array_equal(x, y)
            for x, y in zip(a.pairs(), b.pairs()):
                np.testing.assert_array_equal(x, y)
        sa, sb = a.scalars(), b.scalars()
        assert sa["status"] == 0 and sb["status"] == 0
        assert sa["maxhz"] == sb["maxhz"] and sa["contacts"] == sb["contacts"] and sa["pairs"] == sb["pairs"]
        # the bound count at a re-list
        K = w.relist_interval
        a.step(K - 3)                     # to the window's end
        pos = a.download()[0].reshape(-1, 3)
        a.step(1)                         # the re-list at these positions
        lp, ln, _ = a.pairs()
        r = w.rad.astype(np.float32).astype(np.float64) if prec == "mixed" else w.rad
        mg = r + 0.5 * w.skin
        hx, hy = 0.5 * w.world[0], 0.5 * w.world[1]
        near = ((pos[:, 2] < mg) | (pos[:, 0] + hx < mg) | (hx - pos[:, 0] < mg) | (pos[:, 1] + hy < mg)
                | (hy - pos[:, 1] < mg))
        bound = near.copy()
        bound[lp] = True
        bound[ln] = True
        work = a.window_work()
        assert work["bound"] == int(bound.sum())
        assert work["wall_candidates"] == int(near.sum())
        assert work["pairs"] == lp.size
        a.close()
        b.close()


@pytest.mark.parametrize("case", ["small", "dense"])
@pytest.mark.parametrize("prec,rtol", [("fp64", 1e-9), ("mixed", 2e-4)])
def test_first_step_forces(dem, orc, wl, cuda, prec, rtol, case):
    """Forces of step 1 on overlapping polydisperse packings (strongly
    compressed RSA; gently overlapping lattice)."""
    w = case_workload(dem, wl, case)
    rng = np.random.default_rng(3)
    pdis = rng.normal(0, 1e-6, 3 * w.n)
    angv = rng.normal(0, 1e-6, 3 * w.n)
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    e = dem.Engine(**{**w.engine_kwargs(), "precision": p})
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad, pdis, angv)
    e.record_forces(True)
    e.step(1)
    F, T, C = e.forces()
    cell = e.grid_info()[1]
    mat = dem.material_array(w.pp, w.pw)
    oF, oT, oC, npairs = orc.forces_once(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, prec == "mixed",
                                         pdis, angv)
    assert oC.sum() > w.n // 4, "test needs contacts"
    rel = np.linalg.norm(F - oF) / np.linalg.norm(oF)
    relT = np.linalg.norm(T - oT) / np.linalg.norm(oT)
    assert rel <= rtol, rel
    assert relT <= (rtol if prec == "fp64" else 1e-3), relT
    if prec == "fp64":
        np.testing.assert_array_equal(C, oC)
    else:
        assert np.count_nonzero(C != oC) <= max(2, w.n // 1000)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_trajectory_lattice_2k(dem, orc, wl, cuda, prec):
    """2,000 spheres, 2,000 steps (100 re-lists with history carry)."""
    w = wl.lattice_2k()
    steps = 2000
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    e = make_engine(dem, w, p)
    e.step(steps)
    s = e.scalars()
    pos, pdis, angv = e.download()
    cell = e.grid_info()[1]
    mat = dem.material_array(w.pp, w.pw)
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, prec == "mixed", steps,
                w.relist_interval)
    assert o["status"] == 0
    rms = np.sqrt(np.mean((pos - o["pos"]) ** 2))
    tol = 1e-9 if prec == "fp64" else 1e-5
    assert rms <= tol, rms
    assert s["relists"] == steps // w.relist_interval
    assert s["pairs"] == int(o["npairs"][-1])
    oc = int(o["ncontacts"][-1])
    if prec == "fp64":
        assert s["contacts"] == oc
    assert abs(s["maxhz"] - o["maxhz"][-1]) < 1e-6
    pf_o = np.sum(4.0 / 3.0 * np.pi * w.rad ** 3) / (w.world[0] * w.world[1] * o["maxhz"][-1])
    assert abs(s["packing_fraction"] - pf_o) <= 1e-3
    assert abs(s["mean_cn"] - 2.0 * oc / w.n) <= 0.02


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_config1_full_run(dem, orc, wl, cuda, prec):
    """The 2,000-sphere lattice configuration at its full length, 20,000
    steps (1,000 re-lists; the spheres fall, collide and settle into a bed
    with ~1,650 contacts), stepped in ten calls: the FP64 engine tracks the
    FP64 oracle to 1e-10 d with the same contact count, the mixed engine to
    1e-5 d with the packing fraction within 1e-3 and the mean coordination
    number within 0.02."""
    w = wl.lattice_2k()
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    e = make_engine(dem, w, p)
    for _ in range(10):
        e.step(w.steps // 10)
    s = e.scalars()
    pos, _, _ = e.download()
    cell = e.grid_info()[1]
    e.close()
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(w.pp, w.pw), prec == "mixed",
                w.steps, w.relist_interval)
    assert s["status"] == 0 and o["status"] == 0
    assert s["relists"] == w.steps // w.relist_interval
    oc = int(o["ncontacts"][-1])
    assert oc > 1000                                   # a settled bed, not a free fall
    rms = np.sqrt(np.mean((pos - o["pos"]) ** 2))
    pf_o = np.sum(4.0 / 3.0 * np.pi * w.rad ** 3) / (w.world[0] * w.world[1] * o["maxhz"][-1])
    if prec == "fp64":
        assert rms <= 1e-10, rms
        assert s["contacts"] == oc
    else:
        assert rms <= 1e-5, rms
    assert abs(s["packing_fraction"] - pf_o) <= 1e-3
    assert abs(s["mean_cn"] - 2.0 * oc / w.n) <= 0.02


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_dense_trajectory_and_history_carry(dem, orc, wl, cuda, prec):
    """A bed with ~3,500 persistent contacts, 401 steps (21 re-lists): every
    pair's carried FP64 tangential history, the positions and the contact
    count against the oracle loop."""
    w = dense_lattice(dem)
    rng = np.random.default_rng(5)
    pdis = rng.normal(0, 2e-6, 3 * w.n)
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    e = dem.Engine(**{**w.engine_kwargs(), "precision": p})
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad, pdis, None)
    steps = 20 * w.relist_interval + 1
    e.step(steps)
    s = e.scalars()
    lp, ln, hist = e.pairs()
    cell = e.grid_info()[1]
    mat = dem.material_array(w.pp, w.pw)
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, mat, prec == "mixed", steps,
                w.relist_interval, pdis=pdis)
    assert o["status"] == 0 and s["status"] == 0
    pos_g, _, _ = e.download()
    rms = np.sqrt(np.mean((pos_g - o["pos"]) ** 2))
    assert rms < (1e-10 if prec == "fp64" else 1e-6), rms
    np.testing.assert_array_equal(ln, o["list_ln"])
    live = np.count_nonzero(np.abs(o["list_hist"]) > 0)
    assert live > 1000
    herr = np.linalg.norm(hist - o["list_hist"]) / np.linalg.norm(o["list_hist"])
    assert herr < (1e-8 if prec == "fp64" else 2e-3), herr
    oc = int(o["ncontacts"][-1])
    assert oc > 3000
    if prec == "fp64":
        assert s["contacts"] == oc
    else:
        assert abs(s["contacts"] - oc) <= max(3, oc // 500)


def test_full_size_rsa_500k_list_bit_exact(dem, orc, wl, cuda):
    """The 500,000-sphere workload: FP32 cell keys and the canonical pair set
    match the oracle exactly at full size."""
    w = wl.rsa_500k(precision=dem.PREC_MIXED)
    e = make_engine(dem, w)
    e.step(1)
    keys, ids, st, en = e.cells()
    cell = e.grid_info()[1]
    g, sk, si, cs, ce = oracle_cells(orc, w, cell, True)
    np.testing.assert_array_equal(keys, sk)
    np.testing.assert_array_equal(ids, si)
    lp, ln, _ = e.pairs()
    off, oln, _, _ = orc.build_list(w.pos, w.rad, w.world, cell, w.skin, True)
    np.testing.assert_array_equal(ln, oln)
    np.testing.assert_array_equal(lp, np.repeat(np.arange(w.n, dtype=np.uint32), np.diff(off)))
    # size-independent properties: rows sorted, i < j, each pair once
    assert np.all(lp < ln)
    key = lp.astype(np.uint64) << np.uint64(32) | ln.astype(np.uint64)
    assert np.all(np.diff(key) > 0)


def test_full_size_bidisperse_4m(dem, orc, wl, cuda):
    """The 4,000,000-sphere bidisperse workload (radii 0.4/0.6 mm, 200x200x600
    mm): the canonical pair set at full size matches the oracle exactly, ten
    windows run clean, and the mixed form's packing fraction is the FP64
    form's within 1e-3."""
    w = wl.bidisperse_4m()
    e = make_engine(dem, w)
    e.step(1)
    keys, ids, st, en = e.cells()
    cell = e.grid_info()[1]
    g, sk, si, cs, ce = oracle_cells(orc, w, cell, True)
    np.testing.assert_array_equal(keys, sk)
    np.testing.assert_array_equal(ids, si)
    lp, ln, _ = e.pairs()
    off, oln, _, _ = orc.build_list(w.pos, w.rad, w.world, cell, w.skin, True)
    np.testing.assert_array_equal(ln, oln)
    np.testing.assert_array_equal(lp, np.repeat(np.arange(w.n, dtype=np.uint32), np.diff(off)))
    e.step(10 * w.relist_interval - 1)
    s = e.scalars()
    assert s["status"] == 0 and s["relists"] == 10
    lp, ln, _ = e.pairs()
    key = lp.astype(np.uint64) << np.uint64(32) | ln.astype(np.uint64)
    assert np.all(lp < ln) and np.all(np.diff(key) > 0)
    f = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64})
    f.set_material(w.pp, w.pw)
    f.upload(w.pos, w.rad)
    f.step(10 * w.relist_interval)
    assert abs(f.scalars()["packing_fraction"] - s["packing_fraction"]) <= 1e-3


def test_mixed_vs_fp64_oracle_packing_fraction(dem, orc, wl, cuda):
    """Mixed-precision run of a reduced rsa workload (20,000 spheres, 1,000
    steps) against the FP64 oracle: packing fraction within 1e-3."""
    w = wl.rsa_500k(precision=dem.PREC_MIXED, n=20_000, box=(30.0, 30.0, 120.0))
    steps = 1000
    e = make_engine(dem, w)
    e.step(steps)
    s = e.scalars()
    pos, _, _ = e.download()
    cell = e.grid_info()[1]
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(w.pp, w.pw), False, steps,
                w.relist_interval)
    pf_o = np.sum(4.0 / 3.0 * np.pi * w.rad ** 3) / (w.world[0] * w.world[1] * o["maxhz"][-1])
    assert abs(s["packing_fraction"] - pf_o) <= 1e-3
    assert np.sqrt(np.mean((pos - o["pos"]) ** 2)) <= 1e-5


def test_capacity_overflow_is_reported(dem, wl, cuda):
    w = wl.small_box(n=3000, compress=0.8)
    e = make_engine(dem, w, pair_capacity=10)
    e.step(5)
    with pytest.raises(dem.DemError) as ei:
        e.scalars()
    assert ei.value.code == dem.DEM_ERR_CAPACITY


def test_skin_violation_is_reported(dem, wl, cuda):
    w = wl.small_box(n=2000)
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    pdis = np.zeros(3 * w.n)
    pdis[0::3] = 0.01   # 0.01 d per step: skin/2 = 0.025 passed after 3 steps
    e.upload(w.pos, w.rad, pdis, None)
    e.step(10)
    with pytest.raises(dem.DemError) as ei:
        e.scalars()
    assert ei.value.code == dem.DEM_ERR_SKIN


def test_nonfinite_is_reported(dem, wl, cuda):
    w = wl.small_box(n=2000)
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    pdis = np.zeros(3 * w.n)
    pdis[5] = np.nan
    e.upload(w.pos, w.rad, pdis, None)
    e.step(2)
    with pytest.raises(dem.DemError) as ei:
        e.scalars()
    assert ei.value.code == dem.DEM_ERR_NONFINITE


def test_nonfinite_free_particle_in_a_window_is_reported(dem, wl, cuda):
    """A free particle's non-finite displacement, stepped through whole
    windows (its check made once on the window's final state), is reported."""
    w = wl.small_box(n=2000)
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    pdis = np.zeros(3 * w.n)
    top = int(np.argmax(w.pos[2::3]))   # the highest sphere: free in the first window
    pdis[3 * top] = np.inf
    e.upload(w.pos, w.rad, pdis, None)
    e.step(w.relist_interval)   # one whole window (its graph), re-listed at finite positions
    with pytest.raises(dem.DemError) as ei:
        e.scalars()
    assert ei.value.code == dem.DEM_ERR_NONFINITE


@pytest.mark.parametrize("bad", [0.0, -1e-4, np.nan])
def test_upload_rejects_a_radius_that_is_not_positive(dem, wl, cuda, bad):
    w = wl.small_box(n=2000)
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    rad = w.rad.copy()
    rad[777] = bad
    with pytest.raises(dem.DemError) as ei:
        e.upload(w.pos, rad)
    assert ei.value.code == dem.DEM_ERR_ARG and "777" in str(ei.value)
    e.upload(w.pos, w.rad)   # the context stays usable
    e.step(3)
    assert e.scalars()["status"] == 0


def test_partial_windows_equal_graph_windows(dem, wl, cuda):
    """dem_step_n(1) x N (eager launches) and dem_step_n(N) (graphs) agree bit
    for bit."""
    w = wl.small_box(n=3000)
    a = make_engine(dem, w)
    b = make_engine(dem, w)
    a.step(45)
    for _ in range(45):
        b.step(1)
    pa, da, aa = a.download()
    pb, db, ab = b.download()
    np.testing.assert_array_equal(pa, pb)
    np.testing.assert_array_equal(da, db)
    np.testing.assert_array_equal(aa, ab)


def test_window_timing_graphs_equal_plain_graphs(dem, wl, cuda):
    """Windows replayed from the graph variant with timing events give the
    same state bit for bit, and per-kernel times of the last timed window."""
    w = wl.small_box(n=3000)
    a = make_engine(dem, w)
    b = make_engine(dem, w)
    K = w.relist_interval
    a.step(3 * K)
    b.step(K)
    b.set_window_timing(True)
    b.step(K)
    b.set_window_timing(False)
    b.step(K)
    kt = b.window_kernel_times()
    assert kt["relist_ms"] > 0, kt
    assert kt["window_kernel_ms"] > 0 or (kt["pair_ms"] > 0 and kt["particle_ms"] > 0), kt
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("mode", ["pccp", "pp"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_window_kernel_equals_per_step_kernels(dem, wl, cuda, monkeypatch, prec, mode):
    """Whole windows as one cooperative launch (the default) and as per-step
    kernels (DEM_B200_WINDOW=0: PCCP pair / particle kernels with the forked
    free-particle kernel, or the PP step kernel) agree bit for bit, dense bed
    included."""
    from _cases import dense_lattice
    fm = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    for w in (wl.small_box(n=3000), dense_lattice(dem, nx=8, ny=8, nz=6)):
        p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
        rng = np.random.default_rng(3)
        pdis = rng.normal(0, 2e-6, 3 * w.n)
        a = make_engine(dem, w, p, force_mode=fm)
        a.upload(w.pos, w.rad, pdis, None)
        monkeypatch.setenv("DEM_B200_WINDOW", "0")
        b = make_engine(dem, w, p, force_mode=fm)
        b.upload(w.pos, w.rad, pdis, None)
        monkeypatch.delenv("DEM_B200_WINDOW")
        a.step(3 * w.relist_interval)
        b.step(3 * w.relist_interval)
        for x, y in zip(a.download(), b.download()):
            np.testing.assert_array_equal(x, y)
        sa, sb = a.scalars(), b.scalars()
        assert sa["status"] == 0 and sb["status"] == 0
        assert sa["maxhz"] == sb["maxhz"] and sa["contacts"] == sb["contacts"]
        a.close()
        b.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cluster_batches_equal_grid_barrier_window(dem, wl, cuda, monkeypatch, prec):
    """The cluster-batched window (the default for PCCP: the bound particles'
    connected components packed into batches that one block steps through
    the window in shared memory, the free particles beside them) and the
    grid-barrier window kernel (DEM_B200_BATCH=0) agree bit for bit -- states,
    pair histories, observables -- on a sparse bed, a compressed bed with
    chains of contacts, and a dense lattice that is one component too large
    for a block (which the batched context hands to the grid-barrier kernel)."""
    from _cases import dense_lattice
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    # the compressed bed's overlaps throw spheres past the skin guard: both
    # paths must report it alike (status compared, not required zero there)
    cases = [(wl.small_box(n=3000), 1), (wl.small_box(n=4000, compress=0.85), None),
             (dense_lattice(dem, nx=10, ny=10, nz=8), 0)]
    for w, batched in cases:
        rng = np.random.default_rng(9)
        pdis = rng.normal(0, 2e-6, 3 * w.n)
        angv = rng.normal(0, 2e-5, 3 * w.n)
        a = make_engine(dem, w, p)
        a.upload(w.pos, w.rad, pdis, angv)
        monkeypatch.setenv("DEM_B200_BATCH", "0")
        b = make_engine(dem, w, p)
        b.upload(w.pos, w.rad, pdis, angv)
        monkeypatch.delenv("DEM_B200_BATCH")
        a.step(4 * w.relist_interval)
        b.step(4 * w.relist_interval)
        wa, wb = a.window_work(), b.window_work()
        assert wb["batched"] == -1 and (batched is None or wa["batched"] == batched), (w.name, wa, wb)
        print(f"\n{w.name} n={w.n}: {wa}")
        assert wa["bound"] == wb["bound"] > 0
        for x, y in zip(a.download(), b.download()):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(a.pairs(), b.pairs()):
            np.testing.assert_array_equal(x, y)
        sa, sb = a.scalars(raise_on_status=False), b.scalars(raise_on_status=False)
        assert sa["status"] == sb["status"] and (batched is None or sa["status"] == 0), (sa["status"], sb["status"])
        assert sa["maxhz"] == sb["maxhz"] and sa["contacts"] == sb["contacts"]
        a.close()
        b.close()


@pytest.mark.parametrize("fork", ["0", "2"])
def test_free_particles_fork_point_is_invisible(dem, wl, cuda, monkeypatch, fork):
    """A batched window's free particles stepped from the re-list's second
    stream after the candidate pass (the default), after the fill
    (DEM_B200_FREE_FORK=2) or in the window beside the batches
    (DEM_B200_FREE_FORK=0): the same states, lists and observables, on a
    sparse bed (batched) and a dense lattice (the grid-barrier window kernel
    beside the free kernel)."""
    from _cases import dense_lattice
    for w in (wl.small_box(n=3000), dense_lattice(dem, nx=10, ny=10, nz=8)):
        rng = np.random.default_rng(5)
        pdis = rng.normal(0, 2e-6, 3 * w.n)
        a = make_engine(dem, w)
        a.upload(w.pos, w.rad, pdis, None)
        monkeypatch.setenv("DEM_B200_FREE_FORK", fork)
        b = make_engine(dem, w)
        b.upload(w.pos, w.rad, pdis, None)
        monkeypatch.delenv("DEM_B200_FREE_FORK")
        a.step(6 * w.relist_interval)
        b.step(6 * w.relist_interval)
        assert a.window_work() == b.window_work()
        for x, y in zip(a.download(), b.download()):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(a.pairs(), b.pairs()):
            np.testing.assert_array_equal(x, y)
        sa, sb = a.scalars(), b.scalars()
        assert sa["maxhz"] == sb["maxhz"] and sa["contacts"] == sb["contacts"] and sa["pairs"] == sb["pairs"]
        a.close()
        b.close()


def test_plain_launches_equal_programmatic_launches(dem, wl, cuda, monkeypatch):
    """Re-list and step kernels launched programmatically (the default) and
    launched plainly (DEM_B200_PDL=0) agree bit for bit, with the per-step
    kernels and with the window kernel."""
    w = wl.small_box(n=3000)
    for window in ("0", "1"):
        monkeypatch.setenv("DEM_B200_WINDOW", window)
        monkeypatch.setenv("DEM_B200_PDL", "1")
        a = make_engine(dem, w)
        monkeypatch.setenv("DEM_B200_PDL", "0")
        b = make_engine(dem, w)
        a.step(45)
        b.step(45)
        for x, y in zip(a.download(), b.download()):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(a.pairs(), b.pairs()):
            np.testing.assert_array_equal(x, y)
        a.close()
        b.close()


def test_device_upload_download_roundtrip(dem, wl, cuda):
    torch = cuda
    w = wl.small_box(n=2000)
    e = dem.Engine(**w.engine_kwargs())
    e.set_material(w.pp, w.pw)
    tpos = torch.from_numpy(w.pos).cuda()
    trad = torch.from_numpy(w.rad).cuda()
    e.upload_device(tpos, trad)
    out = torch.empty_like(tpos)
    e.download_device(pos=out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), w.pos)
    g, cell, nc = e.grid_info()
    assert abs(cell - w.cell()) < 1e-15


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("interval", [20, 7])
def test_pp_mode_matches_pccp(dem, wl, cuda, prec, interval):
    """The particle-parallel step (each pair evaluated by both particles, one
    kernel per step, ping-pong buffers) agrees with the pair-parallel step to
    rounding (the compiler may contract multiply-adds differently in the two
    kernels: ~1e-13 relative in FP64); an odd re-list interval exercises the
    buffer parity of the captured windows."""
    w = dense_lattice(dem)
    rng = np.random.default_rng(9)
    pdis = rng.normal(0, 2e-6, 3 * w.n)
    angv = rng.normal(0, 2e-6, 3 * w.n)
    p = dem.PREC_FP64 if prec == "fp64" else dem.PREC_MIXED
    out = []
    for mode in (dem.FORCE_PCCP, dem.FORCE_PP):
        e = dem.Engine(**{**w.engine_kwargs(), "precision": p, "relist_interval": interval, "force_mode": mode})
        e.set_material(w.pp, w.pw)
        e.upload(w.pos, w.rad, pdis, angv)
        e.step(5 * interval + 3)     # graph windows, then an eager partial window
        e.step(interval - 1)
        s = e.scalars()
        lp, ln, hist = e.pairs()
        out.append((e.download(), s, ln, hist))
        e.close()
    (a, sa, lna, ha), (b, sb, lnb, hb) = out
    tol = 1e-9 if prec == "fp64" else 1e-7
    np.testing.assert_allclose(b[0], a[0], rtol=0, atol=tol)                      # positions
    for x, y in zip(a[1:], b[1:]):                                                # per-step motion
        np.testing.assert_allclose(y, x, rtol=0, atol=1e-6 * max(np.abs(x).max(), 1e-30))
    np.testing.assert_array_equal(lna, lnb)
    assert np.linalg.norm(ha - hb) <= 1e-6 * np.linalg.norm(ha)
    assert abs(sa["contacts"] - sb["contacts"]) <= 2 and sa["contacts"] > 1000
    assert abs(sa["maxhz"] - sb["maxhz"]) <= tol


def test_pp_mode_trajectory_vs_oracle(dem, orc, wl, cuda):
    w = wl.lattice_2k()
    steps = 1000
    e = dem.Engine(**{**w.engine_kwargs(), "force_mode": dem.FORCE_PP})
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    e.step(steps)
    pos, _, _ = e.download()
    cell = e.grid_info()[1]
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, cell, w.density, dem.material_array(w.pp, w.pw), False, steps,
                w.relist_interval)
    assert np.sqrt(np.mean((pos - o["pos"]) ** 2)) <= 1e-9


def test_barrier_wait_gives_up_and_context_stays_usable(dem, wl, cuda):
    """The window kernel's grid-barrier wait is bounded: a wait for an arrival
    that never comes gives up after about a second, the status word reports
    DEM_ERR_TIMEOUT, and after a new upload the context steps exactly as a
    fresh one does (no fault, no hang, nothing left behind)."""
    w = wl.small_box(n=2000)
    e = make_engine(dem, w)
    e.step(w.relist_interval)
    ms = e.check_barrier_timeout()
    assert 900.0 <= ms <= 30000.0, ms
    assert e.scalars()["status"] == dem.DEM_ERR_TIMEOUT
    e.upload(w.pos, w.rad)
    e.step(3 * w.relist_interval)
    assert e.scalars()["status"] == 0
    f = make_engine(dem, w)
    f.step(3 * w.relist_interval)
    for x, y in zip(e.download(), f.download()):
        np.testing.assert_array_equal(x, y)


def test_observables_without_a_host_wait(dem, wl, cuda):
    """dem_scalars_enqueue after every window (pinned buffers, no wait), one
    synchronisation, then dem_scalars_from_raw: the same observables, step by
    step, as dem_get_scalars on a second context; a buffer is refused by a
    context of another size."""
    import torch
    w = wl.small_box(n=3000)
    K = w.relist_interval
    a, b = make_engine(dem, w), make_engine(dem, w)
    rb = a.scalars_raw_bytes()
    raws = torch.empty((6, rb), dtype=torch.uint8).pin_memory()
    sync = []
    for k in range(6):
        a.step(K + (k == 3) * 7)                      # one call ends inside a window
        a.scalars_enqueue(raws[k].data_ptr())
        b.step(K + (k == 3) * 7)
        sync.append(b.scalars())
    a.synchronize()
    for k in range(6):
        assert a.scalars_from_raw(raws[k].data_ptr()) == sync[k], k
    other = make_engine(dem, wl.rsa_500k(precision=dem.PREC_MIXED, n=30_000, box=(40.0, 40.0, 120.0)))
    with pytest.raises(dem.DemError) as e:
        other.scalars_from_raw(raws[0].data_ptr())
    assert e.value.code == dem.DEM_ERR_ARG


def _state_header(dem):
    import ctypes

    class StateHeader(ctypes.Structure):   # the state file's header (dem_save_state)
        _fields_ = [("magic", ctypes.c_char * 8), ("version", ctypes.c_int), ("precision", ctypes.c_int),
                    ("force_mode", ctypes.c_int), ("relist_interval", ctypes.c_int), ("n", ctypes.c_longlong),
                    ("step", ctypes.c_longlong), ("relists", ctypes.c_longlong), ("npairs", ctypes.c_longlong),
                    ("dt", ctypes.c_double), ("skin", ctypes.c_double), ("cell", ctypes.c_double),
                    ("density", ctypes.c_double), ("world", ctypes.c_double * 3), ("rmax", ctypes.c_double),
                    ("vol", ctypes.c_double), ("have_mat", ctypes.c_int), ("pouring", ctypes.c_int),
                    ("mat", dem.Material), ("n_active", ctypes.c_longlong), ("pour_nplayer", ctypes.c_longlong),
                    ("pour_tnewpar", ctypes.c_double), ("ordered", ctypes.c_longlong)]
    return StateHeader


@pytest.mark.parametrize("n_side", [2, 9])
def test_upload_order_is_the_cell_order(dem, wl, cuda, tmp_path, n_side):
    """The order a host upload gives the particles, computed on the device, is
    the stable (cell key, id) order on the context's grid (read back from a
    state file); 64 particles or fewer keep the caller's order."""
    w = dense_lattice(dem, nx=n_side, ny=n_side, nz=6)
    rng = np.random.default_rng(23)
    perm = rng.permutation(w.n)
    pos = w.pos.reshape(-1, 3)[perm].reshape(-1).copy()
    rad = w.rad[perm].copy()
    e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_MIXED})
    e.set_material(w.pp, w.pw)
    e.upload(pos, rad)
    e.save_state(tmp_path / "s.bin")
    cs = e.grid_info()[1]
    e.close()
    H = _state_header(dem)
    raw = (tmp_path / "s.bin").read_bytes()
    h = H.from_buffer_copy(raw[:__import__("ctypes").sizeof(H)])
    assert h.magic == b"DEMB200S" and h.n == w.n
    if w.n <= 64:
        assert h.ordered == 0
        return
    assert h.ordered == 1
    got = np.frombuffer(raw, dtype=np.uint32, count=w.n, offset=__import__("ctypes").sizeof(H))
    g = [int(x / cs) + 1 for x in w.world]
    p = pos.reshape(-1, 3)

    def cell(v, gn):
        f = v / cs
        return np.where(~(f >= 0.0), 0, np.where(f >= gn, gn - 1, np.floor(np.maximum(f, 0.0)))).astype(np.int64)

    key = (cell(p[:, 2], g[2]) * g[1] + cell(p[:, 1] + 0.5 * w.world[1], g[1])) * g[0] + \
        cell(p[:, 0] + 0.5 * w.world[0], g[0])
    np.testing.assert_array_equal(got, np.argsort(key, kind="stable"))


def test_cell_order_is_invisible(dem, wl, cuda, monkeypatch):
    """A host upload sorts the particles by cell inside the context; every
    result leaves in the caller's order: the state round-trips exactly, and a
    run agrees with one in the caller's order (DEM_B200_REORDER=0) -- same
    canonical pair set, histories and positions to rounding."""
    w = dense_lattice(dem, nx=9, ny=9, nz=6)
    rng = np.random.default_rng(17)
    perm = rng.permutation(w.n)           # the caller's order: spatially scrambled
    pos = w.pos.reshape(-1, 3)[perm].reshape(-1).copy()
    rad = w.rad[perm].copy()
    pdis = rng.normal(0, 2e-6, 3 * w.n)
    angv = rng.normal(0, 2e-5, 3 * w.n)
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("DEM_B200_REORDER", flag)
        e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64})
        e.set_material(w.pp, w.pw)
        e.upload(pos, rad, pdis, angv)
        p0, d0, a0 = e.download()
        np.testing.assert_array_equal(p0, pos)
        np.testing.assert_array_equal(d0, pdis)
        np.testing.assert_array_equal(a0, angv)
        e.step(5 * w.relist_interval + 3)
        out.append((e.download(), e.pairs(), e.scalars()))
    (sa, pa, ca), (sb, pb, cb) = out
    assert ca["status"] == cb["status"] == 0
    assert ca["contacts"] == cb["contacts"] > 100 and ca["pairs"] == cb["pairs"]
    np.testing.assert_array_equal(pa[0], pb[0])
    np.testing.assert_array_equal(pa[1], pb[1])
    np.testing.assert_allclose(pa[2], pb[2], rtol=0, atol=1e-12 * np.abs(pb[2]).max())
    for x, y in zip(sa, sb):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-12 * max(np.abs(y).max(), 1e-30))
