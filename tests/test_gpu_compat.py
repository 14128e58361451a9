"""GPU parity of the reference-compatible entry points (particleSystem.cu's
extern "C" wrappers + RadixSort) against the CPU oracle's restatement of the
same calls.  Integer/list outputs are compared bit-exactly; FP64 forces to
1e-10 relative (both sides FP64; they differ only by FMA contraction)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-10


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a.copy()).cuda()


def host(t, dtype=None):
    a = t.detach().cpu().numpy()
    if dtype == np.uint32:
        a = a.view(np.uint32)
    return a


def zeros(torch, n, dtype):
    tdt = {np.uint32: torch.int32, np.float64: torch.float64}[dtype]
    return torch.zeros(int(n), dtype=tdt, device="cuda")


def ref_material():
    par = dict(estarp=566830.28, ufricp=0.4, vpois=0.29, dampnp=0.3, damptp=0.25, upp=0.002)
    parw = dict(estarw=566830.28, ufricw=0.35, vpoisw=0.29, dampnw=0.3, damptw=0.2, upw=0.001)
    return par, parw


@pytest.fixture(scope="module")
def setup(dem, orc, cuda):
    par, parw = ref_material()
    dem.compat.set_material(par, parw)
    dem.compat.set_cutoff(1.0, 1.55)
    orc.lib().ref_set_material(orc.P(np.array(list(par.values()))), orc.P(np.array(list(parw.values()))))
    orc.lib().ref_set_cutoff(1.0, 1.55)
    return dem, orc, cuda


def cloud(n, side, seed, zlo=0.0, outside=0.0):
    rng = np.random.default_rng(seed)
    p = np.empty((n, 3))
    p[:, 0] = rng.uniform(-side / 2 - outside, side / 2 + outside, n)
    p[:, 1] = rng.uniform(-side / 2 - outside, side / 2 + outside, n)
    p[:, 2] = rng.uniform(zlo - outside, side + outside, n)
    return p.reshape(-1)


GRID_SIDE = 34.0
CELL = (1.55, 1.55, 1.55)
ORIGIN = (-17.0, -17.0, 0.0)
GS = tuple(int(GRID_SIDE / 1.55) + 1 for _ in range(3))


def test_calc_hash_bit_exact(setup):
    dem, orc, torch = setup
    n = 50_000
    pos = cloud(n, GRID_SIDE, 1, outside=2.0)   # includes positions outside the grid on every side
    ph = zeros(torch, 2 * n, np.uint32)
    dem.compat.calcHash(dev(torch, pos), ph, GS, CELL, ORIGIN, n)
    torch.cuda.synchronize()
    ref = np.empty(2 * n, dtype=np.uint32)
    orc.lib().ref_calcHash(orc.P(pos), orc.P(ref), orc.P(np.array(GS, dtype=np.uint32)), orc.P(np.array(CELL)),
                           orc.P(np.array(ORIGIN)), n)
    np.testing.assert_array_equal(host(ph, np.uint32), ref)


@pytest.mark.parametrize("n,bits", [(1, 32), (2047, 32), (100_003, 32), (1_000_000, 20), (300_001, 24)])
def test_radix_sort_stable_bit_exact(setup, n, bits):
    dem, orc, torch = setup
    rng = np.random.default_rng(n)
    kv = np.empty(2 * n, dtype=np.uint32)
    kv[0::2] = rng.integers(0, min(2 ** bits, 5000 if n > 1000 else 2 ** bits), n, dtype=np.uint64).astype(np.uint32)
    kv[1::2] = np.arange(n, dtype=np.uint32)
    d0 = dev(torch, kv)
    d1 = zeros(torch, 2 * n, np.uint32)
    dem.compat.RadixSort(d0, d1, n, bits)
    torch.cuda.synchronize()
    ref = kv.copy()
    orc.lib().ref_radix_sort(orc.P(ref), n, bits)
    np.testing.assert_array_equal(host(d0, np.uint32), ref)


def test_radix_sort_full_32bit_keys(setup):
    dem, orc, torch = setup
    n = 200_000
    rng = np.random.default_rng(7)
    kv = np.empty(2 * n, dtype=np.uint32)
    kv[0::2] = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    kv[0::2][::5] = 123456   # many ties
    kv[1::2] = rng.permutation(n).astype(np.uint32)
    d0 = dev(torch, kv)
    d1 = zeros(torch, 2 * n, np.uint32)
    dem.compat.RadixSort(d0, d1, n, 32)
    torch.cuda.synchronize()
    ref = kv.copy()
    orc.lib().ref_radix_sort(orc.P(ref), n, 32)
    np.testing.assert_array_equal(host(d0, np.uint32), ref)


def build_reference_list(dem, orc, torch, pos, n, maxppc=30):
    """calcHash -> RadixSort -> findCellStart -> neighborarray on GPU and oracle."""
    ncell = GS[0] * GS[1] * GS[2]
    g_pos = dev(torch, pos)
    ph = zeros(torch, 2 * n, np.uint32)
    tmp = zeros(torch, 2 * n, np.uint32)
    cst = zeros(torch, ncell, np.uint32)
    anei = zeros(torch, n * maxppc, np.uint32)
    njgi = zeros(torch, n, np.uint32)
    njli = zeros(torch, n, np.uint32)
    dem.compat.calcHash(g_pos, ph, GS, CELL, ORIGIN, n)
    dem.compat.RadixSort(ph, tmp, n, 32)
    dem.compat.findCellStart(ph, cst, n, ncell)
    dem.compat.neighborarray(g_pos, ph, cst, GS, CELL, ORIGIN, maxppc, n, anei, njgi, njli)
    torch.cuda.synchronize()
    L = orc.lib()
    h = np.empty(2 * n, dtype=np.uint32)
    gsa, csa, oa = np.array(GS, dtype=np.uint32), np.array(CELL), np.array(ORIGIN)
    L.ref_calcHash(orc.P(pos), orc.P(h), orc.P(gsa), orc.P(csa), orc.P(oa), n)
    L.ref_radix_sort(orc.P(h), n, 32)
    c = np.empty(ncell, dtype=np.uint32)
    L.ref_findCellStart(orc.P(h), orc.P(c), n, ncell)
    A = np.empty(n * maxppc, dtype=np.uint32)
    ng = np.empty(n, dtype=np.uint32)
    nl = np.empty(n, dtype=np.uint32)
    ovf = L.ref_neighborarray(orc.P(pos), orc.P(h), orc.P(c), orc.P(gsa), orc.P(csa), orc.P(oa), maxppc, n,
                              orc.P(A), orc.P(ng), orc.P(nl))
    assert ovf == 0
    gpu = dict(pos=g_pos, ph=ph, cst=cst, anei=anei, njgi=njgi, njli=njli)
    ref = dict(h=h, c=c, A=A, ng=ng, nl=nl)
    return gpu, ref


def test_cell_start_and_neighbor_rows_bit_exact(setup):
    dem, orc, torch = setup
    n = 20_000
    pos = cloud(n, GRID_SIDE, 2)
    gpu, ref = build_reference_list(dem, orc, torch, pos, n)
    np.testing.assert_array_equal(host(gpu["ph"], np.uint32), ref["h"])
    np.testing.assert_array_equal(host(gpu["cst"], np.uint32), ref["c"])
    np.testing.assert_array_equal(host(gpu["njgi"], np.uint32), ref["ng"])
    np.testing.assert_array_equal(host(gpu["njli"], np.uint32), ref["nl"])
    np.testing.assert_array_equal(host(gpu["anei"], np.uint32), ref["A"])
    assert ref["ng"].sum() > 2 * n   # a meaningful number of pairs


def test_neighbor_overflow_reports_capacity(setup):
    dem, orc, torch = setup
    n = 4000
    pos = cloud(n, 8.0, 3)   # dense: rows far above 4 slots
    with pytest.raises(dem.DemError) as ei:
        build_reference_list(dem, orc, torch, pos, n, maxppc=4)
    assert ei.value.code == dem.DEM_ERR_CAPACITY


def test_prefixsum_and_pairlist_with_history_carry(setup):
    dem, orc, torch = setup
    n, maxppc, maxcn = 20_000, 30, 30
    rng = np.random.default_rng(4)
    pos0 = cloud(n, GRID_SIDE, 5)
    L = orc.lib()
    # previous list from the oracle, with random histories, as "old" arrays
    _, r0 = build_reference_list(dem, orc, torch, pos0, n)
    cap = n * maxcn
    sj0 = np.zeros(n, dtype=np.uint32)
    osj = np.zeros(n, dtype=np.uint32)
    tot0 = L.ref_prefixsum(n, orc.P(r0["ng"]), orc.P(sj0), orc.P(osj))
    aref0 = np.empty(n * maxppc, dtype=np.uint32)
    lp0 = np.empty(cap, dtype=np.uint32)
    ln0 = np.empty(cap, dtype=np.uint32)
    dsp0 = np.empty(3 * cap)
    frp0 = np.empty(cap)
    zu = np.zeros(cap, dtype=np.uint32)
    zd3 = np.zeros(3 * cap)
    zd = np.zeros(cap)
    L.ref_pairlist(orc.P(sj0), orc.P(np.zeros(n, dtype=np.uint32)), orc.P(zu), orc.P(r0["A"]), orc.P(r0["ng"]),
                   orc.P(r0["nl"]), orc.P(zd3), orc.P(zd), maxppc, maxcn, n, orc.P(aref0), orc.P(lp0), orc.P(ln0),
                   orc.P(dsp0), orc.P(frp0))
    old_ln = ln0.copy()
    old_dispt = rng.normal(0, 1e-3, 3 * cap)
    old_fricp = rng.uniform(0, 1, cap)
    # move particles a little and rebuild on both sides
    pos1 = pos0 + rng.uniform(-0.05, 0.05, pos0.size)
    gpu, r1 = build_reference_list(dem, orc, torch, pos1, n)
    g_sj = dev(torch, sj0)
    g_osj = zeros(torch, n, np.uint32)
    tot_gpu = dem.compat.prefixsum(n, gpu["njgi"], g_sj, g_osj)
    sj1 = sj0.copy()
    osj1 = np.zeros(n, dtype=np.uint32)
    tot_ref = L.ref_prefixsum(n, orc.P(r1["ng"]), orc.P(sj1), orc.P(osj1))
    assert tot_gpu == tot_ref and tot0 > 0
    np.testing.assert_array_equal(host(g_sj, np.uint32), sj1)
    np.testing.assert_array_equal(host(g_osj, np.uint32), osj1)
    g_aref = zeros(torch, n * maxppc, np.uint32)
    g_lp = zeros(torch, cap, np.uint32)
    g_ln = zeros(torch, cap, np.uint32)
    g_dsp = zeros(torch, 3 * cap, np.float64)
    g_frp = zeros(torch, cap, np.float64)
    dem.compat.pairlist(g_sj, g_osj, dev(torch, old_ln), gpu["anei"], gpu["njgi"], gpu["njli"], dev(torch, old_dispt),
                        dev(torch, old_fricp), maxppc, maxcn, n, g_aref, g_lp, g_ln, g_dsp, g_frp)
    torch.cuda.synchronize()
    aref = np.empty(n * maxppc, dtype=np.uint32)
    lp = np.empty(cap, dtype=np.uint32)
    ln = np.empty(cap, dtype=np.uint32)
    dsp = np.empty(3 * cap)
    frp = np.empty(cap)
    L.ref_pairlist(orc.P(sj1), orc.P(osj1), orc.P(old_ln), orc.P(r1["A"]), orc.P(r1["ng"]), orc.P(r1["nl"]),
                   orc.P(old_dispt), orc.P(old_fricp), maxppc, maxcn, n, orc.P(aref), orc.P(lp), orc.P(ln),
                   orc.P(dsp), orc.P(frp))
    np.testing.assert_array_equal(host(g_aref, np.uint32), aref)
    np.testing.assert_array_equal(host(g_lp, np.uint32), lp)
    np.testing.assert_array_equal(host(g_ln, np.uint32), ln)
    np.testing.assert_array_equal(host(g_dsp), dsp)
    np.testing.assert_array_equal(host(g_frp), frp)
    carried = np.count_nonzero(frp[:tot_ref])
    assert 0 < carried < tot_ref   # some pairs kept their history, some are new


def contact_state(n_side=14, seed=9):
    """Overlapping lattice (spacing 0.999, r = 0.5) with random motion/history,
    near the floor and side walls."""
    rng = np.random.default_rng(seed)
    a = 0.999
    g = np.arange(n_side) * a
    X, Y, Z = np.meshgrid(g - g.mean(), g - g.mean(), g + 0.4995, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    pos += rng.uniform(-3e-4, 3e-4, pos.shape)
    n = pos.shape[0]
    pdis = rng.normal(0, 2e-5, (n, 3))
    angv = rng.normal(0, 2e-5, (n, 3))
    rad = np.full(n, 0.5)
    rmass = 8 * rad ** 3
    inert = 0.4 * rmass * rad ** 2
    world = (n_side * a - 0.0005, n_side * a - 0.0005, 40.0)
    return pos.reshape(-1), pdis.reshape(-1), angv.reshape(-1), rad, rmass, inert, world


def rel_err(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_force_pair_gather_wall_update_vs_oracle(setup):
    dem, orc, torch = setup
    L = orc.lib()
    pos, pdis, angv, rad, rmass, inert, world = contact_state()
    n = rad.size
    maxppc = maxcn = 30
    gpu, r = build_reference_list(dem, orc, torch, pos, n, maxppc)
    cap = n * maxcn
    sj = np.zeros(n, dtype=np.uint32)
    osj = np.zeros(n, dtype=np.uint32)
    tot = L.ref_prefixsum(n, orc.P(r["ng"]), orc.P(sj), orc.P(osj))
    aref = np.empty(n * maxppc, dtype=np.uint32)
    lp = np.empty(cap, dtype=np.uint32)
    ln = np.empty(cap, dtype=np.uint32)
    dsp = np.empty(3 * cap)
    frp = np.empty(cap)
    L.ref_pairlist(orc.P(sj), orc.P(osj), orc.P(np.zeros(cap, dtype=np.uint32)), orc.P(r["A"]), orc.P(r["ng"]),
                   orc.P(r["nl"]), orc.P(np.zeros(3 * cap)), orc.P(np.zeros(cap)), maxppc, maxcn, n, orc.P(aref),
                   orc.P(lp), orc.P(ln), orc.P(dsp), orc.P(frp))
    rng = np.random.default_rng(11)
    dsp[:3 * tot] = rng.normal(0, 1e-5, 3 * tot)   # live tangential histories
    dt = 1e-3
    # ---- pair force
    g = {k: dev(torch, v) for k, v in dict(pos=pos, pdis=pdis, angv=angv, rad=rad, rmass=rmass, lp=lp, ln=ln,
                                              dsp=dsp, frp=frp, inert=inert).items()}
    g_oldln = zeros(torch, cap, np.uint32)
    g_odsp = zeros(torch, 3 * cap, np.float64)
    g_ofrp = zeros(torch, cap, np.float64)
    g_fp = zeros(torch, 3 * cap, np.float64)
    g_ti = zeros(torch, 3 * cap, np.float64)
    g_tj = zeros(torch, 3 * cap, np.float64)
    g_cp = zeros(torch, cap, np.uint32)
    dem.compat.calculateforcepair(g["pos"], g["pdis"], g["angv"], g["rad"], g["rmass"], g["lp"], g["ln"], g_oldln,
                                  g["dsp"], g["frp"], g_odsp, g_ofrp, dt, g_fp, g_ti, g_tj, g_cp, tot)
    oldln = np.zeros(cap, dtype=np.uint32)
    odsp = np.zeros(3 * cap)
    ofrp = np.zeros(cap)
    fp = np.zeros(3 * cap)
    ti = np.zeros(3 * cap)
    tj = np.zeros(3 * cap)
    cp = np.zeros(cap, dtype=np.uint32)
    dsp_o, frp_o = dsp.copy(), frp.copy()
    L.ref_calculateforcepair(orc.P(pos), orc.P(pdis), orc.P(angv), orc.P(rad), orc.P(rmass), orc.P(lp), orc.P(ln),
                             orc.P(oldln), orc.P(dsp_o), orc.P(frp_o), orc.P(odsp), orc.P(ofrp), dt, orc.P(fp),
                             orc.P(ti), orc.P(tj), orc.P(cp), tot)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(g_cp, np.uint32), cp)
    np.testing.assert_array_equal(host(g_oldln, np.uint32)[:tot], oldln[:tot])
    assert cp[:tot].sum() > n   # many touching pairs
    for gv, rv in ((g_fp, fp), (g_ti, ti), (g_tj, tj), (g["dsp"], dsp_o), (g_odsp, odsp), (g["frp"], frp_o)):
        assert rel_err(host(gv)[: rv.size], rv) < FORCE_RTOL
    # ---- gather
    g_aref = dev(torch, aref)
    g_fi = zeros(torch, 3 * n, np.float64)
    g_tq = zeros(torch, 3 * n, np.float64)
    g_ci = zeros(torch, n, np.uint32)
    dem.compat.sumallforcei(maxppc, n, gpu["njgi"], gpu["njli"], g_fp, g_ti, g_tj, g_cp, g_aref, g_fi, g_tq, g_ci)
    fi = np.zeros(3 * n)
    tq = np.zeros(3 * n)
    ci = np.zeros(n, dtype=np.uint32)
    L.ref_sumallforcei(maxppc, n, orc.P(r["ng"]), orc.P(r["nl"]), orc.P(fp), orc.P(ti), orc.P(tj), orc.P(cp),
                       orc.P(aref), orc.P(fi), orc.P(tq), orc.P(ci))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(g_ci, np.uint32), ci)
    assert rel_err(host(g_fi), fi) < FORCE_RTOL
    assert rel_err(host(g_tq), tq) < FORCE_RTOL
    # Newton's third law: pair forces cancel in the sum
    assert abs(fi.reshape(-1, 3).sum(0)).max() < 1e-9 * abs(fi).max()
    # ---- walls + gravity
    dw = rng.normal(0, 1e-5, 3 * n)
    fw = rng.uniform(0, 1, n)
    g_dw, g_fw = dev(torch, dw), dev(torch, fw)
    dem.compat.calculateforceiw(world, g["pos"], g["pdis"], g["angv"], g["rad"], g["rmass"], dt, tot, n, g_dw, g_fw,
                                g_fi, g_tq)
    L.ref_calculateforceiw(orc.P(np.array(world)), orc.P(pos), orc.P(pdis), orc.P(angv), orc.P(rad), orc.P(rmass),
                           dt, tot, n, orc.P(dw), orc.P(fw), orc.P(fi), orc.P(tq))
    torch.cuda.synchronize()
    assert rel_err(host(g_fi), fi) < FORCE_RTOL
    assert rel_err(host(g_tq), tq) < FORCE_RTOL
    assert rel_err(host(g_dw), dw) < FORCE_RTOL
    assert rel_err(host(g_fw), fw) < FORCE_RTOL
    touching_wall = np.count_nonzero(fw)
    assert touching_wall > n // 10
    # ---- integrate
    qi = rng.uniform(-0.2, 0.2, 3 * n)
    g_qi = dev(torch, qi)
    iall_g, mz_g = dem.compat.updateposition(world, n, g["pos"], g["pdis"], g["angv"], g["rmass"], g["inert"], g_fi,
                                             g_tq, g_qi, dt)
    p2, d2, a2, q2 = pos.copy(), pdis.copy(), angv.copy(), qi.copy()
    mz = np.zeros(1)
    iall = L.ref_updateposition(orc.P(np.array(world)), n, orc.P(p2), orc.P(d2), orc.P(a2), orc.P(rmass),
                                orc.P(inert), orc.P(host(g_fi)), orc.P(host(g_tq)), orc.P(q2), dt, orc.P(mz))
    assert iall_g == iall
    assert mz_g == mz[0]
    np.testing.assert_array_equal(host(g["pos"]), p2)
    np.testing.assert_array_equal(host(g["pdis"]), d2)
    np.testing.assert_array_equal(host(g["angv"]), a2)
    np.testing.assert_array_equal(host(g_qi), q2)
    # ---- observables
    pc = dem.compat.outputporositycn(n, g_ci, mz_g, world)
    assert pc == L.ref_outputporositycn(n, orc.P(ci))


def test_compat_step_loop_matches_oracle(setup):
    """The reference's loop (dempacking.cu:535-739) through the compatible
    entry points for 300 steps, re-listing on the displacement flag."""
    dem, orc, torch = setup
    L = orc.lib()
    pos, pdis, angv, rad, rmass, inert, world = contact_state(n_side=10, seed=21)
    n = rad.size
    maxppc = maxcn = 30
    cap = n * maxcn
    dt = 2e-3
    ncell = GS[0] * GS[1] * GS[2]
    G = {}
    G["pos"], G["pdis"], G["angv"] = dev(torch, pos), dev(torch, pdis), dev(torch, angv)
    G["rad"], G["rmass"], G["inert"] = dev(torch, rad), dev(torch, rmass), dev(torch, inert)
    for k, sz, dt_ in (("ph", 2 * n, np.uint32), ("tmp", 2 * n, np.uint32), ("cst", ncell, np.uint32),
                       ("anei", n * maxppc, np.uint32), ("aref", n * maxppc, np.uint32), ("njgi", n, np.uint32),
                       ("njli", n, np.uint32), ("sj", n, np.uint32), ("osj", n, np.uint32), ("lp", cap, np.uint32),
                       ("ln", cap, np.uint32), ("oldln", cap, np.uint32), ("cp", cap, np.uint32),
                       ("ci", n, np.uint32), ("dsp", 3 * cap, np.float64), ("frp", cap, np.float64),
                       ("odsp", 3 * cap, np.float64), ("ofrp", cap, np.float64), ("fp", 3 * cap, np.float64),
                       ("ti", 3 * cap, np.float64), ("tj", 3 * cap, np.float64), ("dw", 3 * n, np.float64),
                       ("fw", n, np.float64), ("fi", 3 * n, np.float64), ("tq", 3 * n, np.float64),
                       ("qi", 3 * n, np.float64)):
        G[k] = zeros(torch, sz, dt_)
    H = dict(pos=pos.copy(), pdis=pdis.copy(), angv=angv.copy())
    for k, sz, dt_ in (("h", 2 * n, np.uint32), ("cst", ncell, np.uint32), ("anei", n * maxppc, np.uint32),
                       ("aref", n * maxppc, np.uint32), ("njgi", n, np.uint32), ("njli", n, np.uint32),
                       ("sj", n, np.uint32), ("osj", n, np.uint32), ("lp", cap, np.uint32), ("ln", cap, np.uint32),
                       ("oldln", cap, np.uint32), ("cp", cap, np.uint32), ("ci", n, np.uint32),
                       ("dsp", 3 * cap, np.float64), ("frp", cap, np.float64), ("odsp", 3 * cap, np.float64),
                       ("ofrp", cap, np.float64), ("fp", 3 * cap, np.float64), ("ti", 3 * cap, np.float64),
                       ("tj", 3 * cap, np.float64), ("dw", 3 * n, np.float64), ("fw", n, np.float64),
                       ("fi", 3 * n, np.float64), ("tq", 3 * n, np.float64), ("qi", 3 * n, np.float64)):
        H[k] = np.zeros(sz, dtype=dt_)
    gsa, csa, oa, wa = np.array(GS, dtype=np.uint32), np.array(CELL), np.array(ORIGIN), np.array(world)
    Pp = orc.P
    iall_g = iall_h = 1
    tot_g = tot_h = 0
    relists = 0
    for it in range(300):
        assert iall_g == iall_h
        if iall_g:
            relists += 1
            G["qi"].zero_()
            dem.compat.calcHash(G["pos"], G["ph"], GS, CELL, ORIGIN, n)
            dem.compat.RadixSort(G["ph"], G["tmp"], n, 32)
            dem.compat.findCellStart(G["ph"], G["cst"], n, ncell)
            dem.compat.neighborarray(G["pos"], G["ph"], G["cst"], GS, CELL, ORIGIN, maxppc, n, G["anei"], G["njgi"],
                                     G["njli"])
            tot_g = dem.compat.prefixsum(n, G["njgi"], G["sj"], G["osj"])
            dem.compat.pairlist(G["sj"], G["osj"], G["oldln"], G["anei"], G["njgi"], G["njli"], G["odsp"], G["ofrp"],
                                maxppc, maxcn, n, G["aref"], G["lp"], G["ln"], G["dsp"], G["frp"])
            H["qi"][:] = 0
            L.ref_calcHash(Pp(H["pos"]), Pp(H["h"]), Pp(gsa), Pp(csa), Pp(oa), n)
            L.ref_radix_sort(Pp(H["h"]), n, 32)
            L.ref_findCellStart(Pp(H["h"]), Pp(H["cst"]), n, ncell)
            L.ref_neighborarray(Pp(H["pos"]), Pp(H["h"]), Pp(H["cst"]), Pp(gsa), Pp(csa), Pp(oa), maxppc, n,
                                Pp(H["anei"]), Pp(H["njgi"]), Pp(H["njli"]))
            tot_h = L.ref_prefixsum(n, Pp(H["njgi"]), Pp(H["sj"]), Pp(H["osj"]))
            L.ref_pairlist(Pp(H["sj"]), Pp(H["osj"]), Pp(H["oldln"]), Pp(H["anei"]), Pp(H["njgi"]), Pp(H["njli"]),
                           Pp(H["odsp"]), Pp(H["ofrp"]), maxppc, maxcn, n, Pp(H["aref"]), Pp(H["lp"]), Pp(H["ln"]),
                           Pp(H["dsp"]), Pp(H["frp"]))
            assert tot_g == tot_h
        dem.compat.calculateforcepair(G["pos"], G["pdis"], G["angv"], G["rad"], G["rmass"], G["lp"], G["ln"],
                                      G["oldln"], G["dsp"], G["frp"], G["odsp"], G["ofrp"], dt, G["fp"], G["ti"],
                                      G["tj"], G["cp"], tot_g)
        dem.compat.sumallforcei(maxppc, n, G["njgi"], G["njli"], G["fp"], G["ti"], G["tj"], G["cp"], G["aref"],
                                G["fi"], G["tq"], G["ci"])
        dem.compat.calculateforceiw(world, G["pos"], G["pdis"], G["angv"], G["rad"], G["rmass"], dt, tot_g, n,
                                    G["dw"], G["fw"], G["fi"], G["tq"])
        iall_g, mz_g = dem.compat.updateposition(world, n, G["pos"], G["pdis"], G["angv"], G["rmass"], G["inert"],
                                                 G["fi"], G["tq"], G["qi"], dt)
        L.ref_calculateforcepair(Pp(H["pos"]), Pp(H["pdis"]), Pp(H["angv"]), Pp(rad), Pp(rmass), Pp(H["lp"]),
                                 Pp(H["ln"]), Pp(H["oldln"]), Pp(H["dsp"]), Pp(H["frp"]), Pp(H["odsp"]),
                                 Pp(H["ofrp"]), dt, Pp(H["fp"]), Pp(H["ti"]), Pp(H["tj"]), Pp(H["cp"]), tot_h)
        L.ref_sumallforcei(maxppc, n, Pp(H["njgi"]), Pp(H["njli"]), Pp(H["fp"]), Pp(H["ti"]), Pp(H["tj"]),
                           Pp(H["cp"]), Pp(H["aref"]), Pp(H["fi"]), Pp(H["tq"]), Pp(H["ci"]))
        L.ref_calculateforceiw(Pp(wa), Pp(H["pos"]), Pp(H["pdis"]), Pp(H["angv"]), Pp(rad), Pp(rmass), dt, tot_h, n,
                               Pp(H["dw"]), Pp(H["fw"]), Pp(H["fi"]), Pp(H["tq"]))
        mz = np.zeros(1)
        iall_h = L.ref_updateposition(Pp(wa), n, Pp(H["pos"]), Pp(H["pdis"]), Pp(H["angv"]), Pp(rmass), Pp(inert),
                                      Pp(H["fi"]), Pp(H["tq"]), Pp(H["qi"]), dt, Pp(mz))
    gp = host(G["pos"])
    rms = np.sqrt(np.mean((gp - H["pos"]) ** 2))
    assert rms < 1e-9, rms
    pc_g = dem.compat.outputporositycn(n, G["ci"], mz_g, world)
    assert pc_g == L.ref_outputporositycn(n, Pp(H["ci"]))
    assert pc_g > n   # the bed is in contact


def test_compat_kernels_match_reference_golden(setup):
    """calcHash, findCellStart and updateposition against the outputs of the
    reference's own kernels (tests/golden/ref_kernels.npz), bit for bit."""
    import pathlib
    dem, orc, torch = setup
    g = dict(np.load(pathlib.Path(__file__).resolve().parent / "golden" / "ref_kernels.npz"))
    pos = g["hash_pos"]
    n = pos.size // 3
    gs = tuple(int(x) for x in g["hash_grid"])
    ph = zeros(torch, 2 * n, np.uint32)
    dem.compat.calcHash(dev(torch, pos), ph, gs, (1.55, 1.55, 1.55), (-10.0, -10.0, 0.0), n)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(ph, np.uint32), g["hash_out"])
    srt, cst = g["cell_sorted"], g["cell_start"]
    gc = zeros(torch, cst.size, np.uint32)
    dem.compat.findCellStart(dev(torch, srt), gc, srt.size // 2, cst.size)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(gc, np.uint32), cst)
    tp, td, ta, tq = (dev(torch, g[k]) for k in ("upd_pos_in", "upd_pdis_in", "upd_angv_in", "upd_qi_in"))
    m = g["upd_rmass"]
    dem.compat.set_cutoff(1.0, 1.55)
    iall, mz = dem.compat.updateposition((20.0, 20.0, 40.0), m.size, tp, td, ta, dev(torch, m),
                                         dev(torch, g["upd_inert"]), dev(torch, g["upd_force"]),
                                         dev(torch, g["upd_torque"]), tq, float(g["upd_scalars"][0]))
    np.testing.assert_array_equal(host(tp), g["upd_pos_out"])
    np.testing.assert_array_equal(host(td), g["upd_pdis_out"])
    np.testing.assert_array_equal(host(ta), g["upd_angv_out"])
    np.testing.assert_array_equal(host(tq), g["upd_qi_out"])
    assert iall == int(g["upd_part_iall"].max())
    assert mz == max(0.0, float(g["upd_part_maxhz"].max()))
