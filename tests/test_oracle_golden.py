"""The CPU oracle against golden vectors produced by the reference's own
kernels (neiglist.cu compiled in place and run on a GPU; see
tests/golden/make_ref_golden.py and oracle/ref_harness/ref_golden.cu).

Pins: calcHashD (incl. its unsigned clamp of negative cell coordinates),
findCellStartD, addTwoArraysD (the inclusive step of prefixsum),
updatepositionD (integrator, re-list flag, max height), vprojec (both
modes), vscale, and the gravity/history bookkeeping of calculateforceiwD and
calculateforcepairD when nothing touches.
"""
import pathlib

import numpy as np
import pytest

GOLD = pathlib.Path(__file__).resolve().parent / "golden" / "ref_kernels.npz"


@pytest.fixture(scope="module")
def g():
    if not GOLD.exists():
        pytest.fail(f"missing {GOLD}")
    return dict(np.load(GOLD))


def test_calc_hash_matches_reference(orc, g):
    pos, out, gs = g["hash_pos"], g["hash_out"], g["hash_grid"].astype(np.uint32)
    n = pos.size // 3
    ref = np.empty(2 * n, dtype=np.uint32)
    orc.lib().ref_calcHash(orc.P(pos), orc.P(ref), orc.P(gs), orc.P(np.array([1.55] * 3)),
                           orc.P(np.array([-10.0, -10.0, 0.0])), n)
    np.testing.assert_array_equal(ref, out)
    # the reference maps a negative cell coordinate to the last cell
    p = pos.reshape(-1, 3)
    below = np.nonzero(p[:, 0] < -10.0)[0]
    assert below.size > 0
    assert np.all(out[2 * below] % gs[0] == gs[0] - 1)


def test_find_cell_start_matches_reference(orc, g):
    srt, cst = g["cell_sorted"], g["cell_start"]
    n = srt.size // 2
    ref = np.empty(cst.size, dtype=np.uint32)
    orc.lib().ref_findCellStart(orc.P(srt), orc.P(ref), n, cst.size)
    np.testing.assert_array_equal(ref, cst)


def test_inclusive_scan_step_matches_reference(orc, g):
    a, b, out = g["add_a"], g["add_b"], g["add_out"]
    np.testing.assert_array_equal((b + a).astype(np.uint32), out)
    # and the oracle's prefixsum is exclusive-scan + that step
    n = a.size
    sj = np.zeros(n, dtype=np.uint32)
    osj = np.zeros(n, dtype=np.uint32)
    tot = orc.lib().ref_prefixsum(n, orc.P(a), orc.P(sj), orc.P(osj))
    np.testing.assert_array_equal(sj, np.cumsum(a, dtype=np.uint64).astype(np.uint32))
    assert tot == int(a.sum())


def test_updateposition_matches_reference(orc, g):
    pos, pdis, angv, qi = (g[k].copy() for k in ("upd_pos_in", "upd_pdis_in", "upd_angv_in", "upd_qi_in"))
    F, T, m, I = g["upd_force"], g["upd_torque"], g["upd_rmass"], g["upd_inert"]
    dt = float(g["upd_scalars"][0])
    n = m.size
    orc.lib().ref_set_cutoff(1.0, 1.55)
    mz = np.zeros(1)
    iall = orc.lib().ref_updateposition(orc.P(np.array([20.0, 20.0, 40.0])), n, orc.P(pos), orc.P(pdis),
                                        orc.P(angv), orc.P(m), orc.P(I), orc.P(F), orc.P(T), orc.P(qi), dt,
                                        orc.P(mz))
    # bit-exact: every operation is a correctly rounded mul/div/add on both sides
    np.testing.assert_array_equal(pos, g["upd_pos_out"])
    np.testing.assert_array_equal(pdis, g["upd_pdis_out"])
    np.testing.assert_array_equal(angv, g["upd_angv_out"])
    np.testing.assert_array_equal(qi, g["upd_qi_out"])
    assert iall == int(g["upd_part_iall"].max())
    # per-block partials of the reference: re-list flag from the single-precision
    # length (|q| > 0.5*(cub-cua)) and the block maximum height
    q = g["upd_qi_out"].reshape(-1, 3)
    rmov = np.sqrt((q * q).sum(1).astype(np.float32)).astype(np.float64)
    flag = rmov > 0.275
    z = g["upd_pos_out"][2::3]
    for b, (pi, pm) in enumerate(zip(g["upd_part_iall"], g["upd_part_maxhz"])):
        sl = slice(256 * b, min(256 * (b + 1), n))
        assert int(flag[sl].any()) == int(pi)
        assert max(z[sl].max(), 0.0 if (b + 1) * 256 > n else -np.inf) == pm
    assert mz[0] == max(0.0, float(g["upd_part_maxhz"].max()))


def test_vprojec_and_vscale_match_reference(orc, g):
    p, u = g["vp_p"].reshape(-1, 3), g["vp_u"].reshape(-1, 3)
    r0, r1 = g["vp_r0"].reshape(-1, 3), g["vp_r1"].reshape(-1, 3)
    L = orc.lib()
    for k in range(p.shape[0]):
        a = np.zeros(3)
        b = np.zeros(3)
        L.ref_vprojec(orc.P(np.ascontiguousarray(p[k])), orc.P(np.ascontiguousarray(u[k])), orc.P(a), 0)
        L.ref_vprojec(orc.P(np.ascontiguousarray(p[k])), orc.P(np.ascontiguousarray(u[k])), orc.P(b), 1)
        # the GPU fuses the cross products' multiply-adds; agreement to a few ulps
        tol0 = 1e-14 * max(np.abs(p[k]).max(), 1e-300)
        assert np.abs(a - r0[k]).max() <= tol0
        assert np.abs(b - r1[k]).max() <= 1e-6 * max(np.abs(r1[k]).max(), 1e-300) + tol0
    v, s1, s2, vo = g["vs_in"].reshape(-1, 3), g["vs_p1"], g["vs_p2"], g["vs_out"].reshape(-1, 3)
    for k in range(v.shape[0]):
        a = np.ascontiguousarray(v[k]).copy()
        L.ref_vscale(orc.P(a), float(s1[k]), float(s2[k]))
        np.testing.assert_array_equal(a, vo[k])


@pytest.mark.parametrize("total", [0, 7])
def test_wall_gravity_bookkeeping_matches_reference(orc, g, total):
    """calculateforceiwD with no wall touched: force = (pair sum if total != 0)
    + (0,0,-m), torque likewise, wall history cleared."""
    keys = ("wall_pos", "wall_pdis", "wall_angv", "wall_rad", "wall_rmass")
    pos, pdis, angv, rad, m = (g[k] for k in keys)
    F, T = g["wall_force_in"].copy(), g["wall_torque_in"].copy()
    dw, fw = g["wall_disptw_in"].copy(), g["wall_fricpw_in"].copy()
    n = rad.size
    orc.lib().ref_calculateforceiw(orc.P(np.array([20.0, 20.0, 40.0])), orc.P(pos), orc.P(pdis), orc.P(angv),
                                   orc.P(rad), orc.P(m), 1e-3, total, n, orc.P(dw), orc.P(fw), orc.P(F), orc.P(T))
    s = f"_t{total}"
    np.testing.assert_array_equal(F, g["wall_force_out" + s])
    np.testing.assert_array_equal(T, g["wall_torque_out" + s])
    np.testing.assert_array_equal(dw, g["wall_disptw_out" + s])
    np.testing.assert_array_equal(fw, g["wall_fricpw_out" + s])


def test_pair_bookkeeping_matches_reference(orc, g):
    """calculateforcepairD when no listed pair touches: outputs zeroed, old
    list slot records j (neiglist.cu:211-231)."""
    lp, ln = g["pair_lp"], g["pair_ln"]
    P = lp.size
    pos = g["pair_pos"]
    n = pos.size // 3
    rad = np.full(n, 0.5)
    rmass = np.ones(n)
    z3 = np.zeros(3 * n)
    dsp, frp = g["pair_dispt_in"].copy(), g["pair_fricp_in"].copy()
    oldln = np.full(P, 12345, dtype=np.uint32)
    odsp = np.full(3 * P, 9.0)
    ofrp = np.full(P, 9.0)
    fp = np.full(3 * P, 9.0)
    ti = np.full(3 * P, 9.0)
    tj = np.full(3 * P, 9.0)
    cp = np.full(P, 7, dtype=np.uint32)
    orc.lib().ref_set_material(orc.P(np.array([5e5, 0.3, 0.29, 0.2, 0.2, 0.0])),
                               orc.P(np.array([5e5, 0.3, 0.29, 0.2, 0.2, 0.0])))
    orc.lib().ref_calculateforcepair(orc.P(pos), orc.P(z3), orc.P(z3), orc.P(rad), orc.P(rmass), orc.P(lp),
                                     orc.P(ln), orc.P(oldln), orc.P(dsp), orc.P(frp), orc.P(odsp), orc.P(ofrp), 1e-3,
                                     orc.P(fp), orc.P(ti), orc.P(tj), orc.P(cp), P)
    for mine, key in ((dsp, "pair_dispt_out"), (frp, "pair_fricp_out"), (odsp, "pair_olddispt_out"),
                      (ofrp, "pair_oldfricp_out"), (fp, "pair_force_out"), (ti, "pair_tpi_out"),
                      (tj, "pair_tpj_out"), (oldln, "pair_oldln_out"), (cp, "pair_contact_out")):
        np.testing.assert_array_equal(mine, g[key])
