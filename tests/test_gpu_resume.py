"""Checkpoint / resume of the context API (dem_save_state / dem_load_state)
on the GPU: a context loaded from a state saved at a re-list boundary steps
on exactly as the saved context does -- positions, displacements, rotations,
the carried tangential history and the observables, bit for bit -- in both
force modes and both precisions, on a bed with live contacts."""
import numpy as np
import pytest

from _cases import dense_lattice

pytestmark = pytest.mark.gpu


def _engine(dem, w, prec, mode):
    e = dem.Engine(**{**w.engine_kwargs(), "precision": prec, "force_mode": mode})
    e.set_material(w.pp, w.pw)
    return e


@pytest.mark.parametrize("prec,mode", [("mixed", "pccp"), ("fp64", "pccp"), ("mixed", "pp"), ("fp64", "pp")])
def test_resume_is_bit_exact(dem, wl, cuda, tmp_path, prec, mode):
    p = dem.PREC_MIXED if prec == "mixed" else dem.PREC_FP64
    m = dem.FORCE_PCCP if mode == "pccp" else dem.FORCE_PP
    w = dense_lattice(dem, nx=8, ny=8, nz=6)
    rng = np.random.default_rng(9)
    pdis = rng.normal(0, 2e-6, 3 * w.n)
    K = w.relist_interval
    a = _engine(dem, w, p, m)
    a.upload(w.pos, w.rad, pdis, None)
    a.step(2 * K)
    path = tmp_path / "state.bin"
    a.save_state(path)
    saved = a.pairs()
    a.step(3 * K + 7)                      # whole windows and a partial one
    b = _engine(dem, w, p, m)
    b.load_state(path)
    assert b.scalars()["step"] == 2 * K
    for x, y in zip(saved, b.pairs()):     # the list and its history as saved
        np.testing.assert_array_equal(x, y)
    b.step(3 * K + 7)
    sa, sb = a.scalars(), b.scalars()
    assert sa["status"] == sb["status"] == 0, (sa["status"], sb["status"])
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)
    for k in ("step", "relists", "pairs", "contacts", "maxhz", "packing_fraction"):
        assert sa[k] == sb[k], k
    assert sa["contacts"] > 100            # the carried history mattered
    la, lna, ha = a.pairs()
    lb, lnb, hb = b.pairs()
    np.testing.assert_array_equal(la, lb)
    np.testing.assert_array_equal(ha, hb)


def test_save_and_load_errors(dem, wl, cuda, tmp_path):
    w = wl.small_box(n=2000)
    a = _engine(dem, w, dem.PREC_MIXED, dem.FORCE_PCCP)
    a.upload(w.pos, w.rad)
    a.step(5)
    with pytest.raises(dem.DemError) as e:          # inside a window
        a.save_state(tmp_path / "x.bin")
    assert e.value.code == dem.DEM_ERR_STATE
    a.step(w.relist_interval - 5)
    a.save_state(tmp_path / "x.bin")
    other = wl.small_box(n=1000)
    b = _engine(dem, other, dem.PREC_MIXED, dem.FORCE_PCCP)
    with pytest.raises(dem.DemError) as e:          # another n
        b.load_state(tmp_path / "x.bin")
    assert e.value.code == dem.DEM_ERR_ARG
    (tmp_path / "junk.bin").write_bytes(b"not a state file at all")
    with pytest.raises(dem.DemError) as e:
        a.load_state(tmp_path / "junk.bin")
    assert e.value.code == dem.DEM_ERR_IO
    # a pair list whose first partner is not above its row: refused before
    # anything reaches the device.  Layout after the header: pos, pdis, angv
    # (3n doubles each), rad (n doubles), q (n x 16 B), wall history (3n
    # doubles), offsets (n+1 uint32), partners (P uint32), history (3P doubles).
    n = w.n
    P = a.scalars()["pairs"]
    assert P > 0
    raw = bytearray((tmp_path / "x.bin").read_bytes())
    head = 13 * n * 8 + 16 * n + 4 * (n + 1)     # the sections before the partners
    ln0 = len(raw) - (head + 28 * P) + head
    raw[ln0:ln0 + 4] = (0).to_bytes(4, "little")
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    with pytest.raises(dem.DemError) as e:
        a.load_state(tmp_path / "bad.bin")
    assert e.value.code == dem.DEM_ERR_IO
