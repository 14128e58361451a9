"""bench.py's byte model, launch count and profile lookups, on the CPU: the
algorithmic bytes the bench line's roofline divides by, the kernels it
claims per window, and the DRAM traffic it reads from the committed ncu
summaries (profiles/)."""
import importlib.util
import pathlib

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_model_mod", ROOT / "bench.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_window_bytes_follow_the_byte_model():
    b = _bench()
    n, win, bp, ncells = 1000, 20, b.BYTES_PER_PARTICLE["mixed"], 50
    work = {"bound": 100, "pairs": 40}
    kernel, relist = b.window_bytes(n, work, win, bp, ncells)
    # bound spheres and pairs every step, free spheres once per window
    assert kernel == win * (100 * 172 + 40 * 56) + (n - 100) * 172
    assert relist == n * (24 + 8 + 16 + 4) + 8 * ncells + 64 * 40


def test_launches_per_window():
    b = _bench()
    # batched: outer check, candidate pass, fill, reverse rows, component
    # pass; exiting window kernel, batches, free particles
    assert b.launches_per_window({"batched": 1}) == 8
    assert b.launches_per_window({"batched": 0}) == 8
    # not batching: the four re-list kernels and the window kernel
    assert b.launches_per_window({"batched": -1}) == 5


def test_roofline_fraction():
    b = _bench()
    r = b.roofline("k_batch", 2e8, 0.05, 6000.0, "measured", "rsa_500k", traffic=2.66e7)
    assert abs(r["achieved"] - 4000.0) < 1e-9 and abs(r["frac"] - 4000.0 / 6000.0) < 1e-12
    assert r["traffic"] == 2.66e7 and r["bound"] == "hbm" and r["unit"] == "GB/s"


def test_committed_profiles_carry_the_traffic_the_bench_reads():
    b = _bench()
    for name in ("k_batch_rsa500k_mixed", "k_window_bed500k_mixed"):
        t = b.profile_traffic(name)
        assert t is not None and t > 1e6, name
    assert b.profile_traffic("no_such_profile") is None
