"""Test-only initial states with sustained contacts."""
import numpy as np


def dense_lattice(dem, nx=14, ny=14, nz=12, spacing=0.999, rmin=0.4985, rmax=0.5005, seed=7, precision=None):
    """Polydisperse spheres on a cubic lattice of spacing 0.999 d, radii
    uniform in [rmin, rmax] (FP32-representable), resting on the floor and
    pressed lightly against the side walls: overlaps <= 0.002 d, so contacts
    persist and stay gentle for hundreds of steps."""
    import dem_b200.workloads as w
    rng = np.random.default_rng(seed)
    gx = (np.arange(nx) - 0.5 * (nx - 1)) * spacing
    gy = (np.arange(ny) - 0.5 * (ny - 1)) * spacing
    gz = np.arange(nz) * spacing
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    n = X.size
    rad = rng.uniform(rmin, rmax, n).astype(np.float32).astype(np.float64)
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel() + rad], 1)
    world = (nx * spacing - 0.0004, ny * spacing - 0.0004, nz * spacing + 20.0)
    pp, pw = w.material(mu=0.3, roll_rel=0.002)
    prec = dem.PREC_FP64 if precision is None else precision
    return w.Workload("dense_lattice", n, pos.reshape(-1).copy(), rad, world, w.reduced_dt(5e-7), 200, 20, 0.05,
                      prec, pp, pw)
