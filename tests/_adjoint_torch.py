"""Test harness only: the DEM window with its adjoint (dem_adjoint_window
through the C ABI) as a torch.autograd.Function of the physical parameters.

    value = DemWindow.apply(E, e, mu, mu_r, rad, setup)

E (Young's modulus, Pa), e (restitution), mu (sliding friction), mu_r
(rolling friction, relative to R*) and rad (every radius, reduced units) are
0-d / 1-d float64 tensors; `setup` carries the bed (positions, initial
motion, the workload's box and time step), the window (steps, checkpoint
interval) and the objective.  The contact parameters follow the workloads'
material map (estar from E, viscous damping from e, the same values for
particle-particle and particle-wall contacts); backward maps the adjoint's
gradients with respect to those parameters back through that map (the two
scalar maps are differentiated by central differences, which are exact to
far below the tests' tolerance)."""
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class WindowSetup:
    dem: object
    wl: object              # the workloads module (material map)
    w: object               # Workload: box, dt, skin, relist interval, density
    pos: np.ndarray
    pdis: np.ndarray
    angv: np.ndarray
    steps: int
    every: int
    objective: int
    precision: int
    cell: float


def _contacts(s: WindowSetup, E, e, mu, mu_r):
    return s.wl.material(E=E, mu=mu, roll_rel=mu_r, e=e)


def _run(s: WindowSetup, E, e, mu, mu_r, rad):
    pp, pw = _contacts(s, E, e, mu, mu_r)
    x = s.dem.Engine(**{**s.w.engine_kwargs(), "precision": s.precision, "cell": s.cell})
    x.set_material(pp, pw)
    x.upload(s.pos, rad, s.pdis, s.angv)
    r = x.adjoint(s.steps, s.every, s.objective)
    assert x.scalars()["status"] == 0
    x.close()
    return r


def window_value(s: WindowSetup, E, e, mu, mu_r, rad):
    """The objective alone (for finite differences)."""
    return _run(s, E, e, mu, mu_r, rad)["value"]


class DemWindow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, e, mu, mu_r, rad, s: WindowSetup):
        Ev, ev, muv, mrv = float(E), float(e), float(mu), float(mu_r)
        r = _run(s, Ev, ev, muv, mrv, rad.detach().cpu().numpy().astype(np.float64))
        dpp, dpw = r["d_pp"], r["d_pw"]
        # estar and the damping depend on E and e only: their map, differentiated
        hE, he = 1e-6 * Ev, 1e-7
        es_p = _contacts(s, Ev + hE, ev, muv, mrv)[0]["estar"]
        es_m = _contacts(s, Ev - hE, ev, muv, mrv)[0]["estar"]
        c_p = _contacts(s, Ev, ev + he, muv, mrv)[0]["damp_n"]
        c_m = _contacts(s, Ev, ev - he, muv, mrv)[0]["damp_n"]
        dE = (dpp["estar"] + dpw["estar"]) * (es_p - es_m) / (2 * hE)
        de = (dpp["damp_n"] + dpp["damp_t"] + dpw["damp_n"] + dpw["damp_t"]) * (c_p - c_m) / (2 * he)
        dmu = dpp["mu"] + dpw["mu"]
        dmr = dpp["roll_rel"] + dpw["roll_rel"]
        grads = torch.tensor([dE, de, dmu, dmr], dtype=torch.float64)
        ctx.save_for_backward(grads, torch.from_numpy(r["d_radii"]).to(torch.float64))
        return torch.tensor(r["value"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        grads, drad = ctx.saved_tensors
        return g * grads[0], g * grads[1], g * grads[2], g * grads[3], g * drad, None
