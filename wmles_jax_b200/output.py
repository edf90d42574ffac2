"""Output fields on the device (derived_fields, wmles/io_vtk.py:269-293).

``derived_fields(solver, Q)`` returns, like the reference, ``{block index: {name: array}}``
with rho, velocity (3, ni, nj, nk), pressure, temperature, mach, mu_t, mu, vorticity_mag
and q_criterion on the interior cells; the fields are computed by ``wm_derived_fields`` on
the device from the state with its ghost cells filled (``Solver.apply_bcs``), so only the
output fields leave the GPU (``as_numpy=False`` keeps them there as torch tensors).
"""
import torch

from . import _native as N

NAMES = ("rho", "u", "v", "w", "pressure", "temperature", "mach", "mu_t", "mu", "vorticity_mag", "q_criterion")


def derived_fields(solver, Q, time=0.0, as_numpy=True):
    Qb = solver.apply_bcs(Q, time=time)
    outs = [torch.empty((N.NDERIVED,) + tuple(b.n), dtype=torch.float64, device=solver.device)
            for b in solver.blocks]
    N.check(solver._lib.wm_derived_fields(solver._case, solver._ptrs(Qb), solver._ptrs(outs), solver._stream()),
            "wm_derived_fields")
    result = {}
    for ib, o in enumerate(outs):
        f = dict(zip(NAMES, o))
        d = {"rho": f["rho"], "velocity": torch.stack([f["u"], f["v"], f["w"]]), "pressure": f["pressure"],
             "temperature": f["temperature"], "mach": f["mach"], "mu_t": f["mu_t"], "mu": f["mu"],
             "vorticity_mag": f["vorticity_mag"], "q_criterion": f["q_criterion"]}
        result[ib] = {k: v.cpu().numpy() for k, v in d.items()} if as_numpy else d
    return result
