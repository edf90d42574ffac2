"""Checkpoint and restart of a device state without pyvista (read_restart,
wmles/io_vtk.py:118-193, returns (Q, step, time) the same way).

``write_restart(path, solver, Q, step, time)`` copies every block's state (ghost cells
included) to the host once and stores it in one ``.npz`` with the step, the time and each
block's name and interior extent; ``read_restart(path, solver)`` checks that the file
matches the solver's blocks and returns the state on the solver's device.  A server can use
the same pair to move a paused case out of device memory and back.
"""
import numpy as np
import torch

FORMAT = 1


def write_restart(path, solver, Q, step, time):
    blocks = solver.blocks
    if len(Q) != len(blocks):
        raise ValueError(f"state has {len(Q)} blocks, solver has {len(blocks)}")
    arrays = {"format": np.array(FORMAT), "step": np.array(int(step)), "time": np.array(float(time)),
              "names": np.array([b.name for b in blocks]), "extents": np.array([list(b.n) for b in blocks])}
    for ib, q in enumerate(Q):
        arrays[f"q{ib}"] = q.detach().cpu().numpy() if isinstance(q, torch.Tensor) else np.asarray(q)
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def read_restart(path, solver):
    with np.load(path) as d:
        if int(d["format"]) != FORMAT:
            raise ValueError(f"{path}: restart format {int(d['format'])}, expected {FORMAT}")
        names, extents = list(d["names"]), d["extents"].tolist()
        want = [b.name for b in solver.blocks]
        if names != want or extents != [list(b.n) for b in solver.blocks]:
            raise ValueError(f"{path}: restart holds blocks {list(zip(names, extents))}, solver expects "
                             f"{[(b.name, list(b.n)) for b in solver.blocks]}")
        Q = tuple(torch.from_numpy(np.ascontiguousarray(d[f"q{ib}"])).to(solver.device) for ib in range(len(want)))
        for q, b in zip(Q, solver.blocks):
            if tuple(q.shape) != (5,) + tuple(b.N):
                raise ValueError(f"{path}: block {b.name} state shape {tuple(q.shape)}")
        return Q, int(d["step"]), float(d["time"])
