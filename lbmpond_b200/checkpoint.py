"""Checkpoint and resume of a Solver: everything the next step reads, in one .npz.

The reference has no restart file: drop() (drop.cu:2-34) writes rho, u and T
as .arr files but not the populations, so a run cannot be continued from
them.  A checkpoint holds the context's parameters, the step counter,
simulated time and dt (LBMParamsHost iStep / curtime / dt), the populations,
density and gauge of the current time level, the energy populations of a
context with them, and the node mask and positions of a 1D mesh context.  A
plain step reads only the current time level, so a resumed context continues
the run exactly (a float32 context's values are exact in float64).

Not stored: a bound predictor of the learned start (attach it again after
resuming), the time-step adaptation policy, and kept histories.
"""
from __future__ import annotations

import numpy as np

FORMAT = 1
# pond_params fields a checkpoint restores (bc is stored beside them)
PARAM_KEYS = ("lattice", "interp", "precision", "tau", "dt", "tol_abs", "tol_rel", "max_iter", "ddf", "ddf_dof")
MESH_SCHEMES = (9, 10)  # POND_GAP2, POND_NONUNIFORM3
NONUNIFORM3 = 10


def state_dict(solver) -> dict:
    """The solver's checkpoint as a dict of numpy values."""
    p = solver.get_params()
    d = {"format": FORMAT, "shape": np.array(solver.shape, dtype=np.int64),
         "bc": np.array([int(p.bc[a]) for a in range(3)], dtype=np.int32)}
    for k in PARAM_KEYS:
        d[k] = getattr(p, k)
    diag = solver.diagnostics()
    d["istep"], d["curtime"] = int(diag["istep"]), float(diag["curtime"])
    d["f"], d["rho"], d["g"] = solver.get_state()
    if p.ddf:
        d["h"] = solver.get_energy()
    if p.interp in MESH_SCHEMES:
        d["mask"] = solver.get_mask()
        if p.interp == NONUNIFORM3:
            d["positions"] = solver.get_positions()
    return d


def write(path: str, d: dict) -> None:
    with open(path, "wb") as fp:
        np.savez_compressed(fp, **{k: np.asarray(v) for k, v in d.items()})


def read(path: str) -> dict:
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    if int(d.get("format", -1)) != FORMAT:
        raise ValueError(f"{path}: not a checkpoint of format {FORMAT}")
    return d


def solver_kwargs(d: dict, device: int = 0) -> dict:
    """Solver(...) arguments that recreate the checkpointed context."""
    kw = dict(lattice=int(d["lattice"]), shape=tuple(int(v) for v in d["shape"]), interp=int(d["interp"]),
              precision=int(d["precision"]), tau=float(d["tau"]), tol_abs=float(d["tol_abs"]),
              tol_rel=float(d["tol_rel"]), max_iter=int(d["max_iter"]), bc=tuple(int(v) for v in d["bc"]),
              device=device, dt=float(d["dt"]))
    if int(d["ddf"]):
        kw["ddf_dof"] = int(d["ddf_dof"])
    return kw


def restore(solver, d: dict) -> None:
    """Load a checkpoint's state into a context made with solver_kwargs(d)."""
    solver.set_state(d["rho"], d["g"], f=d["f"])
    if "h" in d:
        solver.set_energy(d["h"])
    if "mask" in d:
        solver.set_mask(d["mask"])
    if "positions" in d:
        solver.set_positions(d["positions"])
    solver.set_clock(int(d["istep"]), float(d["curtime"]), float(d["dt"]))


def save(solver, path: str) -> None:
    write(path, state_dict(solver))


def load(path: str, device: int = 0):
    """A new Solver continuing the checkpointed run."""
    from . import Solver
    d = read(path)
    s = Solver(**solver_kwargs(d, device))
    try:
        restore(s, d)
    except Exception:
        s.close()
        raise
    return s
