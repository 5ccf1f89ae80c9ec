"""Configuration stamp of a solver, written into checkpoints.

A checkpoint may only be restored into a solver whose time step computes the
same thing.  The stamp therefore records every input of the step: the lattice
and the geometry tables (hashed), the per-id boundary kinds, value modes and
parameters, every material parameter and the Jacobian floor, the collision,
source and closure settings, and the displacement-sweep and F-repair
schedule.  Floats are written with ``repr`` precision, so any change of a
setting changes the stamp.
"""

from __future__ import annotations

import hashlib
import json

import numpy as np

# solver attributes that decide what a step computes (those a class lacks are skipped)
_SETTINGS = (
    "nx", "ny", "nz", "n_active", "dx", "dy", "dz", "dt", "lattice_speed", "collision_omega",
    "collision_model", "ghost_omega", "kinetic_filter_strength",
    "boundary_reconstruction_name", "normal_jacobian_name",
    "neumann_solver_name", "jacobian_floor", "source_mode",
    "local_displacement_interval", "local_displacement_sweeps", "local_displacement_relax",
    "local_displacement_boundary_weight", "local_displacement_boundary_id",
    "local_compatibility_interval", "local_compatibility_blend",
    "local_compatibility_interior_only", "use_dynamic_link_traction",
)


def _plain(v):
    if isinstance(v, np.ndarray):
        return [_plain(x) for x in v.tolist()]
    if isinstance(v, (list, tuple)):
        return [_plain(x) for x in v]
    if isinstance(v, (np.integer,)):
        return int(v)
    if isinstance(v, (np.floating, float)):
        return repr(float(v))
    if isinstance(v, (bool, np.bool_)):
        return bool(v)
    return v


def tables_digest(arrays) -> str:
    """sha256 over the bytes, dtypes and shapes of the given host arrays."""
    h = hashlib.sha256()
    for a in arrays:
        if a is None:
            h.update(b"none")
            continue
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def config_stamp(solver, *, geometry_arrays, boundary_tables, extra=None) -> str:
    """JSON stamp of `solver`'s step configuration (see the module docstring)."""
    m = solver.material
    out = {name: _plain(getattr(solver, name)) for name in _SETTINGS if hasattr(solver, name)}
    out["source_params"] = _plain(np.asarray(solver.source_params, dtype=np.float64))
    out["material"] = {"model": str(m.model),
                       **{k: _plain(getattr(m, k)) for k in ("lam", "mu", "param0", "param1",
                                                             "param2") if hasattr(m, k)}}
    kind, mode, params = boundary_tables
    out["boundary"] = {"kind": _plain(np.asarray(kind)), "mode": _plain(np.asarray(mode)),
                       "params": _plain(np.asarray(params, dtype=np.float64))}
    out["geometry"] = tables_digest(geometry_arrays)
    if extra:
        out.update({k: _plain(v) for k, v in extra.items()})
    return json.dumps(out, sort_keys=True)
