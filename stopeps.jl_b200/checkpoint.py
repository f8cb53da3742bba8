"""The beta0 thermal checkpoint on disk: ``save_checkpoint`` / ``load_checkpoint``.

Restates ``src/io/run_output.jl:4-40``: the checkpoint holds the beta0 PEPO
(site tensors, beta0, log_amplitude), the preparation parameters, the
purification rows, the normalisation history and the run id; loading checks
the format, the model, the lattice, beta0 and the physical space against the
run configuration and fails with the reference's messages.  The reference
writes JLD2 through ``Results.save_result``; this engine writes the same fields
to one NumPy ``.npz`` file (site tensors as arrays in the sector-sorted dense
layout of the C ABI, the records as JSON), format ``CHECKPOINT_FORMAT``.  The
tensors go through the drivers' ops (``export_state`` / ``state_from``), so a
checkpoint moves between the device engine and any other ops.
"""
from __future__ import annotations

import json
import os

import numpy as np

from .config import RunConfig, parameter_dict, same_beta

CHECKPOINT_FORMAT = "stopeps-b200-thermal-npz-1.0.0"


def _jsonable(x):
    if isinstance(x, dict):
        return {str(k): _jsonable(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_jsonable(v) for v in x]
    if isinstance(x, np.ndarray):
        return _jsonable(x.tolist())
    if isinstance(x, (np.floating, np.integer, np.bool_)):
        return x.item()
    return x


def save_checkpoint(path, cp, ops=None, overwrite=False):
    """``save_checkpoint`` (``run_output.jl:13-21``); replacing an existing path needs ``overwrite``."""
    from .driver import DEVICE_OPS
    ops = ops or DEVICE_OPS
    if os.path.exists(path) and not overwrite:
        raise FileExistsError(f"{path} exists; pass overwrite=True to replace it")
    blob = ops.export_state(cp.state)
    sites = [np.asarray(a, np.float64) for a in blob["sites"]]
    meta = dict(format=CHECKPOINT_FORMAT, method="stoPEPS_checkpoint", preparation=_jsonable(cp.preparation),
                purification=_jsonable(cp.purification), history=_jsonable(cp.history), run_id=cp.run_id,
                beta0=float(blob["beta"]), log_amplitude=float(blob["log_amplitude"]),
                is_pepo=bool(blob["is_pepo"]))
    with open(path, "wb") as f:
        np.savez_compressed(f, data=np.concatenate([a.reshape(-1) for a in sites]) if sites else np.zeros(0),
                            dims=np.asarray(blob["dims"], np.int32), meta=np.array(json.dumps(meta)))


def load_checkpoint(path, c: RunConfig, ops=None):
    """``load_checkpoint`` (``run_output.jl:27-40``): the beta0 PEPO and its records,
    checked against ``c``."""
    from .driver import DEVICE_OPS, ThermalCheckpoint
    ops = ops or DEVICE_OPS
    with np.load(path, allow_pickle=False) as d:
        meta = json.loads(str(d["meta"]))
        data = np.asarray(d["data"])
        dims = np.asarray(d["dims"], np.int32)
    if meta.get("format") != CHECKPOINT_FORMAT:
        raise ValueError("unsupported checkpoint format")
    current = parameter_dict(c)
    prep = meta["preparation"]
    if not (prep.get("model") == _jsonable(current["model"]) and prep.get("lattice") == _jsonable(current["lattice"])
            and same_beta(meta["beta0"], c.beta0)):
        raise ValueError("checkpoint model, lattice or beta0 mismatch")
    L = c.lattice.Lx * c.lattice.Ly
    dims = dims.reshape(L, 6, 2)
    if any(tuple(dims[i, 2]) != (c.model.physical_space.n0, c.model.physical_space.n1) for i in range(L)):
        raise ValueError("checkpoint physical space mismatch")
    sites, off = [], 0
    for i in range(L):
        shape = [int(a + b) for a, b in dims[i]]
        n = int(np.prod(shape))
        sites.append(data[off:off + n].reshape(shape))
        off += n
    state = ops.state_from(dict(sites=sites, dims=dims, is_pepo=meta["is_pepo"], beta=meta["beta0"],
                                log_amplitude=meta["log_amplitude"]), c)
    return ThermalCheckpoint(state, dict(prep), list(meta["purification"]), list(meta["history"]), meta["run_id"])
