"""The beta0 checkpoint on disk (``src/io/run_output.jl:13-40``), on the CPU.

A purified checkpoint saved and loaded again gives ``run_stochastic`` the same
result as the checkpoint in memory (``run_stochastic(c; checkpoint_path)``,
``src/driver/run.jl:79-87``); loading checks the format and the model,
lattice and beta0 against the configuration with the reference's messages,
and an existing file is only replaced on request.  The oracle supplies the
numerical ops.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_parallel import OracleOps, _config   # noqa: E402


def test_checkpoint_round_trip_gives_the_same_run(sps, tmp_path):
    c = _config(sps)
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    path = str(tmp_path / "checkpoint.npz")
    sps.save_checkpoint(path, cp, ops=ops)
    loaded = sps.load_checkpoint(path, c, ops=ops)
    assert loaded.run_id == cp.run_id
    assert loaded.purification == [dict(r) for r in loaded.purification]
    a = sps.run_stochastic(c, cp, ops=ops)
    b = sps.run_stochastic(c, ops=ops, checkpoint_path=path)
    for ra, rb in zip(a["observables"]["curve"], b["observables"]["curve"]):
        for k in ("beta", "lnZ", "energy_per_site", "eta"):
            x, y = ra[k], rb[k]
            assert (np.isnan(x) and np.isnan(y)) or x == y, (k, x, y)
    np.testing.assert_array_equal(np.stack([d["configuration"] for d in a["diagnostics"]["born_draws"]]),
                                  np.stack([d["configuration"] for d in b["diagnostics"]["born_draws"]]))


def test_checkpoint_checks(sps, tmp_path):
    c = _config(sps)
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    path = str(tmp_path / "checkpoint.npz")
    sps.save_checkpoint(path, cp, ops=ops)
    with pytest.raises(FileExistsError):
        sps.save_checkpoint(path, cp, ops=ops)
    sps.save_checkpoint(path, cp, ops=ops, overwrite=True)
    import dataclasses
    other = dataclasses.replace(c, beta0=c.beta0 + 0.05, beta_log=[0.15, 0.2], beta_measure=[0.15, 0.2])
    with pytest.raises(ValueError, match="checkpoint model, lattice or beta0 mismatch"):
        sps.load_checkpoint(path, other, ops=ops)
    bad = str(tmp_path / "bad.npz")
    np.savez(bad, data=np.zeros(1), dims=np.zeros(1, np.int32), meta=np.array('{"format": "other"}'))
    with pytest.raises(ValueError, match="unsupported checkpoint format"):
        sps.load_checkpoint(bad, c, ops=ops)
    with pytest.raises(ValueError, match="supply a checkpoint"):
        sps.run_stochastic(c, ops=ops)


def test_result_record_round_trip(sps, tmp_path):
    """``save_result`` / ``load_result`` (``src/io/results.jl:21-80``): the run record
    comes back with the schema version and the same curve; without ``overwrite``
    an existing file is kept; the extension is checked."""
    import math
    c = _config(sps)
    ops = OracleOps(c)
    res = sps.run_stochastic(c, sps.run_purification(c, ops=ops, identity=ops.identity), ops=ops)
    path = str(tmp_path / "run" / "result.json")
    dest = sps.save_run_result(path, res)
    back = sps.load_result(dest)
    assert back["schema_version"] == sps.RESULT_SCHEMA_VERSION == "2.7.0"
    assert back["method"] == "stoPEPS" and "created_at" in back
    for a, b in zip(res["observables"]["curve"], back["observables"]["curve"]):
        for k in ("beta", "lnZ", "energy_per_site", "eta"):
            assert (math.isnan(a[k]) and math.isnan(b[k])) or a[k] == b[k]
    draws = back["diagnostics"]["born_draws"]
    np.testing.assert_array_equal(np.asarray(draws[0]["configuration"]),
                                  res["diagnostics"]["born_draws"][0]["configuration"])
    with pytest.raises(FileExistsError):
        sps.save_run_result(path, res, overwrite=False)
    with pytest.raises(ValueError, match="extension"):
        sps.save_run_result(str(tmp_path / "result.jld2"), res)
