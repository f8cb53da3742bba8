"""Result records on disk: ``save_result`` / ``load_result``.

Restates ``src/io/results.jl:8-80`` (module ``Results``): a result is a
string-keyed record with ``schema_version`` (``RESULT_SCHEMA_VERSION``),
``created_at`` (UTC), ``method``, ``model``, ``parameters``, ``observables``,
``diagnostics`` and ``metadata``; it is written to a temporary file in the
destination directory and then renamed into place (or, without
``overwrite``, published by a hard link, failing if the destination exists).
The reference writes JLD2; this engine writes the same record as JSON (arrays
as nested lists, NaN as the token NaN), so the path must end in ``.json``.
"""
from __future__ import annotations

import datetime
import json
import os
import platform
import tempfile

import numpy as np

from .driver import RESULT_SCHEMA_VERSION


def _plain(x):
    if isinstance(x, dict):
        return {str(k): _plain(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_plain(v) for v in x]
    if isinstance(x, np.ndarray):
        return _plain(x.tolist())
    if isinstance(x, (np.floating, np.integer, np.bool_)):
        return x.item()
    return x


def save_result(path, *, method, model, observables, parameters=None, diagnostics=None, metadata=None,
                overwrite=True):
    """``save_result`` (``results.jl:21-74``); returns the absolute destination."""
    if not str(path).lower().endswith(".json"):
        raise ValueError("result path must use the .json extension")
    destination = os.path.abspath(path)
    if not overwrite and (os.path.exists(destination) or os.path.islink(destination)):
        raise FileExistsError(f"output exists: {destination}; use overwrite=True to replace it")
    directory = os.path.dirname(destination)
    os.makedirs(directory, exist_ok=True)
    record = dict(schema_version=RESULT_SCHEMA_VERSION,
                  created_at=datetime.datetime.now(datetime.timezone.utc).isoformat(),
                  method=str(method), model=_plain(model), parameters=_plain(parameters or {}),
                  observables=_plain(observables), diagnostics=_plain(diagnostics or {}),
                  metadata=dict({"python_version": platform.python_version()}, **_plain(metadata or {})))
    fd, temporary = tempfile.mkstemp(dir=directory, suffix=".tmp")
    try:
        with os.fdopen(fd, "w") as f:
            json.dump(record, f)
        if overwrite:
            os.replace(temporary, destination)
        else:
            os.link(temporary, destination)
            os.remove(temporary)
    except BaseException:
        if os.path.exists(temporary):
            os.remove(temporary)
        raise
    return destination


def load_result(path) -> dict:
    """``load_result`` (``results.jl:76-80``): the record as a string-keyed dict."""
    with open(path) as f:
        return json.load(f)


def save_run_result(path, result: dict, overwrite=True):
    """A ``run_stochastic`` record (schema 2.7.0) through ``save_result``."""
    return save_result(path, method=result["method"], model=result.get("model", {}),
                       parameters=result.get("parameters"), observables=result["observables"],
                       diagnostics=result.get("diagnostics"), metadata=result.get("metadata"),
                       overwrite=overwrite)
