"""The reference's own Python wrapper, replayed against this library on the GPU.

``tests/golden/wrapper_trace/<case>.json`` holds what the reference's unmodified ``pySWE/pyswe.py``
(lines 9-98) declares and calls through ctypes for one run -- Settings_new and its setters,
SWESim_new, set_path_tb, set_settings, init, run_simulation, get_current, delete -- recorded by
``tests/golden/make_wrapper_trace.py``.  Each test binds those functions in this library with the
declared argtypes/restype, makes the same calls in the same order with the same values, and checks
the current it returns against the golden fixture the reference's own build produced for the case.
"""
import ctypes as ct
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_l2

pytestmark = pytest.mark.gpu

TRACES = os.path.join(GOLDEN, "wrapper_trace")


def ctype_of(name: str):
    if name == "None":
        return None
    if name.startswith("ndpointer:"):
        _, dtype, ndim, flags = name.split(":")
        return np.ctypeslib.ndpointer(dtype=np.dtype(dtype), ndim=int(ndim), flags=flags or None)
    return getattr(ct, name)


def replay(trace: dict, lib_path: str, path_tb: str):
    """Makes the trace's calls against ``lib_path``; returns the arrays get_current filled."""
    lib = ct.CDLL(lib_path)
    handles, out = {}, None
    for rec in trace["calls"]:
        fn = getattr(lib, rec["call"])
        fn.argtypes = [ctype_of(t) for t in rec["argtypes"]]
        fn.restype = ctype_of(rec["restype"])
        args = []
        for a in rec["args"]:
            (kind, val), = [(k, v) for k, v in a.items() if k in ("handle", "int", "float", "bytes", "array")]
            if kind == "handle":
                args.append(handles[val])
            elif kind == "int":
                args.append(int(val))
            elif kind == "float":
                args.append(float(val))
            elif kind == "bytes":
                args.append(path_tb.encode("UTF-8"))
            elif a["values"] is not None:
                args.append(np.array(a["values"], dtype=np.dtype(val)))
            else:
                args.append(np.zeros(a["len"], dtype=np.dtype(val)))
        if rec["call"] == "SWESim_get_current":
            out = args[1:]
        res = fn(*args)
        if rec["call"] == "Settings_new":
            handles["settings"] = res
        elif rec["call"] == "SWESim_new":
            handles["swe"] = res
    return out


@pytest.mark.parametrize("name", sorted(f[:-5] for f in os.listdir(TRACES) if f.endswith(".json")))
def test_reference_wrapper_calls_reproduce_golden(name):
    from pySWE import pyswe

    with open(os.path.join(TRACES, f"{name}.json")) as f:
        trace = json.load(f)
    meta, param, t_ref, J_ref = load_golden(name)
    t, jx, jy, jz = replay(trace, pyswe.default_library(), param["path_tb"])
    assert np.array_equal(t, t_ref)
    for a, j in enumerate((jx, jy, jz)):
        if np.abs(J_ref[a]).max() == 0:
            assert np.abs(j).max() == 0, (name, a)
        else:
            assert rel_l2(j, J_ref[a]) < 1e-10, (name, a, rel_l2(j, J_ref[a]))
