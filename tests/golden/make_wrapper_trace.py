"""Record the exact ctypes traffic of the reference's own Python wrapper, for replay on a GPU.

The reference's ``pySWE/pyswe.py`` (lines 9-98) declares every C function it binds (argtypes and
restype) and calls them in a fixed order: ``Settings(param)`` creates and fills a C ``Settings``,
``SWE(settings)`` creates a ``SWESim``, sets the TB path and the settings and runs ``SWESim_init``,
then the user calls ``run_simulation()``, ``get_current()`` and ``delete()``.  The GPU box has no
reference checkout, so this script imports that unmodified file here with ``ctypes.CDLL`` replaced
by a recorder and writes what it declared and called -- function names, declared ctypes, argument
values, with the object handles and the TB path as symbols -- to ``wrapper_trace/<case>.json``.
``tests/test_zy_reference_wrapper_gpu.py`` replays each trace call for call against this library on
the GPU and compares the current with the golden fixture of the same case.

    python tests/golden/make_wrapper_trace.py [--ref /root/reference]
"""
from __future__ import annotations

import argparse
import ctypes as ct
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "wrapper_trace")
CASES = ("c0", "tmd6_8", "haldane_12_pol")


def ctype_name(t) -> str:
    """A portable name for a ctypes argument or result type."""
    if t is None:
        return "None"
    if hasattr(t, "_dtype_"):  # np.ctypeslib.ndpointer(dtype, ndim, flags)
        return f"ndpointer:{np.dtype(t._dtype_).name}:{t._ndim_}:{'C' if (t._flags_ or 0) & 1 else ''}"
    return t.__name__


class _Recorder:
    """Stands in for one ``ctypes.CDLL``: remembers declarations and calls in order."""

    def __init__(self, log: list, handles: dict):
        object.__setattr__(self, "_log", log)
        object.__setattr__(self, "_funcs", {})
        object.__setattr__(self, "_handles", handles)

    def __getattr__(self, name):
        funcs = object.__getattribute__(self, "_funcs")
        if name not in funcs:
            funcs[name] = _Func(name, self)
        return funcs[name]


class _Func:
    def __init__(self, name, rec):
        self.name, self.rec = name, rec
        self.argtypes, self.restype = None, ct.c_int

    def __call__(self, *args):
        handles = self.rec._handles
        enc = []
        for a in args:
            if isinstance(a, np.ndarray):
                enc.append({"array": a.dtype.name, "len": int(a.size),
                            "values": a.tolist() if a.dtype != np.complex128 else None})
            elif isinstance(a, bytes):
                enc.append({"bytes": "<path_tb>"})
            elif isinstance(a, int) and a in handles:
                enc.append({"handle": handles[a]})
            elif isinstance(a, float):
                enc.append({"float": a})
            elif isinstance(a, int):
                enc.append({"int": a})
            else:
                raise TypeError(f"{self.name}: unrecorded argument type {type(a)}")
        self.rec._log.append({"call": self.name, "argtypes": [ctype_name(t) for t in (self.argtypes or [])],
                              "restype": ctype_name(self.restype), "args": enc})
        if self.name in ("Settings_new", "SWESim_new"):
            h = 0x1000 + 0x10 * len(handles)
            handles[h] = "settings" if self.name == "Settings_new" else "swe"
            return h
        return None


def record(ref: str, name: str) -> dict:
    with open(os.path.join(HERE, f"{name}.json")) as f:
        meta = json.load(f)
    spec = importlib.util.spec_from_file_location("reference_pyswe", os.path.join(ref, "pySWE", "pyswe.py"))
    mod = importlib.util.module_from_spec(spec)
    log, handles = [], {}
    real_cdll = ct.CDLL
    ct.CDLL = lambda path, *a, **k: _Recorder(log, handles)  # noqa: E731
    try:
        spec.loader.exec_module(mod)
        p = dict(meta["param"])
        param = dict(p, path_lib="<path_lib>", path_tb="<path_tb>",
                     pol_vec=np.array(p["pol_vec"], dtype=np.float64), phi_vec=np.array(p["phi_vec"], dtype=np.float64))
        settings = mod.Settings(param)
        swe = mod.SWE(settings)
        swe.run_simulation()
        swe.get_current()
        swe.delete()
    finally:
        ct.CDLL = real_cdll
    return {"case": name, "source": "pySWE/pyswe.py of the reference, imported unmodified with ctypes.CDLL recorded",
            "calls": log}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("HHG_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    os.makedirs(OUT, exist_ok=True)
    for name in CASES:
        trace = record(args.ref, name)
        with open(os.path.join(OUT, f"{name}.json"), "w") as f:
            json.dump(trace, f, indent=1)
        print(name, len(trace["calls"]), "calls")


if __name__ == "__main__":
    main()
