import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hhg-solids_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

# The reference checkout (read-only; absent on machines that only run the GPU tests).
REFERENCE_CHECKOUT = os.environ.get("HHG_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def golden_names():
    return sorted(f[:-5] for f in os.listdir(GOLDEN) if f.endswith(".json"))


def load_golden(name):
    """(meta, param dict for pySWE, t, J[3, nt]) of a committed fixture."""
    import tbgen

    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        meta = json.load(f)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    param = dict(meta["param"])
    param["pol_vec"] = np.array(param["pol_vec"], dtype=np.float64)
    param["phi_vec"] = np.array(param["phi_vec"], dtype=np.float64)
    param["path_tb"] = tbgen.model_path(meta["model"])
    return meta, param, z["t"], z["J"]


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()  # builds liboracle.so on first use
    return oracle


def tb_blocks(path):
    """{(n1, n2): H block as stored by the reference reader, flattened nw*nw} of a TB file."""
    lines = open(path).read().split("\n")
    nw, ns = int(lines[4]), int(lines[5])
    i = 6 + (ns - 1) // 15 + 1 + 1
    out = {}
    for _ in range(ns):
        cell = tuple(int(x) for x in lines[i].split()[:2])
        i += 1
        M = np.zeros((nw, nw), dtype=np.complex128)
        for _ in range(nw * nw):
            m, n, re, im = lines[i].split()[:4]
            i += 1
            M[int(n) - 1, int(m) - 1] = float(re) + 1j * float(im)
        i += 1
        out.setdefault(cell, M.reshape(-1))
    return nw, out
