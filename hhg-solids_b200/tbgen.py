"""Seeded synthetic Wannier tight-binding models in the ``*_tb.dat`` layout the reference parses.

The layout is the one ``src/wannier_tb.cpp:15-113`` of rodrigomarher/HHG-Solids reads: a comment
line, three lattice rows (Angstrom), ``num_wann``, ``nrpts``, degeneracy lines (15 per line), a
blank line, then per R cell an ``n1 n2 n3`` line, ``num_wann**2`` lines ``m n Re Im`` (eV) and a
blank line, then the position blocks (``m n xRe xIm yRe yIm zRe zIm``, Angstrom) in the same cell
order.  The reader stores the element of line ``m n`` at ``[n-1][m-1]``; the generators below build
the stored matrices ``M_R[i][j]`` directly and write each as line ``m=j+1 n=i+1``, keeping
``M_{-R} = M_R^+`` so every H(k) is Hermitian.

Models (hexagonal lattice a1 = (a sqrt3/2, -a/2, 0), a2 = (a sqrt3/2, a/2, 0), a3 = (0, 0, 15)):

* :func:`haldane` -- 2 orbitals, a = 2.5 A, on-site -/+0.8 eV, nearest-neighbour -2.7 eV with the
  bond pattern of the reference's ``hmcase0_tb.dat``, next-nearest 0.1 e^{+-i pi/2} eV with opposite
  chirality on the two sublattices, B-orbital centre x = a/sqrt3, cells |n1|,|n2| <= 2 (25 cells).
* :func:`random_tmd` -- ``nw`` orbitals from ``numpy.random.default_rng(seed)``: random Hermitian
  pairs H_{-R} = H_R^+ on a ``window x window`` cell block with |H_R| ~ 0.5 exp(-|R|/1.2 cells) eV,
  on-site energies uniform in [-3, 3] eV, and positions r_R (x, y; z = 0) with the same decay
  x 0.3 A.
"""
from __future__ import annotations

import hashlib
import math
import os

import numpy as np

__all__ = ["haldane", "random_tmd", "write_tb", "model_path", "MODELS"]


def _lattice(a: float) -> np.ndarray:
    return np.array([[a * math.sqrt(3) / 2, -a / 2, 0.0], [a * math.sqrt(3) / 2, a / 2, 0.0], [0.0, 0.0, 15.0]])


def _cells(half: int):
    return [(n1, n2) for n1 in range(-half, half + 1) for n2 in range(-half, half + 1)]


def write_tb(path: str, comment: str, lattice: np.ndarray, cells, H: dict, X: dict, degeneracy: dict | None = None) -> str:
    """Write a model; ``H[cell]`` is the stored nw x nw complex matrix, ``X[cell]`` is (3, nw, nw),
    ``degeneracy[cell]`` the Wigner-Seitz weight written in the header (1 when omitted).

    Returns the sha256 of the file."""
    nw = next(iter(H.values())).shape[0]
    lines = [comment]
    for row in lattice:
        lines.append(" ".join(f"{v:.18e}" for v in row))
    lines.append(str(nw))
    lines.append(str(len(cells)))
    deg = [str(int((degeneracy or {}).get(c, 1))) for c in cells]
    for i in range(0, len(deg), 15):
        lines.append(" ".join(deg[i : i + 15]))
    lines.append("")
    for c in cells:
        lines.append(f"{c[0]:5d}{c[1]:5d}{0:5d}")
        M = H[c]
        for i in range(nw):  # stored row i <- file column index n = i+1
            for j in range(nw):
                v = M[i, j]
                lines.append(f"{j + 1:4d}{i + 1:4d}  {v.real: .16e} {v.imag: .16e}")
        lines.append("")
    for c in cells:
        lines.append(f"{c[0]:5d}{c[1]:5d}{0:5d}")
        P = X[c]
        for i in range(nw):
            for j in range(nw):
                vals = " ".join(f"{P[a, i, j].real: .16e} {P[a, i, j].imag: .16e}" for a in range(3))
                lines.append(f"{j + 1:4d}{i + 1:4d}  {vals}")
        lines.append("")
    text = "\n".join(lines) + "\n"
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
        f.write(text)
    os.replace(tmp, path)
    return hashlib.sha256(text.encode()).hexdigest()


def haldane(path: str, a: float = 2.5, onsite: float = 0.8, t1: float = -2.7, t2: float = 0.1) -> str:
    cells = _cells(2)
    z = lambda: np.zeros((2, 2), dtype=np.complex128)  # noqa: E731
    H = {c: z() for c in cells}
    X = {c: np.zeros((3, 2, 2), dtype=np.complex128) for c in cells}
    H[(0, 0)][0, 0] = -onsite
    H[(0, 0)][1, 1] = onsite
    # Nearest neighbours: stored [1][0] at R in {0, -a1, -a2}, [0][1] at R in {0, a1, a2}.
    for c in [(0, 0), (-1, 0), (0, -1)]:
        H[c][1, 0] += t1
    for c in [(0, 0), (1, 0), (0, 1)]:
        H[c][0, 1] += t1
    # Next-nearest neighbours along d1 = a1, d2 = a2 - a1, d3 = -a2 (a closed triangle).
    ph = t2 * np.exp(1j * math.pi / 2)
    for d in [(1, 0), (-1, 1), (0, -1)]:
        md = (-d[0], -d[1])
        H[d][0, 0] += ph
        H[md][0, 0] += np.conj(ph)
        H[d][1, 1] += np.conj(ph)
        H[md][1, 1] += ph
    X[(0, 0)][0, 1, 1] = a / math.sqrt(3)
    return write_tb(path, "synthetic Haldane-like 2-orbital model (hhg-b200 tbgen)", _lattice(a), cells, H, X)


def random_tmd(path: str, nw: int = 11, seed: int = 7, window: int = 7, a: float = 2.5) -> str:
    rng = np.random.default_rng(seed)
    half = window // 2
    cells = _cells(half)
    H = {c: np.zeros((nw, nw), dtype=np.complex128) for c in cells}
    X = {c: np.zeros((3, nw, nw), dtype=np.complex128) for c in cells}

    def decay(c):
        return math.exp(-math.sqrt(c[0] ** 2 + c[1] ** 2 + c[0] * c[1]) / 1.2)

    def cgauss(shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2)

    for c in cells:
        mc = (-c[0], -c[1])
        if c == (0, 0):
            G = cgauss((nw, nw)) * 0.5
            H[c] = (G + G.conj().T) / 2 + np.diag(rng.uniform(-3.0, 3.0, nw))
            for ax in range(2):
                P = cgauss((nw, nw)) * 0.3
                X[c][ax] = (P + P.conj().T) / 2
        elif c > mc:  # draw each (R, -R) pair once
            H[c] = cgauss((nw, nw)) * 0.5 * decay(c)
            H[mc] = H[c].conj().T
            for ax in range(2):
                X[c][ax] = cgauss((nw, nw)) * 0.3 * decay(c)
                X[mc][ax] = X[c][ax].conj().T
    return write_tb(path, f"synthetic TMD-like {nw}-orbital model, seed {seed} (hhg-b200 tbgen)", _lattice(a),
                    cells, H, X)


def _deg_model(nw: int, seed: int, window: int, a: float):
    """A random model with Wannier90-style degeneracies (2 on the edge of the cell window, 4 at its
    corners), as (cells, stored H, stored X, degeneracy)."""
    rng = np.random.default_rng(seed)
    half = window // 2
    cells = _cells(half)
    H, X, deg = {}, {}, {}
    for c in cells:
        mc = (-c[0], -c[1])
        deg[c] = (2 if abs(c[0]) == half else 1) * (2 if abs(c[1]) == half else 1)
        if c in H:
            continue
        if c == (0, 0):
            G = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) * 0.4
            H[c] = (G + G.conj().T) / 2 + np.diag(rng.uniform(-3.0, 3.0, nw))
            X[c] = np.zeros((3, nw, nw), dtype=np.complex128)
            for ax in range(2):
                P = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) * 0.2
                X[c][ax] = (P + P.conj().T) / 2
        else:
            s = 0.4 * math.exp(-math.hypot(c[0], c[1]) / 1.2)
            H[c] = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) * s
            H[mc] = H[c].conj().T
            X[c] = np.zeros((3, nw, nw), dtype=np.complex128)
            X[mc] = np.zeros((3, nw, nw), dtype=np.complex128)
            for ax in range(2):
                X[c][ax] = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) * 0.5 * s
                X[mc][ax] = X[c][ax].conj().T
    return cells, H, X, deg


def tmd_deg(path: str, nw: int = 6, seed: int = 5, window: int = 5, a: float = 2.5) -> str:
    """A model file with non-unit degeneracies, read as Wannier90 defines them with
    SWE(..., tb_convention="faithful")."""
    cells, H, X, deg = _deg_model(nw, seed, window, a)
    return write_tb(path, f"synthetic {nw}-orbital model with degeneracies, seed {seed} (hhg-b200 tbgen)",
                    _lattice(a), cells, H, X, deg)


def tmd_deg_equiv(path: str, nw: int = 6, seed: int = 5, window: int = 5, a: float = 2.5) -> str:
    """The same model rewritten so that the reference's own reading (transposed blocks, degeneracies
    ignored) gives the faithful reading of tmd_deg: stored blocks M^T / degeneracy, unit degeneracies."""
    cells, H, X, deg = _deg_model(nw, seed, window, a)
    H2 = {c: H[c].T / deg[c] for c in cells}
    X2 = {c: np.stack([X[c][ax].T for ax in range(3)]) / deg[c] for c in cells}
    return write_tb(path, f"synthetic {nw}-orbital model, degeneracies applied, seed {seed} (hhg-b200 tbgen)",
                    _lattice(a), cells, H2, X2)


# name -> (generator, kwargs)
MODELS = {
    "haldane": (haldane, {}),
    "tmd11_s7": (random_tmd, {"nw": 11, "seed": 7}),
    "tmd6_s1": (random_tmd, {"nw": 6, "seed": 1}),
    "tmd6_s2": (random_tmd, {"nw": 6, "seed": 2}),
    "tmd6_s3": (random_tmd, {"nw": 6, "seed": 3}),
    "tmd11_s1": (random_tmd, {"nw": 11, "seed": 1}),
    "tmd11_s3": (random_tmd, {"nw": 11, "seed": 3}),
    "tmd11_s2": (random_tmd, {"nw": 11, "seed": 2}),
    "tmd12_s1": (random_tmd, {"nw": 12, "seed": 1}),
    "tmd12_s2": (random_tmd, {"nw": 12, "seed": 2}),
    "tmd12_s3": (random_tmd, {"nw": 12, "seed": 3}),
    "tmd5_s4": (random_tmd, {"nw": 5, "seed": 4, "window": 5}),
    "tmd16_s1": (random_tmd, {"nw": 16, "seed": 1, "window": 5}),
    "tmd1_s2": (random_tmd, {"nw": 1, "seed": 2, "window": 5}),
    "tmd6_deg": (tmd_deg, {}),
    "tmd6_deg_equiv": (tmd_deg_equiv, {}),
}


def model_path(name: str, directory: str | None = None) -> str:
    """Generate (once) and return the path of a named model file."""
    if directory is None:
        directory = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_models")
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, f"{name}_tb.dat")
    if not os.path.exists(path):
        gen, kw = MODELS[name]
        gen(path, **kw)
    return path
