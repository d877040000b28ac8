"""Host-side readers for the path's input formats (product code, not the oracle).

read_homeltab   CollapseTable.read_homeltab (CollapseTable.jl:96-115): header
                3 x Int32 (Nx, Ny, Nz) + 6 x Float32 (X1, X2, Y1, Y2, Z1, Z2), then the
                Float32 table, column-major.
read_filterbank Filters.read_filterbank (Filters.jl:39-51): first line nic, then
                nic lines "id fcrit Rf".
"""
from __future__ import annotations

import numpy as np


def read_homeltab(path: str):
    """Return (table (nz, ny, nx) float32 -- Julia's column-major bytes --,
    (X1, X2, Y1, Y2, Z1, Z2) as float64 of the Float32 header values)."""
    raw = open(path, "rb").read()
    nx, ny, nz = (int(v) for v in np.frombuffer(raw[:12], dtype="<i4"))
    axes = tuple(float(v) for v in np.frombuffer(raw[12:36], dtype="<f4"))
    need = 36 + 4 * nx * ny * nz
    if len(raw) < need:
        raise ValueError(f"{path}: truncated HomelTab ({len(raw)} < {need} bytes)")
    table = np.frombuffer(raw[36:need], dtype="<f4").reshape(nz, ny, nx).copy()
    return table, axes


def write_homeltab(path: str, table: np.ndarray, axes) -> None:
    nz, ny, nx = table.shape
    with open(path, "wb") as f:
        f.write(np.array([nx, ny, nz], dtype="<i4").tobytes())
        f.write(np.array(axes, dtype="<f4").tobytes())
        f.write(np.ascontiguousarray(table, dtype="<f4").tobytes())


def read_filterbank(path: str):
    """List of (id, fcrit, Rf) tuples."""
    lines = open(path).read().splitlines()
    nic = int(lines[0].strip())
    out = []
    for ln in lines[1:1 + nic]:
        parts = ln.split()
        out.append((int(parts[0]), float(parts[1]), float(parts[2])))
    return out


def log_filterbank(n: int, rmin: float, rmax: float, fcrit: float = 1.686):
    """A bank of n log-spaced filter radii, largest first (the order the drivers use,
    MultiResolution.jl:725)."""
    r = np.exp(np.linspace(np.log(rmin), np.log(rmax), n))[::-1]
    return [(i + 1, fcrit, float(v)) for i, v in enumerate(r)]
