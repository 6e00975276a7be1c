"""ATUS-2 ``.bin`` wave-function files.

A ``.bin`` file is a 1380-byte ``generic_header`` followed by the grid data,
row-major with x slowest, as interleaved complex128 (``fftw_complex``) or as
float64 for real arrays.  The header layout is ``struct generic_header`` with
``#pragma pack(4)`` (include/my_structs.h:40-72); ``Read_header`` reads it raw
(include/CRT_shared.h:131-172), ``Save_Phi`` / ``Append_Phi`` write it
followed by the data (include/CRT_Base.h:606-641) and ``python/readbin_demo.py``
checks ``header[0] == 1380``.  Packed appends (``Seq_<n>_<c>.bin``) are
several header+data records back to back.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

HEADER_SIZE = 1380

HEADER_DTYPE = np.dtype(
    [
        ("nself", "<i8"),
        ("nDatatyp", "<i8"),
        ("nself_and_data", "<i8"),
        ("nDims", "<i8"),
        ("nDimX", "<i8"),
        ("nDimY", "<i8"),
        ("nDimZ", "<i8"),
        ("bAtom", "<i4"),
        ("bComplex", "<i4"),
        ("t", "<f8"),
        ("xMin", "<f8"),
        ("xMax", "<f8"),
        ("yMin", "<f8"),
        ("yMax", "<f8"),
        ("zMin", "<f8"),
        ("zMax", "<f8"),
        ("dx", "<f8"),
        ("dy", "<f8"),
        ("dz", "<f8"),
        ("dkx", "<f8"),
        ("dky", "<f8"),
        ("dkz", "<f8"),
        ("dt", "<f8"),
        ("ks", "<i4"),
        ("fs", "<i4"),
        ("nFuture", "<i4", (99,)),
        ("dFuture", "<f8", (100,)),
    ],
    align=False,
)
assert HEADER_DTYPE.itemsize == HEADER_SIZE


def make_header(dim: int, n, lo, hi, t: float = 0.0, dt: float = 0.001, complex_data: bool = True):
    """Header of a grid on [lo, hi) per axis, as gen_psi_0 and
    ParameterHandler::Get_Header build it (source/utils/src/gen_psi_0.cpp:40-93,
    ParameterHandler.cpp:488-563): dx = |hi-lo|/N, dk = 2*pi/|hi-lo|."""
    h = np.zeros((), dtype=HEADER_DTYPE)
    h["nself"] = HEADER_SIZE
    h["nDatatyp"] = 16 if complex_data else 8
    h["nDims"] = dim
    h["bAtom"] = 1
    h["bComplex"] = 1 if complex_data else 0
    h["t"] = t
    h["dt"] = dt
    n = list(n) + [1] * (3 - len(n))
    lo = list(lo) + [0.0] * (3 - len(lo))
    hi = list(hi) + [0.0] * (3 - len(hi))
    for a, ax in enumerate("XYZ"):
        h[f"nDim{ax}"] = n[a]
    for a, ax in enumerate("xyz"):
        h[f"{ax}Min"] = lo[a]
        h[f"{ax}Max"] = hi[a]
        if a < dim:
            L = math.fabs(hi[a] - lo[a])
            h[f"d{ax}"] = L / float(n[a])
            h[f"dk{ax}"] = 2 * math.pi / L
    return h


@dataclass
class BinFile:
    header: np.ndarray  # structured scalar of HEADER_DTYPE
    data: np.ndarray  # complex128 or float64, shape (nx[, ny[, nz]])

    @property
    def dim(self) -> int:
        return int(self.header["nDims"])

    @property
    def shape(self):
        return grid_shape(self.header)


def grid_shape(header) -> tuple:
    dim = int(header["nDims"])
    n = [int(header["nDimX"]), int(header["nDimY"]), int(header["nDimZ"])]
    return tuple(n[:dim])


def read_bin(path: str, record: int = 0, complex_data: bool | None = None) -> BinFile:
    """Read one header+data record (``record`` counts packed appends)."""
    with open(path, "rb") as f:
        raw = f.read(HEADER_SIZE)
        if len(raw) != HEADER_SIZE:
            raise ValueError(f"{path}: truncated header")
        h = np.frombuffer(raw, dtype=HEADER_DTYPE)[0].copy()
        if int(h["nself"]) != HEADER_SIZE:
            raise ValueError(f"{path}: header size field is {int(h['nself'])}, expected {HEADER_SIZE}")
        shape = grid_shape(h)
        npts = int(np.prod(shape))
        is_c = bool(h["bComplex"]) if complex_data is None else complex_data
        nbytes = npts * (16 if is_c else 8)
        if record:
            f.seek(record * (HEADER_SIZE + nbytes))
            raw = f.read(HEADER_SIZE)
            if len(raw) != HEADER_SIZE:
                raise ValueError(f"{path}: no record {record}")
            h = np.frombuffer(raw, dtype=HEADER_DTYPE)[0].copy()
        buf = f.read(nbytes)
        if len(buf) != nbytes:
            raise ValueError(f"{path}: truncated data ({len(buf)} of {nbytes} bytes)")
    data = np.frombuffer(buf, dtype=np.complex128 if is_c else np.float64).reshape(shape).copy()
    return BinFile(h, data)


def write_bin(path: str, header, data: np.ndarray, append: bool = False) -> None:
    """Write header + data (``append`` adds a record, as Append_Phi does)."""
    h = np.asarray(header, dtype=HEADER_DTYPE).copy()
    arr = np.ascontiguousarray(data)
    with open(path, "ab" if append else "wb") as f:
        f.write(h.tobytes())
        f.write(arr.tobytes())


def x_coords(header, axis: int) -> np.ndarray:
    """x_i = (i - N/2) * dx, cft_{1,2,3}d::Get_x (cft_3d.cpp:128-138)."""
    ax = "xyz"[axis]
    n = int(header[f"nDim{ax.upper()}"])
    return (np.arange(n, dtype=np.int64) - n // 2).astype(np.float64) * float(header[f"d{ax}"])


def k_coords(header, axis: int) -> np.ndarray:
    """Wrapped k of cft_{1,2,3}d::Get_k with SetFix(false) (cft_3d.cpp:145-166):
    k_i = dk * (((i + N/2) mod N) - N/2)."""
    ax = "xyz"[axis]
    n = int(header[f"nDim{ax.upper()}"])
    i = np.arange(n, dtype=np.int64)
    return float(header[f"dk{ax}"]) * (((i + n // 2) % n) - n // 2).astype(np.float64)


def file_exists(path: str) -> bool:
    return os.path.isfile(path)
