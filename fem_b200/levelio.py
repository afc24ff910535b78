"""Reader/writer of the sample generator's level<L>_*.bin files.

Format (Utilities/include/cfgUtilities.h:780-870, written by
SamplesGenerator/SamplesGeneratorImpl.cpp:3811-3851): a flat vector is an
int32 count followed by the raw values; a vector of vectors is an int32 count
of vectors, each stored as a flat vector.  matAssignments/baseMat are int32,
params/elasticityTensors float32 (cfgScalar in the default float build).
"""
from __future__ import annotations

import os
import struct
from typing import Sequence

import numpy as np


def write_vector(path: str, values, dtype=np.float32) -> None:
    a = np.ascontiguousarray(values, dtype=dtype).ravel()
    with open(path, "wb") as f:
        f.write(struct.pack("<i", a.size))
        f.write(a.tobytes())


def read_vector(path: str, dtype=np.float32) -> np.ndarray:
    with open(path, "rb") as f:
        (n,) = struct.unpack("<i", f.read(4))
        a = np.frombuffer(f.read(n * np.dtype(dtype).itemsize), dtype=dtype)
    if a.size != n:
        raise ValueError(f"{path}: truncated ({a.size} of {n} values)")
    return a.copy()


def write_vectors(path: str, vectors: Sequence, dtype=np.int32) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<i", len(vectors)))
        for v in vectors:
            a = np.ascontiguousarray(v, dtype=dtype).ravel()
            f.write(struct.pack("<i", a.size))
            f.write(a.tobytes())


def read_vectors(path: str, dtype=np.int32) -> list[np.ndarray]:
    out = []
    with open(path, "rb") as f:
        (n,) = struct.unpack("<i", f.read(4))
        for _ in range(n):
            (m,) = struct.unpack("<i", f.read(4))
            a = np.frombuffer(f.read(m * np.dtype(dtype).itemsize), dtype=dtype)
            if a.size != m:
                raise ValueError(f"{path}: truncated")
            out.append(a.copy())
    return out


def level_paths(directory: str, level: int, postfix: str = "") -> dict:
    root = os.path.join(directory, f"level{level}_" + (postfix + "_" if postfix else ""))
    return {k: root + k + ".bin" for k in ("params", "baseMat", "matAssignments", "elasticityTensors")}


def tensors_to_level_file(path: str, C: np.ndarray) -> None:
    """Append-order of NumericalCoarseningUsingMultiGrid.cpp:315-324: for every
    structure the 21 lower-triangle entries C(i, j), j <= i, row by row."""
    C = np.asarray(C).reshape(-1, 6, 6)
    vals = [C[s, i, j] for s in range(C.shape[0]) for i in range(6) for j in range(i + 1)]
    write_vector(path, np.array(vals), np.float32)
