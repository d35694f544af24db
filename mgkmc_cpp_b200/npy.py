"""``.npy`` modulus-field input with the reference reader's rules.

read_npy_double follows material_generator.hpp:23-116: versions 1 and 2,
``<f8`` (or no descr) and ``<f4`` (widened to float64), data in C order (the
reference does not look at ``fortran_order``).  Errors raise ValueError with the
reference's messages.  write_npy writes version-1 ``<f8`` C-order files.
"""
from __future__ import annotations

import struct
from typing import List, Tuple

import numpy as np


def read_npy_double(path: str) -> Tuple[np.ndarray, List[int]]:
    try:
        f = open(path, "rb")
    except OSError:
        raise ValueError("Failed to open npy file: " + path)
    with f:
        magic = f.read(6)
        if magic != b"\x93NUMPY":
            raise ValueError("Invalid npy magic bytes")
        major = f.read(1)[0]
        f.read(1)
        if major == 1:
            hlen = struct.unpack("<H", f.read(2))[0]
        elif major == 2:
            hlen = struct.unpack("<I", f.read(4))[0]
        else:
            raise ValueError("Unsupported npy version: %d" % major)
        header = f.read(hlen).decode("latin1")
        sp = header.find("'shape'")
        if sp < 0:
            sp = header.find('"shape"')
        if sp < 0:
            raise ValueError("Could not find 'shape' in npy header")
        colon = header.find(":", sp)
        op = header.find("(", colon)
        cp = header.find(")", op)
        if op < 0 or cp < 0:
            raise ValueError("Invalid shape format in npy header")
        shape = [int(t) for t in header[op + 1:cp].replace(" ", "").split(",") if t]
        descr = ""
        dp = header.find("'descr'")
        if dp < 0:
            dp = header.find('"descr"')
        if dp >= 0:
            c = header.find(":", dp)
            q1 = min(i for i in (header.find("'", c), header.find('"', c)) if i >= 0)
            q2 = min(i for i in (header.find("'", q1 + 1), header.find('"', q1 + 1)) if i >= 0)
            descr = header[q1 + 1:q2]
        n = int(np.prod(shape)) if shape else 1
        if descr in ("<f4", "f4", "|f4"):
            data = np.frombuffer(f.read(4 * n), dtype="<f4", count=n).astype(np.float64)
        elif descr in ("<f8", "f8", "|f8", ""):
            data = np.frombuffer(f.read(8 * n), dtype="<f8", count=n).astype(np.float64)
        else:
            raise ValueError("Unsupported dtype in npy header: " + descr)
    return data, shape


def write_npy(path: str, arr) -> None:
    np.save(path, np.ascontiguousarray(np.asarray(arr, dtype=np.float64)))
