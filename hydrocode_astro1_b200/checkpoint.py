"""Reader of the library's binary checkpoint files (hc_checkpoint_save).

    from hydrocode_astro1_b200.checkpoint import read_checkpoint
    ck = read_checkpoint("run.ckpt")   # ck["state"]: (5, nx, ny, nz), ck["phi"], ck["phig"], ck["t"], ...

Layout (native little-endian, no padding): a 136-byte header

    char[8] magic "HCCKPT01"; int32 version (1), header_bytes (136), nx, ny, nz,
    precision (0 FP64, 1 FP32), gravity (0/1), parity; int64 step; float64 t,
    lo[3], hi[3], gamma, G; uint64 payload_bytes, checksum (FNV-1a 64 of the payload)

then the payload: the 5 conserved fields (rho, rho u, rho v, rho w, E), each
nx*ny*nz values with k fastest, as float64 (FP64 contexts) or float32 (FP32
contexts); then, when gravity is on, the potential and the potential of the
last converged solve, nx*ny*nz float64 each.
"""
from __future__ import annotations

import numpy as np

HEADER = np.dtype([("magic", "S8"), ("version", "<i4"), ("header_bytes", "<i4"), ("nx", "<i4"), ("ny", "<i4"),
                   ("nz", "<i4"), ("precision", "<i4"), ("gravity", "<i4"), ("parity", "<i4"), ("step", "<i8"),
                   ("t", "<f8"), ("lo", "<f8", 3), ("hi", "<f8", 3), ("gamma", "<f8"), ("G", "<f8"),
                   ("payload_bytes", "<u8"), ("checksum", "<u8")])
assert HEADER.itemsize == 136


def fnv1a64(data: bytes) -> int:
    """FNV-1a 64-bit hash of the payload (the header's checksum)."""
    h = 14695981039346656037
    prime = 1099511628211
    mask = (1 << 64) - 1
    for b in data:
        h = ((h ^ b) * prime) & mask
    return h


def read_checkpoint(path, verify=False):
    """Header fields plus the arrays; verify=True also checks the checksum
    (pure Python: slow for large files)."""
    with open(path, "rb") as f:
        raw = f.read()
    h = np.frombuffer(raw[:HEADER.itemsize], dtype=HEADER)[0]
    if h["magic"] != b"HCCKPT01" or int(h["version"]) != 1 or int(h["header_bytes"]) != HEADER.itemsize:
        raise ValueError(f"{path}: not a version-1 checkpoint")
    nx, ny, nz = int(h["nx"]), int(h["ny"]), int(h["nz"])
    n = nx * ny * nz
    word = np.float64 if int(h["precision"]) == 0 else np.float32
    payload = raw[HEADER.itemsize:]
    if len(payload) != int(h["payload_bytes"]):
        raise ValueError(f"{path}: payload is {len(payload)} bytes, header says {int(h['payload_bytes'])}")
    if verify and fnv1a64(payload) != int(h["checksum"]):
        raise ValueError(f"{path}: checksum mismatch")
    out = {k: h[k] for k in ("step", "t", "gamma", "G", "parity", "precision", "gravity")}
    out["lo"], out["hi"], out["shape"] = tuple(h["lo"]), tuple(h["hi"]), (nx, ny, nz)
    ws = np.dtype(word).itemsize
    out["state"] = np.frombuffer(payload, dtype=word, count=5 * n).reshape(5, nx, ny, nz)
    if int(h["gravity"]):
        out["phi"] = np.frombuffer(payload, dtype=np.float64, count=n, offset=5 * n * ws).reshape(nx, ny, nz)
        out["phig"] = np.frombuffer(payload, dtype=np.float64, count=n, offset=5 * n * ws + 8 * n).reshape(nx, ny, nz)
    return out
