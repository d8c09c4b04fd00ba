"""Minimal NIfTI-1 writer for test inputs (352-byte header + data)."""
import struct

import numpy as np


def write_nifti(path, data, dtype_code):
    """data: (X, Y, Z) or (X, Y, Z, T) array; dtype_code 2 = uint8, 16 = float32, 64 = float64."""
    data = np.asarray(data)
    dims = list(data.shape) + [1] * (4 - data.ndim)
    hdr = bytearray(352)
    struct.pack_into("<i", hdr, 0, 348)
    struct.pack_into("<8h", hdr, 40, 4 if data.ndim == 4 else 3, dims[0], dims[1], dims[2], dims[3], 1, 1, 1)
    bitpix = {2: 8, 16: 32, 64: 64}[dtype_code]
    struct.pack_into("<hh", hdr, 70, dtype_code, bitpix)
    struct.pack_into("<f", hdr, 108, 352.0)
    hdr[344:348] = b"n+1\0"
    npdt = {2: np.uint8, 16: np.float32, 64: np.float64}[dtype_code]
    # NIfTI order: x fastest, then y, z, t
    body = np.asarray(data, npdt).transpose(*reversed(range(data.ndim))).tobytes()
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(body)


def volume_from_series(bold_TxN, shape):
    """Place N voxel series into a (X, Y, Z, T) volume in x-fastest order."""
    T, N = bold_TxN.shape
    X, Y, Z = shape
    assert X * Y * Z >= N
    vol = np.zeros((X * Y * Z, T), np.float32)
    vol[:N] = bold_TxN.T
    # flat index k = x + X*(y + Y*z)  ->  array index [x, y, z]
    return vol.reshape(Z, Y, X, T).transpose(2, 1, 0, 3)
