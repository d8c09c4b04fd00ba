"""Minimal NIfTI-1 writer for test inputs (352-byte header + data)."""
import struct

import numpy as np

_NP = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64}
_BITPIX = {2: 8, 4: 16, 8: 32, 16: 32, 64: 64}


def write_nifti(path, data, dtype_code, endian="<", extension=b"", slope=0.0, inter=0.0):
    """data: (X, Y, Z) or (X, Y, Z, T) array; dtype_code 2 = uint8, 4 = int16,
    8 = int32, 16 = float32, 64 = float64.  endian '>' writes a big-endian
    file; `extension` bytes (a multiple of 16 after the 4-byte flag) move the
    data to vox_offset = 352 + len(extension); slope/inter fill scl_slope and
    scl_inter (the stored values are written as given)."""
    data = np.asarray(data)
    dims = list(data.shape) + [1] * (4 - data.ndim)
    hdr = bytearray(352)
    struct.pack_into(endian + "i", hdr, 0, 348)
    struct.pack_into(endian + "8h", hdr, 40, 4 if data.ndim == 4 else 3, dims[0], dims[1], dims[2], dims[3], 1, 1, 1)
    struct.pack_into(endian + "hh", hdr, 70, dtype_code, _BITPIX[dtype_code])
    struct.pack_into(endian + "f", hdr, 108, float(352 + len(extension)))
    struct.pack_into(endian + "ff", hdr, 112, slope, inter)
    hdr[344:348] = b"n+1\0"
    if extension:
        hdr[348] = 1
    npdt = np.dtype(_NP[dtype_code]).newbyteorder(endian)
    # NIfTI order: x fastest, then y, z, t
    body = np.asarray(data).astype(npdt).transpose(*reversed(range(data.ndim))).tobytes()
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(extension)
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
