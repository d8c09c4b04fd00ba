"""The reference-compatible CLI tools: built, and argument errors are
reported before any GPU work (CPU only)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "pagani-toolkit_b200", "bin")
TOOLS = ["CUCorMat", "CUCorMat_weighted", "Degree", "Cp", "BFS_MulCPU", "CUBFW_Lp", "CUBC",
         "Newman_Modularity", "Newman_Modularity_weighted", "CUEC", "PC_CPU", "Maslov", "SmallWorldProperty", "ConvertNII"]


@pytest.mark.parametrize("tool", TOOLS)
def test_tool_usage(tool):
    exe = os.path.join(BIN, tool)
    assert os.path.exists(exe), f"{exe} not built"
    p = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1
    assert "Input format" in (p.stderr + p.stdout)


def test_cucormat_rejects_bad_threshold_type(tmp_path):
    exe = os.path.join(BIN, "CUCorMat")
    p = subprocess.run([exe, str(tmp_path), "0.5", "n", "n", "x", "0.3"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "threshold type error" in p.stderr


@pytest.mark.parametrize("avg", ["y", "b", "yx", "x", "q"])
def test_cucormat_rejects_bad_average_mode(tmp_path, avg):
    """to_average must be n, yf, yn, bf or bn (the reference silently leaves
    the average at zero for y or b alone)."""
    exe = os.path.join(BIN, "CUCorMat")
    p = subprocess.run([exe, str(tmp_path), "0.5", avg, "n", "r", "0.3"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "to_average must be" in p.stderr


# ---------------------------------------------------------------- ConvertNII
def _write_nm(path, x):
    with open(path, "wb") as f:
        np.array([len(x)], np.int32).tofile(f)
        np.asarray(x, np.float32).tofile(f)


def _convert_expected(mask_flat, hdr, x, cut):
    """The reference's output: the mask's 352 header bytes with datatype 16 and
    bitpix 32 (ConvertNII.cpp:139-142), then float32 values in mask voxels."""
    out = bytearray(hdr)
    out[70:74] = np.array([16, 32], np.int16).tobytes()
    vol = np.zeros(mask_flat.size, np.float32)
    vol[mask_flat >= cut] = x
    return bytes(out) + vol.tobytes()


def _flat(mask_xyz):
    return np.asarray(mask_xyz).transpose(2, 1, 0).reshape(-1)   # x fastest


@pytest.mark.parametrize("code,cut", [(2, None), (16, 0.4)])
def test_convertnii_matches_reference_layout(tmp_path, code, cut):
    from tests.nifti import write_nifti
    rng = np.random.default_rng(3)
    mask = (rng.random((5, 4, 3)) > 0.5).astype(np.uint8) if code == 2 else rng.random((5, 4, 3)).astype(np.float32)
    write_nifti(tmp_path / "mask.nii", mask, code)
    flat = _flat(mask).astype(np.float32)
    c = 0.5 if cut is None else cut
    n = int((flat >= c).sum())
    d = tmp_path / "nm"
    d.mkdir()
    x = rng.standard_normal(n).astype(np.float32)
    _write_nm(d / "subj_deg.nm", x)
    _write_nm(d / "bad_cp.nm", x[:-1])            # wrong length: skipped and logged
    (d / "notes.nmx").write_bytes(b"x")            # other extensions are ignored
    args = [os.path.join(BIN, "ConvertNII"), str(d), str(tmp_path / "mask.nii")] + ([] if cut is None else [str(cut)])
    p = subprocess.run(args, capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert p.returncode == 0, p.stderr
    hdr = (tmp_path / "mask.nii").read_bytes()[:352]
    assert (d / "subj_deg.nii").read_bytes() == _convert_expected(flat, hdr, x, c)
    assert not (d / "bad_cp.nii").exists()
    assert "bad_cp.nm" in (tmp_path / "BNA_time_log").read_text()


def test_convertnii_robust_masks(tmp_path):
    """Big-endian mask, a mask with a header extension, a mask with value
    scaling: the voxels and values land as for the plain mask."""
    from tests.nifti import write_nifti
    rng = np.random.default_rng(5)
    m = (rng.random((6, 5, 2)) > 0.4).astype(np.float32)
    n = int(m.sum())
    x = rng.standard_normal(n).astype(np.float32)
    flat = _flat(m)
    want = np.zeros(flat.size, np.float32)
    want[flat >= 0.5] = x
    variants = {
        "big": dict(endian=">"),
        "ext": dict(extension=b"\x01\x00\x00\x00" + bytes(12)),
        "scaled": dict(slope=2.0, inter=0.0),    # stored 0.5 reads as 1.0
    }
    for name, kw in variants.items():
        d = tmp_path / name
        d.mkdir()
        stored = m / 2 if name == "scaled" else m
        write_nifti(d / "mask.nii", stored, 16, **kw)
        _write_nm(d / "v.nm", x)
        p = subprocess.run([os.path.join(BIN, "ConvertNII"), str(d), str(d / "mask.nii")], capture_output=True,
                           text=True, timeout=60, cwd=d)
        assert p.returncode == 0, p.stderr
        raw = (d / "v.nii").read_bytes()
        endian = ">" if name == "big" else "<"
        import struct
        assert struct.unpack_from(endian + "hh", raw, 70) == (16, 32)
        assert struct.unpack_from(endian + "f", raw, 108)[0] == 352.0
        if name == "scaled":
            assert struct.unpack_from("<ff", raw, 112) == (0.0, 0.0)
        got = np.frombuffer(raw[352:], np.dtype(np.float32).newbyteorder(endian))
        np.testing.assert_array_equal(got, want)


# ------------------------------------------------------- corrupt input files
def _csr_bytes(R, C, V=None):
    parts = [np.array([len(R)], np.int32), np.asarray(R, np.int32), np.array([len(C)], np.int32),
             np.asarray(C, np.int32)]
    if V is not None:
        parts += [np.array([len(V)], np.int32), np.asarray(V, np.float32)]
    return b"".join(p.tobytes() for p in parts)


_R = [0, 2, 3, 4]
_C = [1, 2, 0, 0]

CORRUPT_CSR = {
    "empty": (b"", "bad row header"),
    "truncated_rows": (_csr_bytes(_R, _C)[:10], "truncated row array"),
    "missing_columns": (_csr_bytes(_R, _C)[:20], "bad column header"),
    "truncated_columns": (_csr_bytes(_R, _C)[:-4], "truncated column array"),
    "negative_rows": (np.array([-3], np.int32).tobytes(), "bad row header"),
    "rowptr_mismatch": (_csr_bytes([0, 2, 3, 5], _C), "does not match the column count"),
    "decreasing_rows": (_csr_bytes([0, 3, 2, 4], _C), "row offsets decrease"),
    "column_out_of_range": (_csr_bytes(_R, [1, 7, 0, 0]), "column index out of range"),
    "value_length": (_csr_bytes(_R, _C) + np.array([3], np.int32).tobytes() + np.zeros(3, np.float32).tobytes(),
                     "value length differs"),
    "truncated_values": (_csr_bytes(_R, _C, [1, 1, 1, 1])[:-4], "truncated value array"),
}


@pytest.mark.parametrize("case", list(CORRUPT_CSR))
def test_corrupt_csr_is_rejected_before_any_gpu_work(tmp_path, case):
    """The .csr reader (the format of CorMat.cpp:285-294 / manual p10) checks
    every header, length and index; the Maslov tool reads its graph before it
    opens a GPU context, so a corrupt file ends with exit status 1 and the
    reason, on any machine."""
    data, msg = CORRUPT_CSR[case]
    path = tmp_path / f"{case}.csr"
    path.write_bytes(data)
    p = subprocess.run([os.path.join(BIN, "Maslov"), str(path)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1
    assert msg in p.stderr, p.stderr
    assert not (tmp_path / f"{case}_Maslov.csr").exists()


def test_corrupt_mask_nifti_is_rejected(tmp_path):
    """CUCorMat reads the mask before opening a GPU context: a truncated
    header, truncated data or an unsupported data type stop it with status 1."""
    from tests.nifti import write_nifti
    write_nifti(tmp_path / "mask.nii", np.ones((4, 4, 2), np.uint8), 2)
    full = (tmp_path / "mask.nii").read_bytes()
    cases = {"truncated NIfTI header": full[:200], "truncated data": full[:352 + 5]}
    bad_type = bytearray(full)
    bad_type[70:72] = np.array([128], np.int16).tobytes()        # RGB: not a supported type
    cases["data type is not"] = bytes(bad_type)
    for msg, data in cases.items():
        (tmp_path / "mask.nii").write_bytes(data)
        p = subprocess.run([os.path.join(BIN, "CUCorMat"), str(tmp_path), "0.5", "n", "n", "r", "0.3"],
                           capture_output=True, text=True, timeout=60)
        assert p.returncode == 1 and msg in p.stderr, (msg, p.stderr)
