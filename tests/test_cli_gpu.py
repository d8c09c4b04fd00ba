"""The reference-compatible CLI tools end to end on the GPU: NIfTI in,
.csr/.nm/.modu/.txt out with the reference's names, contents checked against
the oracle."""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth
from tests.nifti import volume_from_series, write_nifti

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "pagani-toolkit_b200", "bin")


def run(*args, cwd=None):
    p = subprocess.run([os.path.join(BIN, args[0]), *map(str, args[1:])], capture_output=True, text=True,
                       timeout=600, cwd=cwd)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def read_csr(path):
    raw = np.fromfile(path, np.int32)
    rl = raw[0]
    R = raw[1:1 + rl]
    cl = raw[1 + rl]
    C = raw[2 + rl:2 + rl + cl]
    V = raw[3 + rl + cl:].view(np.float32) if len(raw) > 2 + rl + cl else None
    return R, C, V


def read_nm(path):
    raw = np.fromfile(path, np.int32)
    return raw[1:].view(np.float32)


@pytest.fixture(scope="module")
def subject_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("bold")
    N, T, shape = 600, 150, (10, 10, 7)
    mask = np.zeros(shape, np.uint8)
    flat = np.zeros(np.prod(shape), np.uint8)
    flat[:N] = 1
    mask[:] = flat.reshape(shape[2], shape[1], shape[0]).transpose(2, 1, 0)
    write_nifti(d / "mask.nii", mask, 2)
    bold = synth.bold_series(N, T, 10, 777)
    write_nifti(d / "subj01.nii", volume_from_series(bold, shape), 16)
    return d, bold


def test_cucormat_r_and_s(subject_dir):
    d, bold = subject_dir
    run("CUCorMat", d, 0.5, "n", "y", "r", 0.3)
    run("CUCorMat", d, 0.5, "n", "n", "s", 2)
    N = bold.shape[1]
    z, _ = O.zscore(bold)
    r = O.corr_packed(z)
    Ro, Co, _ = O.graph_r(r, N, np.float32(0.3))
    s_r = 100.0 * len(Co) / (N * (N - 1) // 2) / 2
    f_r = d / f"subj01_{N}_spa{np.float32(s_r):.3f}%_cor0.300.csr"
    R, C, V = read_csr(f_r)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co) and V is None
    cm = np.fromfile(d / f"subj01_{N}.cormat", np.float32)[1:]
    assert np.max(np.abs(cm - r)) < 1e-6
    k = O.sparsity_k(N, 2.0)
    Rk, Ck, _, tau = O.graph_k(r, N, k)
    f_s = glob.glob(str(d / f"subj01_{N}_spa2.000%_cor*.csr"))
    assert len(f_s) == 1
    R, C, _ = read_csr(f_s[0])
    assert np.array_equal(R, Rk) and np.array_equal(C, Ck)


def test_metric_tools(subject_dir, tmp_path):
    d, bold = subject_dir
    N = bold.shape[1]
    z, _ = O.zscore(bold)
    R, C, _ = O.graph_r(O.corr_packed(z), N, 0.3)
    g = tmp_path / "g"
    g.mkdir()
    raw = np.concatenate([[len(R)], R, [len(C)], C]).astype(np.int32)
    raw.tofile(g / "net.csr")
    run("Degree", g)
    assert np.array_equal(read_nm(g / "net_deg.nm"), O.degree(R)[0])
    run("Cp", g, 2, "gnk")
    assert np.array_equal(read_nm(g / "net_cp.nm"), O.cp_binary(R, C)[1])
    assert len(open(g / "net_cp.txt").read().split()) == 3 and (g / "net_gamma.txt").exists()
    run("BFS_MulCPU", g, 1, "b")
    inv, _, lp, _ = O.bfs_paths(R, C)
    np.testing.assert_allclose(read_nm(g / "net_eff.nm"), inv / (N - 1), rtol=1e-6)
    assert float(open(g / "net_Lp.txt").read().split()[0]) == pytest.approx(lp, rel=1e-5)
    run("CUBC", g)
    np.testing.assert_allclose(read_nm(g / "net_bc.nm"), O.brandes(R, C), rtol=1e-6, atol=1e-3)
    run("Newman_Modularity", g, 0)
    lab = np.fromfile(g / "net.modu", np.int32)[1:]
    assert np.array_equal(lab, O.newman(R, C)[0])
    assert "Round:" in open(g / "net_modu.txt").read()
    run("Maslov", g / "net.csr")
    R2, C2, _ = read_csr(g / "net_Maslov.csr")
    assert np.array_equal(np.diff(R2), np.diff(R))


def test_weighted_tools_and_smallworld(subject_dir, tmp_path):
    d, bold = subject_dir
    w = tmp_path / "w"
    w.mkdir()
    for f in ("mask.nii", "subj01.nii"):
        os.symlink(d / f, w / f)
    run("CUCorMat_weighted", w, 0.5, "n", "n", "r", 0.25)
    files = glob.glob(str(w / "*_weighted.csr"))
    assert len(files) == 1
    R, C, V = read_csr(files[0])
    N = bold.shape[1]
    z, _ = O.zscore(bold)
    r = O.corr_packed(z, weighted=True)
    Ro, Co, Vo = O.graph_r(r, N, O.weighted_r_threshold(np.float32(0.25)), weighted=True)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co)
    assert np.array_equal(V, Vo)                   # V = float(FP64 r) for every edge
    gdir = tmp_path / "wg"
    gdir.mkdir()
    os.symlink(files[0], gdir / os.path.basename(files[0]))
    run("CUBFW_Lp", gdir, 2, "gnl")
    run("Cp", gdir, 2, "2", "gnk")
    run("SmallWorldProperty", gdir)
    sw = glob.glob(str(gdir / "*_smallWorld.txt"))
    assert len(sw) == 1
    lam = float(open(glob.glob(str(gdir / "*_lambda.txt"))[0]).read())
    gam = float(open(glob.glob(str(gdir / "*_gamma.txt"))[0]).read())
    assert float(open(sw[0]).read()) == pytest.approx(gam / lam, rel=1e-5)


def write_csr(path, R, C, V=None):
    with open(path, "wb") as f:
        np.array([len(R)], np.int32).tofile(f)
        np.asarray(R, np.int32).tofile(f)
        np.array([len(C)], np.int32).tofile(f)
        np.asarray(C, np.int32).tofile(f)
        if V is not None:
            np.array([len(V)], np.int32).tofile(f)
            np.asarray(V, np.float32).tofile(f)


def test_cuec_unweighted_and_weighted(tmp_path):
    from tests import graphs as G
    Ru, Cu, _ = G.from_bold(500, 150, 0.3, 41)
    Rw, Cw, Vw = G.from_bold(450, 150, 0.25, 42, weighted=True)
    write_csr(tmp_path / "bin_500.csr", Ru, Cu)
    write_csr(tmp_path / "wei_450.csr", Rw, Cw, Vw)
    run("CUEC", tmp_path)
    for stem, (R, C, V) in (("bin_500", (Ru, Cu, None)), ("wei_450", (Rw, Cw, Vw))):
        ec = read_nm(tmp_path / f"{stem}_ec.nm")
        ec_or, lam_or, it_or, _ = O.eigen_centrality(R, C, V, raw=V is not None)
        np.testing.assert_allclose(ec, ec_or.astype(np.float32), rtol=1e-5, atol=1e-7)
        lam = float(open(tmp_path / f"{stem}_evalue.txt").read().split()[0])
        assert lam == pytest.approx(lam_or, rel=1e-5)


def test_cucormat_robust_nifti_inputs(tmp_path):
    """The same subject stored big-endian, with a header extension, and as
    halved values with scl_slope 2: CUCorMat writes byte-identical graphs."""
    N, T, shape = 400, 120, (10, 8, 5)
    bold = synth.bold_series(N, T, 10, 4242)
    mask = np.zeros(shape, np.uint8)
    flat = np.zeros(np.prod(shape), np.uint8)
    flat[:N] = 1
    mask[:] = flat.reshape(shape[2], shape[1], shape[0]).transpose(2, 1, 0)
    vol = volume_from_series(bold, shape)
    variants = {"plain": {}, "big": dict(endian=">"), "ext": dict(extension=b"\x01\x00\x00\x00" + bytes(28)),
                "scaled": dict(slope=2.0)}
    out = {}
    for name, kw in variants.items():
        d = tmp_path / name
        d.mkdir()
        write_nifti(d / "mask.nii", mask, 2, **({"endian": kw["endian"]} if "endian" in kw else {}))
        write_nifti(d / "subj01.nii", vol / 2 if name == "scaled" else vol, 16, **kw)
        run("CUCorMat", d, 0.5, "n", "n", "s", 2)
        f = glob.glob(str(d / f"subj01_{N}_spa2.000%_cor*.csr"))
        assert len(f) == 1
        out[name] = open(f[0], "rb").read()
    for name in variants:
        assert out[name] == out["plain"], name


def test_pc_cpu_tool(tmp_path):
    from tests import graphs as G
    R, C, V = G.from_bold(500, 150, 0.25, 43, weighted=True)
    n = len(R) - 1
    mod = np.random.default_rng(7).integers(1, 12, n).astype(np.float32)
    write_csr(tmp_path / "s1.csr", R, C, V)
    with open(tmp_path / "s1_modu.nm", "wb") as f:
        np.array([n], np.int32).tofile(f)
        mod.tofile(f)
    write_csr(tmp_path / "s2.csr", R, C, V)      # no module file: skipped
    run("PC_CPU", tmp_path)
    pc_or, pn_or, _ = O.participation(R, C, V, mod)
    assert np.array_equal(read_nm(tmp_path / "s1_pc.nm"), pc_or)
    assert np.array_equal(read_nm(tmp_path / "s1_pc.nm_Normalized.nm"), pn_or)
    assert not (tmp_path / "s2_pc.nm").exists()


def test_newman_weighted_tool(tmp_path):
    """Newman_Modularity_weighted: float labels in X_modu.nm equal to the
    oracle's weighted partition; a file without values is skipped."""
    from tests import graphs as G
    R, C, V = G.from_bold(400, 120, 0.25, 44, weighted=True)
    write_csr(tmp_path / "w1.csr", R, C, V)
    write_csr(tmp_path / "b1.csr", R, C)
    run("Newman_Modularity_weighted", tmp_path, 1)
    lab, Q, nm = O.newman_weighted(R, C, V)
    assert np.array_equal(read_nm(tmp_path / "w1_modu.nm"), lab.astype(np.float32))
    assert "Round:" in open(tmp_path / "w1_modu.txt").read()
    assert not (tmp_path / "b1_modu.nm").exists()


@pytest.mark.parametrize("tool,avg,mode,thr", [("CUCorMat", "bf", "s", 2.0), ("CUCorMat_weighted", "yn", "r", 0.15)])
def test_cucormat_subject_average(tmp_path, tool, avg, mode, thr):
    """to_average: the averaged graph and .cormat (named after the directory,
    with the subject count) equal the oracle's cohort average; bf also writes
    every subject's own graph."""
    N, shape = 500, (10, 10, 6)
    d = tmp_path / "cohortdir"
    d.mkdir()
    mask = np.zeros(shape, np.uint8)
    flat = np.zeros(np.prod(shape), np.uint8)
    flat[:N] = 1
    mask[:] = flat.reshape(shape[2], shape[1], shape[0]).transpose(2, 1, 0)
    write_nifti(d / "mask.nii", mask, 2)
    bolds = [synth.bold_series(N, T, 10, 5150 + T) for T in (120, 90)]
    for k, b in enumerate(bolds):
        write_nifti(d / f"s{k}.nii", volume_from_series(b, shape), 16)
    run(tool, d, 0.5, avg, "y", mode, thr)
    weighted = tool.endswith("weighted")
    keys = O.cohort_keys(bolds, fisher=avg[1] == "f", weighted=weighted)
    base = f"cohortdir_2_{N}"
    cm = np.fromfile(d / f"{base}.cormat", np.float32)
    assert np.frombuffer(open(d / f"{base}.cormat", "rb").read(4), np.int32)[0] == N * (N - 1) // 2
    assert np.array_equal(cm[1:], keys.astype(np.float32))
    if mode == "s":
        Ro, Co, _, tau = O.graph_k(keys, N, O.sparsity_k(N, thr), weighted=weighted)
        f = d / f"{base}_spa{thr:.3f}%_cor{np.float32(tau):.3f}.csr"
    else:
        Ro, Co, Vo = O.graph_r(keys, N, thr, weighted=weighted)
        s = np.float32(100.0 * len(Co) / (N * (N - 1) // 2) / 2)
        f = d / f"{base}_spa{s:.3f}%_cor{thr:.3f}.csr"
    R, C, V = read_csr(f)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co)
    if weighted:
        assert np.array_equal(V, Vo)
    per_subject = glob.glob(str(d / "s*_500_spa*.csr"))
    assert len(per_subject) == (2 if avg[0] == "b" else 0)


def test_cucormat_volume_size_mismatch(tmp_path):
    """A subject whose volume differs from the mask is skipped with a message
    in per-subject mode (the others are processed) and stops an averaging run
    (the average would silently lose a subject)."""
    N, T, shape = 300, 80, (10, 10, 3)
    flat = np.zeros(np.prod(shape), np.uint8)
    flat[:N] = 1
    write_nifti(tmp_path / "mask.nii", flat.reshape(shape[2], shape[1], shape[0]).transpose(2, 1, 0), 2)
    good = synth.bold_series(N, T, 6, 901)
    write_nifti(tmp_path / "a_good.nii", volume_from_series(good, shape), 16)
    write_nifti(tmp_path / "b_bad.nii", volume_from_series(synth.bold_series(N, T, 6, 902), (10, 10, 4)), 16)
    p = subprocess.run([os.path.join(BIN, "CUCorMat"), str(tmp_path), "0.5", "n", "n", "r", "0.3"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0
    assert "volume size differs from the mask" in p.stderr
    assert glob.glob(str(tmp_path / "a_good_*.csr")) and not glob.glob(str(tmp_path / "b_bad_*.csr"))
    p = subprocess.run([os.path.join(BIN, "CUCorMat"), str(tmp_path), "0.5", "yn", "n", "r", "0.3"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 1 and "volume size differs from the mask" in p.stderr
