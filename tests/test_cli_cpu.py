"""The reference-compatible CLI tools: built, and argument errors are
reported before any GPU work (CPU only)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "pagani-toolkit_b200", "bin")
TOOLS = ["CUCorMat", "CUCorMat_weighted", "Degree", "Cp", "BFS_MulCPU", "CUBFW_Lp", "CUBC",
         "Newman_Modularity", "CUEC", "Maslov", "SmallWorldProperty"]


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
