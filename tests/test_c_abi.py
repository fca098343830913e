"""A plain C program (tests/c_abi_smoke.c) drives the C ABI: the header compiles
as C99 and the program links against libvqemps.so (CPU); on a GPU it runs the
two-qubit known answer of the reference's install checks (1e-10), sampling and
the error path."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "graph-vqe_b200" / "vqemps"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def _build(out):
    from vqemps import build
    build.build()
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.fail("no C compiler found")
    cmd = [cc, "-std=c99", "-Wall", "-Werror", "-O1", str(ROOT / "tests" / "c_abi_smoke.c"), "-o", str(out),
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", f"-L{LIBDIR}", "-lvqemps",
           f"-L{CUDA / 'lib64'}", "-lcudart", "-lm", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return out


def test_c_caller_compiles_and_links(tmp_path):
    assert _build(tmp_path / "c_abi_smoke").exists()


@pytest.mark.gpu
def test_c_caller_runs_known_answer(tmp_path, cuda_device):
    exe = _build(tmp_path / "c_abi_smoke")
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "all checks passed" in res.stdout
