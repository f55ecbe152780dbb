"""The C++ drop-in headers (gshtrans_b200/cpp/GSHTrans): they compile against
the reference's interface as its tests use it and link to libgsht_cuda.so
(CPU); the checks program then runs on the GPU (coefficient round trips,
Legendre values, the addition theorem, fused field expressions)."""

import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
LIB_DIR = ROOT / "gshtrans_b200"
SOURCE = ROOT / "tests" / "cpp" / "dropin_checks.cpp"


def _compile(out_dir: pathlib.Path) -> pathlib.Path:
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not (LIB_DIR / "libgsht_cuda.so").exists():
        pytest.fail("libgsht_cuda.so is not built")
    exe = out_dir / "dropin_checks"
    cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror",
           f"-I{LIB_DIR / 'cpp'}", f"-I{ROOT / 'include'}", str(SOURCE),
           f"-L{LIB_DIR}", "-lgsht_cuda", f"-Wl,-rpath,{LIB_DIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_dropin_headers_compile_and_link(tmp_path):
    exe = _compile(tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_dropin_checks_run(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "0 failed" in r.stdout
