"""The C ABI from plain C (tests/c_client/trisk_client.c): built with gcc against
include/trisk_b200.h and linked to libtrisk_b200.so and the C oracle, as a non-Python caller
would bind them. On CPU it checks the struct layouts, error reporting, mesh and grid
generation, the host-side tables, and that creating a model fails loudly without a GPU; on
the GPU the tendency and RK4 steps through the ABI equal the oracle bit for bit."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    lib = os.path.join(ROOT, "dmplex_b200", "lib")
    oracle = os.path.join(ROOT, "oracle")
    exe = str(tmp_path / "trisk_client")
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-D_DEFAULT_SOURCE",
           os.path.join(ROOT, "tests", "c_client", "trisk_client.c"),
           "-I", os.path.join(ROOT, "include"), "-I", oracle,
           "-L", lib, "-ltrisk_b200", "-L", oracle, "-ltrisk_oracle", "-lm",
           f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{oracle}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_c_client_on_cpu(tmp_path):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present: the GPU form runs instead")
    out = subprocess.run([_build(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "cpu ok"


@pytest.mark.gpu
def test_c_client_on_gpu(require_gpu, tmp_path):
    out = subprocess.run([_build(tmp_path), "gpu"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "gpu ok"
