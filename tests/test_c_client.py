"""The C ABI from a plain C99 program (tests/c_client/abi_client.c): the
header compiles as C with warnings as errors, the program links against the
library, and it runs -- without a device it checks the documented status
codes; with one (-m gpu) it solves M^+M x = b on a 4^4 cold configuration."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "bqcd-r399-quda_b200", "lib")


@pytest.fixture(scope="module")
def client(tmp_path_factory):
    import importlib.util
    spec = importlib.util.spec_from_file_location("bqbuild", os.path.join(ROOT, "bqcd-r399-quda_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    m.build()
    exe = str(tmp_path_factory.mktemp("c") / "abi_client")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_client", "abi_client.c"), "-L", LIBDIR, "-lbqcdg",
                    "-Wl,-rpath," + LIBDIR, "-lm", "-o", exe], check=True)
    return exe


def test_c_client_without_device(client):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    out = subprocess.run([client], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok (no device)"


@pytest.mark.gpu
def test_c_client_on_device(client):
    out = subprocess.run([client], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok (device)"
