"""The stencil kernels' index arithmetic against BQCD's neighbour table, on
CPU.  The kernels read no nn table: they compute each neighbour from the
site index (site_coords / neighbour in csrc/bqcdg_internal.cuh, with a
multiply-shift division) and apply the fermion boundary sign by hop_sign.
Those same functions, compiled for the host by nvcc in
tests/c_client/neighbour_map.cu, must reproduce the oracle's nn(volh, 0:1,
4, 0:1) of init_common.F90:43-205 exactly, and their signs must be those of
flip_bc.F90:97-121 on the link each hop uses (forward: U_mu(x); backward:
U_mu(x - mu) of the other parity)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ragged (6^4, x/2 odd), extent 2 (forward and backward x-neighbours
# coincide), and the benchmark's 32^3x64
LATTICES = [(4, 4, 4, 4), (6, 4, 8, 4), (8, 8, 8, 8), (6, 6, 6, 6), (2, 4, 6, 4), (10, 6, 2, 8),
            (32, 32, 32, 64)]


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("nn") / "neighbour_map")
    subprocess.run([os.environ.get("NVCC", "nvcc"), "-std=c++17", "-O1", "-o", out,
                    os.path.join(ROOT, "tests", "c_client", "neighbour_map.cu")], check=True)
    return out


@pytest.mark.parametrize("L", LATTICES, ids=lambda L: "x".join(map(str, L)))
def test_kernel_neighbours_and_signs_equal_bqcd_tables(exe, oracle, tmp_path, L):
    g = oracle.Geom(L, (1, 1, 1, -1))
    volh = g.volh
    f = str(tmp_path / "nn.bin")
    subprocess.run([exe, *map(str, L), "-1", f], check=True)
    tab = np.fromfile(f, dtype=np.int32).reshape(2, 2, 4, 2, volh)     # [nn|sign][fb][mu][eo][i]
    import ctypes as C
    fn = oracle.lib().oqc_nn
    fn.argtypes, fn.restype = [C.c_void_p], C.POINTER(C.c_int)
    ref = np.ctypeslib.as_array(fn(g.h), shape=(2 * 4 * 2 * volh,)).reshape(2, 4, 2, volh).copy()
    assert np.array_equal(tab[0], ref)
    # the sign of each hop = the sign flip_bc puts on the link it uses
    u = np.zeros((4, 2, volh, 3, 3), np.complex128)
    u[..., 0, 0] = 1.0
    g.flip_bc(u)
    s = u[..., 0, 0].real.astype(np.int32)                              # [mu][eo][i]
    fwd = s
    bwd = np.stack([np.stack([s[mu, 1 - eo][ref[1, mu, eo]] for eo in range(2)]) for mu in range(4)])
    assert np.array_equal(tab[1, 0], fwd)
    assert np.array_equal(tab[1, 1], bwd)
