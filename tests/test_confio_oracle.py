"""The oracle of BQCD's configuration files (conf.F90, comm/field_io_mpi.F90,
conf_info.F90, cksum.c), on CPU: its check sum against the system's POSIX
``cksum`` command, its byte layout against conf_seq's loop nest written out
site by site, and a write/read round trip with a corrupted file."""
import os
import subprocess

import numpy as np
import pytest

from oracle import confio


def system_cksum(path):
    out = subprocess.run(["cksum", path], capture_output=True, text=True, check=True).stdout.split()
    return int(out[0]), int(out[1])


@pytest.mark.parametrize("n", [0, 1, 7, 255, 256, 4099, 65536, (1 << 20) + 3])
def test_cksum_matches_the_cksum_command(tmp_path, n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    p = tmp_path / "x.bin"
    p.write_bytes(data)
    assert (confio.cksum(data), n) == system_cksum(str(p))


@pytest.fixture(scope="module")
def links(oracle):
    L = (4, 6, 2, 4)
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(7)
    return L, g, g.hot()


def test_slice_layout_follows_conf_seq(links):
    """Byte offset of u(c1, c2, mu) of site (x, y, z) in the file of slice t:
    records by z, then y, then x; 24 big-endian complex numbers per site
    with c1 fastest, then c2 (columns 1, 2), then mu."""
    L, g, u = links
    nx, ny, nz, nt = L
    for t in (0, nt - 1):
        data = confio.slice_bytes(L, u, t)
        assert len(data) == nx * ny * nz * 24 * 16
        for (x, y, z) in [(0, 0, 0), (nx - 1, 1, 0), (1, ny - 1, nz - 1), (2, 3, 1)]:
            ilex = x + nx * (y + ny * (z + nz * t))
            i, eo = ilex // 2, (x + y + z + t) % 2
            site = ((z * ny + y) * nx + x) * 24
            for mu in range(4):
                for c2 in range(2):
                    for c1 in range(3):
                        off = (site + (mu * 2 + c2) * 3 + c1) * 16
                        re, im = np.frombuffer(data[off:off + 16], dtype=">f8")
                        assert re == u[mu, eo, i, c2, c1].real and im == u[mu, eo, i, c2, c1].imag


def test_round_trip_rebuilds_the_third_column(links, tmp_path):
    L, g, u = links
    base = str(tmp_path / "conf")
    meta = dict(run=1, traj=10, ensemble=(1, 1), beta=(5.29, 5.29), kappa=(0.13, 0.13), csw=(1.9192, 1.9192),
                csw_kappa=(0.249496, 0.249496), h=(0.0, 0.0))
    sums = confio.write(base, L, (1, 1, 1, -1), u, 0.5, meta)
    for t, (name, s, n) in enumerate(sums):
        assert (s, n) == system_cksum(os.path.join(str(tmp_path), name))
    v, keys = confio.read(base + ".info", L, g.volh)
    assert np.abs(v - u).max() < 1e-14
    assert [int(x) for x in keys["bc_fermions"]] == [1, 1, 1, -1]
    # one flipped byte in one slice is caught by its check sum
    name = os.path.join(str(tmp_path), sums[2][0])
    data = bytearray(open(name, "rb").read())
    data[1000] ^= 0x10
    open(name, "wb").write(bytes(data))
    with pytest.raises(ValueError):
        confio.read(base + ".info", L, g.volh)
