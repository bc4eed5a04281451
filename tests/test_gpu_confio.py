"""BQCD configuration files written and read on the device (conf.F90:219-470,
comm/field_io_mpi.F90, conf_info.F90, cksum.c) against the oracle's
restatement of the format: byte-identical slice files, check sums equal to
the system's POSIX cksum, round trips, and the error paths of conf_read."""
import os
import subprocess

import numpy as np
import pytest

from oracle import confio

pytestmark = pytest.mark.gpu

META = dict(run=3, traj=120, ensemble=(1, 1), beta=(5.29, 5.29), kappa=(0.13, 0.13), csw=(1.9192, 1.9192),
            csw_kappa=(1.9192 * 0.13, 1.9192 * 0.13), h=(0.0, 0.0))


def system_cksum(path):
    out = subprocess.run(["cksum", path], capture_output=True, text=True, check=True).stdout.split()
    return int(out[0]), int(out[1])


@pytest.fixture(params=[(4, 6, 2, 4), (6, 6, 6, 6), (16, 16, 16, 4)], ids=lambda L: "x".join(map(str, L)))
def system(request, oracle, bq):
    L = request.param
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(11)
    u = g.hot()
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.load_gauge(u, flipped=False)
    yield L, g, u, lat
    lat.close()


def test_device_writer_matches_the_format(system, tmp_path, bq):
    """Every slice file equals the oracle's bytes, and the info file lists
    the cksum and size of each as the cksum command computes them."""
    L, g, u, lat = system
    base = str(tmp_path / "bqcd.003.1.1.00120")
    para = bq.HmcPara(kappa=0.13, csw=1.9192)
    meta = lat.conf_write(base, run=3, traj=120, para=para, beta=5.29)
    assert meta["L"] == list(L) and meta["bc"] == [1, 1, 1, -1]
    assert abs(meta["plaq_energy"] - g.sg(u) / (6.0 * 2 * g.volh)) < 1e-12
    keys, sums = confio.read_info(base + ".info")
    assert [int(v) for v in keys["L"]] == list(L) and int(keys["Format"][0]) == 3
    assert len(sums) == L[3]
    for t in range(L[3]):
        name = confio.slice_name(base, t)
        data = open(name, "rb").read()
        assert data == confio.slice_bytes(L, u, t), t
        assert sums[t][0] == os.path.basename(name)
        assert (sums[t][1], sums[t][2]) == system_cksum(name)


def test_device_reader_round_trip(system, tmp_path, bq):
    """Files written by the oracle are read back on the device: the links
    (third columns rebuilt by u_complete) and the operator built on them
    equal the originals."""
    L, g, u, lat = system
    base = str(tmp_path / "conf")
    confio.write(base, L, (1, 1, 1, -1), u, 0.5, META)
    other = bq.Lattice(L, (1, 1, 1, -1))
    meta = other.conf_read(base + ".info")
    assert meta["run"] == 3 and meta["traj"] == 120 and meta["bc"] == [1, 1, 1, -1]
    assert abs(meta["kappa"][0] - 0.13) < 1e-15 and abs(meta["plaq_energy"] - 0.5) < 1e-14
    v = other.get_gauge(flipped=False)
    assert np.abs(v - u).max() < 1e-14
    psi = g.gauss_spinor(1)
    ref = g.d(0, 1, psi, g.flip_bc(u.copy()))
    got = other.d(0, 1, psi)
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)
    other.close()


def test_reader_errors(oracle, bq, tmp_path):
    """A flipped byte gives BQCDG_ECHECKSUM and leaves no links loaded; a
    configuration of another lattice gives BQCDG_EINVAL; a missing slice
    file gives BQCDG_EIO."""
    L = (4, 4, 4, 4)
    g = oracle.Geom(L, (1, 1, 1, -1))
    oracle.ranset(3)
    u = g.hot()
    base = str(tmp_path / "c")
    sums = confio.write(base, L, (1, 1, 1, -1), u, 0.5, META)
    lat = bq.Lattice(L, (1, 1, 1, -1))
    lat.conf_read(base + ".info")
    name = str(tmp_path / sums[1][0])
    data = bytearray(open(name, "rb").read())
    data[5] ^= 0x01
    open(name, "wb").write(bytes(data))
    with pytest.raises(bq.BqcdgError) as e:
        lat.conf_read(base + ".info")
    assert e.value.status == bq.ECHECKSUM
    with pytest.raises(bq.BqcdgError) as e:
        lat.sg()
    assert e.value.status == bq.ENOGAUGE
    os.remove(name)
    with pytest.raises(bq.BqcdgError) as e:
        lat.conf_read(base + ".info")
    assert e.value.status == bq.EIO
    lat.close()
    other = bq.Lattice((4, 4, 4, 8), (1, 1, 1, -1))
    with pytest.raises(bq.BqcdgError) as e:
        other.conf_read(base + ".info")
    assert e.value.status == bq.EINVAL
    other.close()
