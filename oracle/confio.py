"""Configuration files of BQCD -- TEST INFRASTRUCTURE ONLY (the oracle of the
device reader and writer; only tests/ use it).

A restatement in numpy of the file layout that conf_write / conf_read
(conf.F90:219-470) produce through conf_seq (conf.F90:219-259) and
field_io (comm/field_io_mpi.F90:28-190, single PE), and of the info file of
conf_info.F90:28-190:

* one binary file per time slice t, named ``<base>.<tt>.u`` (files.F90:219-234
  with the time as i2.2);
* the file holds NZ records, one per z; a record runs over y, then x, and
  each site holds u_io(c1, c2, mu) for rows c1 = 1..3 (fastest), the first
  two columns c2 = 1, 2 and mu = 1..4 (x, y, z, t): 24 complex numbers as
  big-endian REAL(8) pairs (swap_endian8, misc.F90:197-240);
* the third column is not stored; reading rebuilds it with u_complete
  (su3.F90:301-310);
* the info file ``<base>.info`` holds the ConfInfoHeader block (the format
  version 3 of module_bqcd.F90:38, lattice, boundary conditions, REAL kind,
  PlaqEnergy, and two ensembles' parameters) and the CheckSum block with one
  line per slice: the file name, its POSIX cksum and its byte count
  (write_cksum, conf_info.F90:165-190);
* the check sum is POSIX.2 cksum (cksum.c), restated in oracle_capi.c and
  pinned against the system's ``cksum`` command by the tests.

Links use the oracle's numpy convention: complex128 (4, 2, volh, 3, 3),
[mu][eo][site][col][row], sites in BQCD's even/odd order (index.F90:58-76).
"""
import os

import numpy as np

from . import oracle as _o

CONF_INFO_VERSION = 3


def cksum(data):
    """POSIX cksum of a bytes-like object (cksum.c:130-165)."""
    buf = np.frombuffer(bytes(data), dtype=np.uint8)
    return int(_o.lib().oqc_cksum(buf.ctypes.data, buf.size))


def _slice_sites(L, t):
    """even/odd index and parity of the sites of time slice t in file order
    (z outermost, then y, then x)."""
    nx, ny, nz, _ = L
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ilex = x + nx * (y + ny * (z + nz * t))
    return (ilex // 2).ravel(), ((x + y + z + t) % 2).ravel()


def slice_bytes(L, u, t):
    """The bytes of the file of time slice t (conf_seq + field_io)."""
    i, eo = _slice_sites(L, t)
    sites = u[:, eo, i, 0:2, :]                 # (mu, site, col 1..2, row)
    rec = np.ascontiguousarray(np.transpose(sites, (1, 0, 2, 3)))   # (site, mu, col, row)
    return rec.astype(">c16").tobytes()


def slice_to_links(L, data, t, u):
    """Fill the sites of slice t of u from the file bytes (the inverse of
    slice_bytes), rebuilding the third column with u_complete."""
    i, eo = _slice_sites(L, t)
    rec = np.frombuffer(data, dtype=">c16").astype(np.complex128).reshape(len(i), 4, 2, 3)
    m = np.zeros((len(i), 4, 3, 3), np.complex128)
    m[:, :, 0:2, :] = rec
    c1, c2 = m[:, :, 0, :], m[:, :, 1, :]       # [.., row] of columns 1 and 2
    m[:, :, 2, 0] = np.conj(c1[..., 1] * c2[..., 2] - c1[..., 2] * c2[..., 1])
    m[:, :, 2, 1] = np.conj(c1[..., 2] * c2[..., 0] - c1[..., 0] * c2[..., 2])
    m[:, :, 2, 2] = np.conj(c1[..., 0] * c2[..., 1] - c1[..., 1] * c2[..., 0])
    u[:, eo, i] = np.transpose(m, (1, 0, 2, 3))


def slice_name(base, t):
    return "%s.%02d.u" % (base, t)


def write(base, L, bc, u, plaq_energy, meta):
    """Write the slice files and the info file of configuration u.
    meta: run, traj, ensemble (2), beta, kappa, csw, csw_kappa, h (2 each)."""
    sums = []
    for t in range(L[3]):
        data = slice_bytes(L, u, t)
        name = slice_name(base, t)
        with open(name, "wb") as f:
            f.write(data)
        sums.append((os.path.basename(name), cksum(data), len(data)))
    with open(base + ".info", "w") as f:
        f.write(info_text(L, bc, plaq_energy, meta, sums))
    return sums


def info_text(L, bc, plaq_energy, meta, sums):
    """The info file: the header block and the check-sum block."""
    lines = [" >BeginConfInfoHeader",
             " Format %d" % CONF_INFO_VERSION,
             " Program bqcd-b200 1",
             " Run %d" % meta["run"],
             " Traj %d" % meta["traj"],
             " Host b200",
             " Date - -",
             " L" + "".join("%3d" % v for v in L),
             " bc_fermions" + "".join("%3d" % v for v in bc),
             " REAL_kind 8",
             " PlaqEnergy %25.14E" % plaq_energy]
    names = [("ensemble", "beta", "kappa", "csw", "csw_kappa", "h"),
             ("former_ensemble", "former_beta", "former_kappa", "former_csw", "former_csw_kappa", "former_h")]
    for k in range(2):
        lines.append(" %s %d" % (names[k][0], meta["ensemble"][k]))
        for key, name in zip(("beta", "kappa", "csw", "csw_kappa", "h"), names[k][1:]):
            lines.append(" %s %.17g" % (name, meta[key][k]))
    lines.append(" >EndConfInfoHeader")
    lines.append(" >BeginCheckSum")
    for name, s, n in sums:
        lines.append(" %s %d %d" % (name, s, n))
    lines.append(" >EndCheckSum")
    return "\n".join(lines) + "\n"


def read_info(path):
    """Keyword values of the header and the check-sum lines (read_keyword_*,
    read_cksum of conf_info.F90:65-160)."""
    keys, sums = {}, []
    block = None
    with open(path) as f:
        for line in f:
            w = line.split()
            if not w:
                continue
            if w[0].startswith(">Begin"):
                block = w[0][6:]
                continue
            if w[0].startswith(">End"):
                block = None
                continue
            if block == "CheckSum":
                sums.append((w[0], int(w[1]), int(w[2]) if len(w) > 2 else None))
            elif block == "ConfInfoHeader":
                keys[w[0]] = w[1:]
    return keys, sums


def read(info_path, L, volh):
    """Links of a configuration written by write() or by the device."""
    keys, sums = read_info(info_path)
    if int(keys["Format"][0]) != CONF_INFO_VERSION:
        raise ValueError("wrong file format")
    if [int(v) for v in keys["L"]] != list(L):
        raise ValueError("L inconsistent")
    u = np.zeros((4, 2, volh, 3, 3), np.complex128)
    d = os.path.dirname(info_path)
    for t, (name, s, _) in enumerate(sums):
        with open(os.path.join(d, name), "rb") as f:
            data = f.read()
        if cksum(data) != s:
            raise ValueError("check sum error in file " + name)
        slice_to_links(L, data, t, u)
    return u, keys
