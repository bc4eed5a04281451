"""The time-slab domain decomposition on CPU: the face packing, the exchange
pattern and the ghost-aware neighbour map of the slab kernels, run as gloo
ranks.

The slab kernels' index functions (csrc/decomp.cuh, with neighbour /
hop_sign of csrc/bqcdg_internal.cuh) are compiled for the host in
tests/c_client/dd_maps.cu.  Each rank takes its slab of a global odd-site
spinor and of the periodic links, packs the two faces with those maps
(spins of the first slice for rank-1, of the last slice for rank+1,
comm/xbound_mpi.F90:418-461), sends them and U_t of its last slice over gloo,
and evaluates the hopping term D_eo (d/D21.F90:29-77) of its even sites in
numpy, reading each neighbour where the map says: a local site, or an entry of
a received face.  The slabs together must equal the oracle's single-domain
d / d_dag on BQCD's flipped links, to 1e-13."""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

S1 = np.array([[0, 1], [1, 0]], complex)
S2 = np.array([[0, -1j], [1j, 0]])
S3 = np.array([[1, 0], [0, -1]], complex)


def gammas():
    """BQCD's basis (d/D21xyzt.F90): gamma_k = [[0, i s_k], [-i s_k, 0]] for
    x, y, z and gamma_4 = diag(1, 1, -1, -1)."""
    g = []
    for s in (S1, S2, S3):
        m = np.zeros((4, 4), complex)
        m[:2, 2:] = 1j * s
        m[2:, :2] = -1j * s
        g.append(m)
    g.append(np.diag([1, 1, -1, -1]).astype(complex))
    return g


def build_maps(L, bct, nranks, rank, dag, tmpdir):
    exe = os.path.join(tmpdir, "dd_maps")
    if not os.path.exists(exe):
        subprocess.run([os.environ.get("NVCC", "nvcc"), "-std=c++17", "-O1", "-o", exe,
                        os.path.join(ROOT, "tests", "c_client", "dd_maps.cu")], check=True, capture_output=True)
    f = os.path.join(tmpdir, "m_%d_%d_%d.bin" % (nranks, rank, int(dag)))
    subprocess.run([exe, *map(str, L), str(bct), str(nranks), str(rank), str(int(dag)), f], check=True)
    V3h = L[0] * L[1] * L[2] // 2
    volh = V3h * (L[3] // nranks)
    a = np.fromfile(f, dtype=np.int32)
    site = a[:2 * V3h].reshape(2, V3h)
    comp = a[2 * V3h:2 * V3h + 12].reshape(2, 6)
    rest = a[2 * V3h + 12:]
    nb = rest[:8 * volh].reshape(4, 2, volh)
    sg = rest[8 * volh:].reshape(4, 2, volh)
    return site, comp, nb, sg


def pack(psi_loc, site, comp, side):
    """[6][V3h] face of one side: component k is colour comp // 4, spin comp % 4."""
    return np.stack([psi_loc[site[side], c // 4, c % 4] for c in comp[side]])


def slab_dslash(psi_loc, u_loc, ghost_fwd, ghost_bwd, ghost_link, comp, nb, sg, dag):
    """D_eo of the slab's even sites with the neighbours the map names."""
    G = gammas()
    one = np.eye(4)
    volh = nb.shape[2]
    out = np.zeros((volh, 3, 4), complex)
    for mu in range(4):
        for fb in range(2):
            j = nb[mu, fb]
            loc = j >= 0
            nbr = np.zeros((volh, 3, 4), complex)
            nbr[loc] = psi_loc[j[loc]]
            gh = ghost_fwd if fb == 0 else ghost_bwd
            face_comp = comp[0] if fb == 0 else comp[1]   # the sender's face layout
            for k, c in enumerate(face_comp):
                nbr[~loc, c // 4, c % 4] = gh[k][-1 - j[~loc]]
            if fb == 0:
                U = u_loc[mu, 0]                       # U_mu(x), even
                chi = np.einsum("icr,ics->irs", U, nbr)
                P = one + G[mu] if dag else one - G[mu]
            else:
                U = np.zeros((volh, 3, 3), complex)   # U_mu(x - mu), odd
                U[loc] = u_loc[mu, 1, j[loc]]
                U[~loc] = ghost_link[1][-1 - j[~loc]]
                chi = np.einsum("irc,ics->irs", np.conj(U), nbr)
                P = one - G[mu] if dag else one + G[mu]
            out += sg[mu, fb][:, None, None] * np.einsum("ts,irs->irt", P, chi)
    return out


def run_rank(rank, world, L, dag, tmpdir, exchange):
    from oracle import oracle as O
    g = O.Geom(L, (1, 1, 1, -1))
    O.ranset(0)
    u = g.hot()
    uf = g.flip_bc(u.copy())
    psi = g.gauss_spinor(1)
    ref = g.d(0, 1, psi, uf, dag)
    site, comp, nb, sg = build_maps(L, -1, world, rank, dag, tmpdir)
    volh = nb.shape[2]
    rows = slice(rank * volh, (rank + 1) * volh)
    psi_loc = psi[rows]
    u_loc = u[:, :, rows]
    to_prev, to_next = pack(psi_loc, site, comp, 0), pack(psi_loc, site, comp, 1)
    links_next = u_loc[3][:, site[1]]                  # U_t of the last slice, both parities
    ghost_fwd, ghost_bwd, ghost_link = exchange(to_prev, to_next, links_next)
    got = slab_dslash(psi_loc, u_loc, ghost_fwd, ghost_bwd, ghost_link, comp, nb, sg, dag)
    return float(np.linalg.norm(got - ref[rows]) / np.linalg.norm(ref[rows]))


@pytest.mark.parametrize("dag", [False, True])
def test_one_slab_with_its_own_faces(tmp_path, dag):
    """nranks = 1: the faces go back to the same slab (periodic in t)."""
    err = run_rank(0, 1, (4, 4, 6, 8), dag, str(tmp_path), lambda p, n, l: (p, n, l))
    assert err < 1e-13


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, L, dag, tmpdir, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    prev, nxt = (rank - 1) % world, (rank + 1) % world

    def exchange(to_prev, to_next, links_next):
        # to rank-1 its forward ghost, to rank+1 its backward ghost and the links
        def swap(send, dst, src, shape):
            out = torch.empty(shape, dtype=torch.complex128)
            reqs = [dist.isend(torch.from_numpy(np.ascontiguousarray(send)), dst), dist.irecv(out, src)]
            for r in reqs:
                r.wait()
            return out.numpy()
        gf = swap(to_prev, prev, nxt, to_prev.shape)
        gb = swap(to_next, nxt, prev, to_next.shape)
        gl = swap(links_next, nxt, prev, links_next.shape)
        return gf, gb, gl

    try:
        q.put((rank, run_rank(rank, world, L, dag, tmpdir, exchange)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,L", [(2, (8, 8, 8, 8)), (3, (4, 6, 4, 12))], ids=["2x8^4", "3x4x6x4x12"])
@pytest.mark.parametrize("dag", [False, True])
def test_gloo_slabs_equal_the_single_domain_operator(tmp_path, world, L, dag):
    # the map program once, before the ranks start
    build_maps(L, -1, world, 0, dag, str(tmp_path))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, L, dag, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res) == list(range(world))
    assert max(res.values()) < 1e-13, res


def test_interior_and_boundary_launches_partition_the_slab(tmp_path):
    """A slab pass runs as an interior launch (slices 1 .. Lt_loc-2, while the
    faces are exchanged) and a boundary launch (slices 0 and Lt_loc-1): every
    site in exactly one of them, no interior site reading a ghost, every
    boundary site reading one (tests/c_client/dd_parts.cu over decomp.cuh)."""
    exe = os.path.join(str(tmp_path), "dd_parts")
    subprocess.run([os.environ.get("NVCC", "nvcc"), "-std=c++17", "-O1", "-o", exe,
                    os.path.join(ROOT, "tests", "c_client", "dd_parts.cu")], check=True, capture_output=True)
    r = subprocess.run([exe, "8,8,8,2", "8,8,8,4", "4,6,4,6", "6,4,6,12", "2,2,2,8"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
