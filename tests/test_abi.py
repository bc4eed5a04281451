"""CPU checks of the drop-in boundary: the C ABI library exists, loads, exports
every symbol include/bqcdg.h declares, and rejects bad calls without a GPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bqcdg.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bqcdg_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def so():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bqbuild", os.path.join(ROOT, "bqcd-r399-quda_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.build()


def test_header_declares_the_reference_entry_points():
    syms = declared_symbols()
    for need in ("bqcdg_d", "bqcdg_d_dag", "bqcdg_clover_mult_a", "bqcdg_clover_mult_ao", "bqcdg_clover_mult_b",
                 "bqcdg_mtil", "bqcdg_mtil_dag", "bqcdg_mtdagmt", "bqcdg_w_mult", "bqcdg_w_mult_dag",
                 "bqcdg_w_dagger_w", "bqcdg_cg", "bqcdg_quda_solver", "bqcdg_dsf", "bqcdg_clover_dsf",
                 "bqcdg_clover_dsd", "bqcdg_clover_init", "bqcdg_clover_action"):
        assert need in syms


def test_library_exports_every_declared_symbol(so):
    lib = C.CDLL(so)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_error_strings_and_argument_checks(so):
    lib = C.CDLL(so)
    lib.bqcdg_error_string.restype = C.c_char_p
    assert lib.bqcdg_error_string(0) == b"ok"
    assert lib.bqcdg_error_string(3) == b"no convergence"
    h = C.c_void_p()
    L = (C.c_int * 4)(4, 4, 4, 4)
    bad = (C.c_int * 4)(5, 4, 4, 4)          # odd extent: init_common.F90:67
    bc = (C.c_int * 4)(1, 1, 1, -1)
    badbc = (C.c_int * 4)(1, 1, 1, 0)
    assert lib.bqcdg_create(C.byref(h), bad, bc, 0) == 1
    assert lib.bqcdg_create(C.byref(h), L, badbc, 0) == 1
    assert lib.bqcdg_create(None, L, bc, 0) == 1
    assert lib.bqcdg_destroy(None) == 1
    assert lib.bqcdg_d(None, 0, 1, None, None) == 1
    ha, hb = (C.c_int * 9)(*range(9)), (C.c_int * 9)(*range(9))
    re_, im_ = (C.c_double * 9)(), (C.c_double * 9)()
    assert lib.bqcdg_field_cdot_pairs(None, 2, ha, hb, re_, im_) == 1
    assert lib.bqcdg_field_cdot_pairs(None, 9, ha, hb, re_, im_) == 1   # more than BQCDG_MAX_DOT_PAIRS


def test_no_device_is_reported_not_faulted(so):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = C.CDLL(so)
    h = C.c_void_p()
    rc = lib.bqcdg_create(C.byref(h), (C.c_int * 4)(4, 4, 4, 4), (C.c_int * 4)(1, 1, 1, -1), 0)
    assert rc == 10  # BQCDG_ENODEVICE


def test_python_mirror_fails_loudly_without_gpu(bq):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(bq.BqcdgError):
        bq.Lattice((4, 4, 4, 4))


def test_noalloc_argument_and_size_checks(so, bq):
    """bqcdg_mdagm_noalloc rejects missing arguments and a lattice larger
    than its static scratch before it touches a device."""
    lib = C.CDLL(so)
    f = lib.bqcdg_mdagm_noalloc
    f.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(bq.Params), C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    bc = (C.c_int * 4)(1, 1, 1, -1)
    one = C.c_void_p(1)            # never dereferenced: the checks come first
    big = (C.c_int * 4)(16, 16, 16, 16)     # volh 32768 > BQCDG_NOALLOC_MAX_VOLH
    prm = bq.Params(0.13, 0.0, 0.0, 0.0)
    assert f(big, bc, one, one, one, C.byref(prm), one, one, None) == bq.EINVAL
    small = (C.c_int * 4)(4, 4, 4, 4)
    assert f(small, bc, None, one, one, C.byref(prm), one, one, None) == bq.EINVAL
    assert f(small, bc, one, one, one, None, one, one, None) == bq.EINVAL
    assert f((C.c_int * 4)(5, 4, 4, 4), bc, one, one, one, C.byref(prm), one, one, None) == bq.EINVAL
    clov = bq.Params(0.13, 0.25, 0.0, 0.0)  # csw != 0 needs both clover parts
    assert f(small, bc, one, None, one, C.byref(clov), one, one, None) == bq.ENOCLOVER


def test_slab_decomposition_shape_is_checked(bq):
    """bqcdg_dd_create_local refuses slabs that do not divide the time
    extent into an even number of slices each, before it touches a device."""
    with pytest.raises(bq.BqcdgError) as e:
        bq.SlabDecomposition.local((8, 8, 8, 8), 3)        # 8 slices do not split into 3
    assert e.value.status == bq.EINVAL
    with pytest.raises(bq.BqcdgError) as e:
        bq.SlabDecomposition.local((8, 8, 8, 12), 4)       # slabs of 3 slices would mix parities
    assert e.value.status == bq.EINVAL


def test_slab_solvers_check_their_arguments(so, bq):
    """bqcdg_dd_cg and bqcdg_dd_solve refuse a missing decomposition or
    missing arrays before they touch a device."""
    lib = C.CDLL(so)
    one = C.c_void_p(1)            # never dereferenced: the checks come first
    prm = bq.Params(0.13, 0.0, 0.0, 0.0)
    cgp = bq.CgPara(1e-20, 100, 0)
    opts = bq.SolverOpts(bq.PREC_HALF, 100, 1, 1e-10, 0.1, 1, 0, 0)
    info = bq.SolveInfo()
    it = C.c_int()
    lib.bqcdg_dd_cg.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(bq.Params), C.POINTER(bq.CgPara),
                                C.POINTER(C.c_int), C.POINTER(bq.SolveInfo)]
    lib.bqcdg_dd_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(bq.Params),
                                   C.POINTER(bq.SolverOpts), C.POINTER(bq.SolveInfo)]
    assert lib.bqcdg_dd_cg(None, one, one, C.byref(prm), C.byref(cgp), C.byref(it), C.byref(info)) == bq.EINVAL
    assert lib.bqcdg_dd_solve(None, one, one, C.byref(prm), C.byref(opts), C.byref(info)) == bq.EINVAL
    assert lib.bqcdg_dd_op(None, 0, one, one, C.byref(prm)) == bq.EINVAL
    assert lib.bqcdg_dd_volh(None) == -1
