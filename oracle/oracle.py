"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker.  It restates BQCD's algorithms (see bqcd_oracle.c for
the reference file:line of each routine) and is pinned to the reference's
golden outputs ranf_test.reference and work/out.quick-test.reference.

Array conventions (numpy, C order, matching the Fortran memory layouts):
  spinor  complex128 (volh, 3, 4)          [site][colour][spin]
  gauge   complex128 (4, 2, volh, 3, 3)    [mu][eo][site][col][row]
  clover  complex128 (2, volh, 2, 18)      [eo][site][chi][slot]
  p       float64    (4, 2, volh, 8)       [mu][eo][site][generator]
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        so, _ = _build.build()
        L = C.CDLL(so)
        vp = C.c_void_p
        L.oqc_geom_new.restype = vp
        L.oqc_geom_new.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oqc_geom_delete.argtypes = [vp]
        L.oqc_volh.argtypes = [vp]
        L.oqc_ranset.argtypes = [C.c_longlong, C.c_longlong]
        L.oqc_ranget.restype = C.c_longlong
        L.oqc_ranf.restype = C.c_double
        L.oqc_cksum.argtypes = [C.c_void_p, C.c_longlong]
        L.oqc_cksum.restype = C.c_uint
        for n in ("oqc_conf_hot", "oqc_conf_cold", "oqc_conf_relax", "oqc_flip_bc"):
            getattr(L, n).argtypes = [vp, C.c_void_p]
        L.oqc_sg.argtypes = [vp, C.c_void_p]
        L.oqc_sg.restype = C.c_double
        L.oqc_ran_gauss_volh.argtypes = [vp, C.c_int, C.c_void_p, C.c_double, C.c_int]
        L.oqc_d.argtypes = [vp, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.oqc_clover_init.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.oqc_clover_mult.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oqc_clover_action.argtypes = [vp, C.c_void_p]
        L.oqc_clover_action.restype = C.c_double
        L.oqc_op.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]
        L.oqc_cg.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_float, C.c_int,
                             C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.oqc_dsf.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                              C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.oqc_clover_dsf.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.oqc_clover_dsd.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.oqc_dsg.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_double, C.c_double]
        L.oqc_gen2u.argtypes = [C.c_void_p, C.c_void_p]
        L.oqc_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def ranset(seed, skip=0):
    lib().oqc_ranset(seed, skip)


def ranget():
    return lib().oqc_ranget()


def ranf():
    return lib().oqc_ranf()


class Geom:
    """Single-process lattice geometry (init_common.F90)."""

    def __init__(self, L, bc=(1, 1, 1, -1)):
        Li = (C.c_int * 4)(*L)
        bci = (C.c_int * 4)(*bc)
        self.h = lib().oqc_geom_new(Li, bci)
        if not self.h:
            raise ValueError("bad lattice %r" % (L,))
        self.L = tuple(L)
        self.bc = tuple(bc)
        self.volh = lib().oqc_volh(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oqc_geom_delete(self.h)
            self.h = None

    # -- field constructors --
    def spinor(self):
        return np.zeros((self.volh, 3, 4), np.complex128)

    def gauge(self):
        return np.zeros((4, 2, self.volh, 3, 3), np.complex128)

    def clover(self):
        return np.zeros((2, self.volh, 2, 18), np.complex128)

    def momenta(self):
        return np.zeros((4, 2, self.volh, 8), np.float64)

    # -- RNG-driven inputs --
    def gauss_spinor(self, eo=0, var=0.5):
        s = self.spinor()
        lib().oqc_ran_gauss_volh(self.h, 12, _p(s), var, eo)
        return s

    def gauss_momenta(self):
        p = self.momenta()
        for mu in range(4):
            for eo in range(2):
                lib().oqc_ran_gauss_volh(self.h, 4, p[mu, eo].ctypes.data, 1.0, eo)
        return p

    def hot(self):
        u = self.gauge()
        lib().oqc_conf_hot(self.h, _p(u))
        return u

    def cold(self):
        u = self.gauge()
        lib().oqc_conf_cold(self.h, _p(u))
        return u

    def relax(self, u, n=1):
        for _ in range(n):
            lib().oqc_conf_relax(self.h, _p(u))
        return u

    def flip_bc(self, u):
        lib().oqc_flip_bc(self.h, _p(u))
        return u

    def sg(self, u):
        return lib().oqc_sg(self.h, _p(u))

    # -- operators --
    def d(self, e, o, inp, u, dag=False):
        out = self.spinor()
        lib().oqc_d(self.h, e, o, _p(out), _p(np.ascontiguousarray(inp)), _p(u), int(dag))
        return out

    def clover_init(self, u, csw_kappa):
        a, ai, b = self.clover(), self.clover(), self.clover()
        lib().oqc_clover_init(self.h, _p(a), _p(ai), _p(b), _p(u), csw_kappa)
        return a, ai, b

    def clover_mult(self, which, blk_eo, inp):
        out = self.spinor()
        lib().oqc_clover_mult(self.h, which, _p(np.ascontiguousarray(blk_eo)), _p(out),
                              _p(np.ascontiguousarray(inp)))
        return out

    def clover_action(self, b_eo):
        return lib().oqc_clover_action(self.h, _p(np.ascontiguousarray(b_eo)))

    OPS = {"mtil": 0, "mtil_dag": 1, "mtdagmt": 2, "w_mult": 3, "w_mult_dag": 4, "w_dagger_w": 5}

    def op(self, name, inp, u, clov, kappa, csw_kappa, h=0.0, rho=0.0):
        a, ai, b = clov if clov is not None else (None, None, None)
        out = self.spinor()
        lib().oqc_op(self.h, self.OPS[name], _p(out), _p(np.ascontiguousarray(inp)), _p(u), _p(a), _p(ai),
                     _p(b), kappa, csw_kappa, h, rho)
        return out

    def cg(self, name, x, bvec, u, clov, kappa, csw_kappa, h=0.0, rho=0.0, rest=1e-5, maxiter=1000, log=2):
        a, ai, b = clov if clov is not None else (None, None, None)
        x = np.array(x, copy=True)
        it = C.c_int(0)
        rtr = C.c_double(0)
        rc = lib().oqc_cg(self.h, self.OPS[name], _p(x), _p(np.ascontiguousarray(bvec)), _p(u), _p(a), _p(ai),
                          _p(b), kappa, csw_kappa, h, rho, rest, maxiter, log, C.byref(it), C.byref(rtr))
        return x, it.value, rtr.value, rc

    def dsf(self, p, u_flipped, clov, step, kappa, csw_kappa, a, b, h=0.0):
        """dsf.F90: p updated in place; u_flipped is modified back to periodic."""
        ca, ci, cb = clov if clov is not None else (None, None, None)
        lib().oqc_dsf(self.h, _p(p), _p(u_flipped), _p(ca), _p(ci), _p(cb), step, kappa, csw_kappa, h,
                      _p(np.ascontiguousarray(a)), _p(np.ascontiguousarray(b)))
        return p

    def clover_dsf(self, eo, p, b, a, s, u):
        lib().oqc_clover_dsf(self.h, eo, _p(p), _p(np.ascontiguousarray(b)), _p(np.ascontiguousarray(a)), s,
                             _p(u))
        return p

    def clover_dsd(self, eo, p, bfield, s, u):
        lib().oqc_clover_dsd(self.h, eo, _p(p), _p(bfield), s, _p(u))
        return p

    def dsg(self, p, u, step, beta):
        lib().oqc_dsg(self.h, _p(p), _p(u), step, beta)
        return p


def gen2u(h):
    u = np.zeros((3, 3), np.complex128)
    hh = np.ascontiguousarray(h, dtype=np.float64)
    lib().oqc_gen2u(u.ctypes.data, hh.ctypes.data)
    return u


def threads():
    return lib().oqc_threads()
