"""Python host mirror of BQCD's fermion hot path on the B200 library.

The routines keep the reference's names and argument meaning (d, d_dag,
clover_mult_a/ao/b, mtil, mtil_dag, mtdagmt, w_mult, w_mult_dag, w_dagger_w,
cg, quda_solver, dsf, clover_dsf, clover_dsd, clover_init, clover_action) and
call the CUDA library lib/libbqcdg.so through its C ABI (include/bqcdg.h).
There is no fallback: without the built library or a GPU every call raises.

Array conventions (numpy, C order, the Fortran memory layouts of defs.h):
  spinor  complex128 (volh, 3, 4)        SPINCOL_FIELD  [site][colour][spin]
  gauge   complex128 (4, 2, volh, 3, 3)  GAUGE_FIELD    [mu][eo][site][col][row]
  clover  complex128 (2, volh, 2, 18)    CLOVER_FIELD_A/B [eo][site][chi][slot]
  p       float64    (4, 2, volh, 8)     GENERATOR_FIELD
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.environ.get("BQCDG_LIB", os.path.join(HERE, "..", "lib", "libbqcdg.so"))

OK, EINVAL, ECUDA, ENOCONV, ENAN, ENOGAUGE, ENOCLOVER, ENOMEM, EUNSUPPORTED, ENOTSU3, ENODEVICE, ECHECKSUM, EIO = \
    range(13)
PREC_DOUBLE, PREC_SINGLE, PREC_HALF = 0, 1, 2
EVEN, ODD = 0, 1


class BqcdgError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__("%s: %s (status %d)" % (what, _lib_handle().bqcdg_error_string(status).decode(), status))


class Params(C.Structure):
    """bqcdg_params: kappa, csw_kappa, h, rho (type(hmc_para) subset)."""
    _fields_ = [("kappa", C.c_double), ("csw_kappa", C.c_double), ("h", C.c_double), ("rho", C.c_double)]


class CgPara(C.Structure):
    """bqcdg_cg_para = type(type_cg_para) (cg.F90:30-34)."""
    _fields_ = [("rest", C.c_float), ("maxiter", C.c_int), ("log", C.c_int)]


class SolverOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("maxiter", C.c_int), ("relative", C.c_int), ("tol", C.c_double),
                ("delta", C.c_double), ("check_true_residual", C.c_int), ("time_kernels", C.c_int),
                ("rhs_per_thread", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("niter", C.c_int), ("reliable_updates", C.c_int), ("rtr", C.c_double), ("true_rtr", C.c_double),
                ("b2", C.c_double), ("seconds", C.c_double), ("stencil_ms", C.c_double),
                ("stencil_launches", C.c_int), ("converged", C.c_int), ("kernel_launches", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ConfMeta(C.Structure):
    """bqcdg_conf_meta: the ConfInfoHeader of a configuration (conf_info.F90)."""
    _fields_ = [("run", C.c_int), ("traj", C.c_int), ("ensemble", C.c_int * 2), ("beta", C.c_double * 2),
                ("kappa", C.c_double * 2), ("csw", C.c_double * 2), ("csw_kappa", C.c_double * 2),
                ("h", C.c_double * 2), ("plaq_energy", C.c_double), ("L", C.c_int * 4), ("bc", C.c_int * 4)]

    def as_dict(self):
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = list(v) if hasattr(v, "__len__") else v
        return out


_LIB = None


def _lib_handle():
    global _LIB
    if _LIB is None:
        path = os.path.abspath(LIBPATH)
        if not os.path.exists(path):
            raise RuntimeError("libbqcdg.so is not built (%s); run bqcd-r399-quda_b200/build.py" % path)
        L = C.CDLL(path)
        vp, ip, dp, i = C.c_void_p, C.c_void_p, C.c_void_p, C.c_int
        P = C.POINTER
        L.bqcdg_error_string.restype = C.c_char_p
        L.bqcdg_error_string.argtypes = [i]
        L.bqcdg_create.argtypes = [P(vp), P(C.c_int), P(C.c_int), i]
        L.bqcdg_destroy.argtypes = [vp]
        L.bqcdg_volh.argtypes = [vp]
        L.bqcdg_device_bytes.argtypes = [vp]
        L.bqcdg_device_bytes.restype = C.c_longlong
        L.bqcdg_load_gauge.argtypes = [vp, dp, i]
        L.bqcdg_get_gauge.argtypes = [vp, dp, i]
        L.bqcdg_load_clover.argtypes = [vp, dp, dp, dp]
        L.bqcdg_get_clover.argtypes = [vp, dp, dp, dp]
        L.bqcdg_load_clover_solver.argtypes = [vp, dp, dp]
        L.bqcdg_clover_init.argtypes = [vp, C.c_double]
        L.bqcdg_clover_init_solver.argtypes = [vp, C.c_double]
        L.bqcdg_clover_init_t.argtypes = [vp, C.c_double]
        L.bqcdg_solve_block.argtypes = [vp, i, P(C.c_int), P(C.c_int), P(Params), P(SolverOpts), P(SolveInfo)]
        L.bqcdg_solve_batch_kappa.argtypes = [vp, i, P(C.c_int), P(C.c_int), P(Params), dp, dp, dp,
                                              P(SolverOpts), i, P(SolveInfo)]
        L.bqcdg_release_scratch.argtypes = [vp, i]
        L.bqcdg_conf_write.argtypes = [vp, C.c_char_p, P(ConfMeta)]
        L.bqcdg_conf_read.argtypes = [vp, C.c_char_p, P(ConfMeta)]
        L.bqcdg_clover_action.argtypes = [vp, i, P(C.c_double)]
        for n in ("bqcdg_d", "bqcdg_d_dag"):
            getattr(L, n).argtypes = [vp, i, i, dp, dp]
        L.bqcdg_clover_mult_a.argtypes = [vp, i, dp, dp]
        L.bqcdg_clover_mult_ao.argtypes = [vp, i, dp]
        L.bqcdg_clover_mult_b.argtypes = [vp, i, dp]
        for n in ("bqcdg_mtil", "bqcdg_mtil_dag", "bqcdg_mtdagmt", "bqcdg_w_mult", "bqcdg_w_mult_dag",
                  "bqcdg_w_dagger_w"):
            getattr(L, n).argtypes = [vp, dp, dp, P(Params)]
        L.bqcdg_cg.argtypes = [vp, dp, dp, P(Params), P(CgPara), P(C.c_int), P(SolveInfo)]
        L.bqcdg_quda_solver.argtypes = [vp, dp, dp, P(Params), P(CgPara), P(C.c_int), P(SolveInfo)]
        L.bqcdg_solve.argtypes = [vp, dp, dp, P(Params), P(SolverOpts), P(SolveInfo)]
        L.bqcdg_solver_opts_default.argtypes = [P(SolverOpts)]
        L.bqcdg_solver_opts_default.restype = None
        L.bqcdg_dsf.argtypes = [vp, dp, C.c_double, P(Params), dp, dp]
        L.bqcdg_clover_dsf.argtypes = [vp, i, dp, dp, dp, C.c_double]
        L.bqcdg_clover_dsd.argtypes = [vp, i, dp, C.c_double]
        L.bqcdg_field_create.argtypes = [vp, P(C.c_int)]
        L.bqcdg_field_upload.argtypes = [vp, i, dp]
        L.bqcdg_field_download.argtypes = [vp, i, dp]
        L.bqcdg_field_destroy.argtypes = [vp, i]
        L.bqcdg_solve_dev.argtypes = [vp, i, i, P(Params), P(SolverOpts), P(SolveInfo)]
        L.bqcdg_mdagm_dev.argtypes = [vp, i, i, P(Params), i, i, P(C.c_double)]
        L.bqcdg_time_pass.argtypes = [vp, i, P(Params), i, i, P(C.c_double)]
        L.bqcdg_time_pass_batch.argtypes = [vp, i, P(C.c_int), P(Params), i, i, i, P(C.c_double)]
        L.bqcdg_solve_batch.argtypes = [vp, i, P(C.c_int), P(C.c_int), P(Params), P(SolverOpts), i,
                                        P(SolveInfo)]
        L.bqcdg_solve_batch_shifted.argtypes = [vp, i, P(C.c_int), P(C.c_int), P(Params), dp, dp, P(SolverOpts),
                                                i, P(SolveInfo)]
        L.bqcdg_ranset.argtypes = [vp, C.c_longlong, C.c_longlong]
        L.bqcdg_ranget.argtypes = [vp, P(C.c_longlong)]
        L.bqcdg_conf_hot.argtypes = [vp]
        L.bqcdg_conf_cold.argtypes = [vp]
        L.bqcdg_conf_relax.argtypes = [vp, i]
        L.bqcdg_sg.argtypes = [vp, P(C.c_double)]
        L.bqcdg_field_gauss.argtypes = [vp, i, C.c_double]
        d, pd = C.c_double, P(C.c_double)
        for n in ("bqcdg_mom_gauss", "bqcdg_mom_mark", "bqcdg_gauge_save"):
            getattr(L, n).argtypes = [vp]
        L.bqcdg_mom_set.argtypes = [vp, dp]
        L.bqcdg_mom_get.argtypes = [vp, dp]
        L.bqcdg_mom_action.argtypes = [vp, pd]
        L.bqcdg_mom_change.argtypes = [vp, pd]
        L.bqcdg_dsg_dev.argtypes = [vp, d, d]
        L.bqcdg_hmc_u_dev.argtypes = [vp, d, d]
        L.bqcdg_dsf_dev.argtypes = [vp, d, P(Params), i, i]
        L.bqcdg_dsd_dev.argtypes = [vp, d, P(Params)]
        L.bqcdg_gauge_restore.argtypes = [vp, d]
        L.bqcdg_ranf.argtypes = [vp, pd]
        L.bqcdg_op_dev.argtypes = [vp, i, i, i, P(Params)]
        L.bqcdg_cg_dev.argtypes = [vp, i, i, P(Params), P(CgPara), P(C.c_int), P(SolveInfo)]
        L.bqcdg_field_cdot.argtypes = [vp, i, i, pd, pd]
        L.bqcdg_field_caxpby.argtypes = [vp, i, d, d, d, i]
        L.bqcdg_field_cdot_pairs.argtypes = [vp, i, P(C.c_int), P(C.c_int), pd, pd]
        L.bqcdg_dd_create_local.argtypes = [P(vp), P(C.c_int), P(C.c_int), i, i]
        L.bqcdg_dd_nccl_unique_id.argtypes = [C.c_char_p]
        L.bqcdg_dd_create_nccl.argtypes = [P(vp), P(C.c_int), P(C.c_int), i, i, i, C.c_char_p]
        L.bqcdg_dd_destroy.argtypes = [vp]
        L.bqcdg_dd_volh.argtypes = [vp]
        L.bqcdg_dd_load_gauge.argtypes = [vp, dp, i]
        L.bqcdg_dd_load_clover.argtypes = [vp, dp, dp]
        L.bqcdg_dd_op.argtypes = [vp, i, dp, dp, P(Params)]
        L.bqcdg_dd_cg.argtypes = [vp, dp, dp, P(Params), P(CgPara), P(C.c_int), P(SolveInfo)]
        L.bqcdg_dd_solve.argtypes = [vp, dp, dp, P(Params), P(SolverOpts), P(SolveInfo)]
        _LIB = L
    return _LIB


def lib():
    return _lib_handle()


def _ptr(a, dtype):
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == dtype and a.flags.c_contiguous):
        raise TypeError("expected a C-contiguous %s array" % np.dtype(dtype).name)
    return a.ctypes.data


def _check(status, what):
    if status != OK:
        raise BqcdgError(status, what)


@dataclass
class HmcPara:
    """The hot-path part of type(hmc_para) (modules/typedef_hmc.F90:32-44)."""
    kappa: float
    csw: float = 0.0
    h: float = 0.0
    rho: float = 0.0

    @property
    def csw_kappa(self):
        return self.csw * self.kappa  # bqcd.F90:170

    def params(self, rho=None):
        return Params(self.kappa, self.csw_kappa, self.h, self.rho if rho is None else rho)


class Lattice:
    """One GPU context over a whole single-process lattice."""

    def __init__(self, L, bc=(1, 1, 1, -1), device=0):
        self.L = tuple(int(x) for x in L)
        self.bc = tuple(int(x) for x in bc)
        h = C.c_void_p()
        _check(lib().bqcdg_create(C.byref(h), (C.c_int * 4)(*self.L), (C.c_int * 4)(*self.bc), device),
               "bqcdg_create")
        self.h = h
        self.volh = lib().bqcdg_volh(h)

    def close(self):
        if getattr(self, "h", None):
            lib().bqcdg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def device_bytes(self):
        return lib().bqcdg_device_bytes(self.h)

    # ---- fields ----
    def spinor(self):
        return np.zeros((self.volh, 3, 4), np.complex128)

    def load_gauge(self, u, flipped):
        _check(lib().bqcdg_load_gauge(self.h, _ptr(u, np.complex128), int(flipped)), "load_gauge")

    def get_gauge(self, flipped=False):
        u = np.zeros((4, 2, self.volh, 3, 3), np.complex128)
        _check(lib().bqcdg_get_gauge(self.h, u.ctypes.data, int(flipped)), "get_gauge")
        return u

    def load_clover(self, a=None, ainv=None, b=None):
        _check(lib().bqcdg_load_clover(self.h, _ptr(a, np.complex128), _ptr(ainv, np.complex128),
                                       _ptr(b, np.complex128)), "load_clover")

    def clover_init(self, csw_kappa):
        """clover_init(a, i, b, u, csw_kappa) on the device from the loaded links."""
        _check(lib().bqcdg_clover_init(self.h, csw_kappa), "clover_init")

    def release_scratch(self, solver=True, hmc=False):
        """Free the device buffers that later calls re-create on demand:
        the solver's work vectors and staging (solver), the resident momenta,
        saved links and force buffers (hmc)."""
        _check(lib().bqcdg_release_scratch(self.h, (1 if solver else 0) | (2 if hmc else 0)), "release_scratch")

    def conf_write(self, base, run=1, traj=0, ensemble=(1, 1), para=None, beta=0.0):
        """conf_write: the resident links to BQCD's slice files <base>.<tt>.u
        and the info file <base>.info; returns the header written."""
        m = ConfMeta()
        m.run, m.traj = run, traj
        for k in range(2):
            m.ensemble[k] = ensemble[k]
            m.beta[k] = beta
            if para is not None:
                m.kappa[k], m.csw[k], m.csw_kappa[k], m.h[k] = para.kappa, para.csw, para.csw_kappa, para.h
        _check(lib().bqcdg_conf_write(self.h, base.encode(), C.byref(m)), "conf_write")
        return m.as_dict()

    def conf_read(self, info_file):
        """conf_read: the configuration of an info file becomes the resident
        links; returns its header."""
        m = ConfMeta()
        _check(lib().bqcdg_conf_read(self.h, info_file.encode(), C.byref(m)), "conf_read")
        return m.as_dict()

    def clover_init_solver(self, csw_kappa):
        """clover_init keeping only the two parts the even-odd solver uses (A
        even, A^-1 odd): a third of the clover memory of clover_init."""
        _check(lib().bqcdg_clover_init_solver(self.h, csw_kappa), "clover_init_solver")

    def load_clover_solver(self, a, ainv):
        """load_clover keeping only what the even-odd solver reads: A of the
        even sites and A^-1 of the odd ones, from the full arrays."""
        _check(lib().bqcdg_load_clover_solver(self.h, _ptr(a, np.complex128), _ptr(ainv, np.complex128)),
               "load_clover_solver")

    def get_clover(self):
        out = [np.zeros((2, self.volh, 2, 18), np.complex128) for _ in range(3)]
        _check(lib().bqcdg_get_clover(self.h, *[o.ctypes.data for o in out]), "get_clover")
        return tuple(out)

    def clover_action(self, eo=ODD):
        v = C.c_double()
        _check(lib().bqcdg_clover_action(self.h, eo, C.byref(v)), "clover_action")
        return v.value

    # ---- operators (reference names) ----
    def d(self, e, o, inp):
        out = self.spinor()
        _check(lib().bqcdg_d(self.h, e, o, out.ctypes.data, _ptr(inp, np.complex128)), "d")
        return out

    def d_dag(self, e, o, inp):
        out = self.spinor()
        _check(lib().bqcdg_d_dag(self.h, e, o, out.ctypes.data, _ptr(inp, np.complex128)), "d_dag")
        return out

    def clover_mult_a(self, eo, inp):
        out = self.spinor()
        _check(lib().bqcdg_clover_mult_a(self.h, eo, out.ctypes.data, _ptr(inp, np.complex128)), "clover_mult_a")
        return out

    def clover_mult_ao(self, eo, x):
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        _check(lib().bqcdg_clover_mult_ao(self.h, eo, x.ctypes.data), "clover_mult_ao")
        return x

    def clover_mult_b(self, eo, x):
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        _check(lib().bqcdg_clover_mult_b(self.h, eo, x.ctypes.data), "clover_mult_b")
        return x

    def _op(self, name, inp, para):
        out = self.spinor()
        prm = para.params() if isinstance(para, HmcPara) else para
        _check(getattr(lib(), "bqcdg_" + name)(self.h, out.ctypes.data, _ptr(inp, np.complex128), C.byref(prm)),
               name)
        return out

    def mtil(self, inp, para):
        return self._op("mtil", inp, para)

    def mtil_dag(self, inp, para):
        return self._op("mtil_dag", inp, para)

    def mtdagmt(self, inp, para):
        return self._op("mtdagmt", inp, para)

    def w_mult(self, inp, para):
        return self._op("w_mult", inp, para)

    def w_mult_dag(self, inp, para):
        return self._op("w_mult_dag", inp, para)

    def w_dagger_w(self, inp, para):
        return self._op("w_dagger_w", inp, para)

    # ---- solvers ----
    def cg(self, x, b, para, rest, maxiter=1000, log=0, rho=None):
        """cg(w_dagger_w or mtdagmt, x, b, ...) (cg.F90:51): x is the initial
        guess; returns (x, iterations, info).  Raises on no convergence unless
        log == 2 (then info.converged is 0)."""
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        it = C.c_int()
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        cp = CgPara(rest, maxiter, log)
        _check(lib().bqcdg_cg(self.h, x.ctypes.data, _ptr(b, np.complex128), C.byref(prm), C.byref(cp),
                              C.byref(it), C.byref(info)), "cg")
        return x, it.value, info

    def quda_solver(self, x, b, para, rest, maxiter=1000, log=0, rho=None):
        """quda_solver(matrix_mult, x, b, para, conf, iterations, rho)
        (invert_quda.F90:96): mixed precision, absolute stop, true residual
        re-checked in FP64."""
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        it = C.c_int()
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        cp = CgPara(rest, maxiter, log)
        _check(lib().bqcdg_quda_solver(self.h, x.ctypes.data, _ptr(b, np.complex128), C.byref(prm), C.byref(cp),
                                       C.byref(it), C.byref(info)), "quda_solver")
        return x, it.value, info

    def solve(self, x, b, para, precision=PREC_HALF, tol=1e-10, relative=True, maxiter=100000, delta=0.1,
              time_kernels=False, rho=None, inplace=False):
        """x (initial guess) -> solution; a copy unless inplace, in which
        case x must be a C-contiguous complex128 array (it may live in pinned
        host memory, so that its transfers run at the link's rate)."""
        if inplace:
            _ptr(x, np.complex128)
        else:
            x = np.array(x, dtype=np.complex128, copy=True, order="C")
        o = SolverOpts(precision, maxiter, int(relative), tol, delta, 1, int(time_kernels))
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        st = lib().bqcdg_solve(self.h, x.ctypes.data, _ptr(b, np.complex128), C.byref(prm), C.byref(o),
                               C.byref(info))
        if st not in (OK, ENOCONV):
            _check(st, "solve")
        return x, info

    # ---- forces ----
    def dsf(self, p, step, para, a, b):
        """dsf(p, conf, step, para, a, b) (dsf.F90:28); p is updated in place."""
        prm = para.params() if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_dsf(self.h, _ptr(p, np.float64), step, C.byref(prm), _ptr(a, np.complex128),
                               _ptr(b, np.complex128)), "dsf")
        return p

    def clover_dsf(self, eo, p, b, a, s):
        _check(lib().bqcdg_clover_dsf(self.h, eo, _ptr(p, np.float64), _ptr(b, np.complex128),
                                      _ptr(a, np.complex128), s), "clover_dsf")
        return p

    def clover_dsd(self, eo, p, s):
        _check(lib().bqcdg_clover_dsd(self.h, eo, _ptr(p, np.float64), s), "clover_dsd")
        return p

    # ---- seeded inputs on the device (ranf.F90, ran.F90, conf.F90, cooling.F90) ----
    def ranset(self, seed, skip=0):
        _check(lib().bqcdg_ranset(self.h, seed, skip), "ranset")

    def ranget(self):
        s = C.c_longlong()
        _check(lib().bqcdg_ranget(self.h, C.byref(s)), "ranget")
        return s.value

    def conf_hot(self):
        _check(lib().bqcdg_conf_hot(self.h), "conf_hot")

    def conf_cold(self):
        _check(lib().bqcdg_conf_cold(self.h), "conf_cold")

    def conf_relax(self, n=1):
        _check(lib().bqcdg_conf_relax(self.h, n), "conf_relax")

    def sg(self):
        v = C.c_double()
        _check(lib().bqcdg_sg(self.h, C.byref(v)), "sg")
        return v.value

    def plaq_energy(self):
        """sg / (6 V) as BQCD prints it (mc.F90:63)."""
        return self.sg() / (6.0 * 2 * self.volh)

    def field_gauss(self, handle, var=0.5):
        _check(lib().bqcdg_field_gauss(self.h, handle, var), "field_gauss")

    # ---- resident fields ----
    def field(self, host=None):
        h = C.c_int()
        _check(lib().bqcdg_field_create(self.h, C.byref(h)), "field_create")
        if host is not None:
            _check(lib().bqcdg_field_upload(self.h, h.value, _ptr(host, np.complex128)), "field_upload")
        return h.value

    def field_get(self, handle):
        out = self.spinor()
        _check(lib().bqcdg_field_download(self.h, handle, out.ctypes.data), "field_download")
        return out

    def field_set(self, handle, host):
        _check(lib().bqcdg_field_upload(self.h, handle, _ptr(host, np.complex128)), "field_upload")

    def field_cdot(self, ha, hb):
        """<a, b> = sum conj(a) b of two resident fields."""
        re, im = C.c_double(), C.c_double()
        _check(lib().bqcdg_field_cdot(self.h, ha, hb, C.byref(re), C.byref(im)), "field_cdot")
        return complex(re.value, im.value)

    MAX_DOT_PAIRS = 8   # BQCDG_MAX_DOT_PAIRS

    def field_cdot_pairs(self, pairs):
        """[<a, b> for (a, b) in pairs] of resident fields, each equal to
        field_cdot(a, b) bit for bit, in launches of up to MAX_DOT_PAIRS
        pairs with one read-back each."""
        out = []
        for k in range(0, len(pairs), self.MAX_DOT_PAIRS):
            chunk = pairs[k:k + self.MAX_DOT_PAIRS]
            n = len(chunk)
            ha = (C.c_int * n)(*[a for a, _ in chunk])
            hb = (C.c_int * n)(*[b for _, b in chunk])
            re, im = (C.c_double * n)(), (C.c_double * n)()
            _check(lib().bqcdg_field_cdot_pairs(self.h, n, ha, hb, re, im), "field_cdot_pairs")
            out.extend(complex(re[j], im[j]) for j in range(n))
        return out

    def field_caxpby(self, hy, ay, a, hx):
        """y = ay y + a x (a complex) on resident fields."""
        a = complex(a)
        _check(lib().bqcdg_field_caxpby(self.h, hy, float(ay), a.real, a.imag, hx), "field_caxpby")

    def field_copy(self, hdst, hsrc):
        self.field_caxpby(hdst, 0.0, 1.0, hsrc)

    OPS = {"mtil": 0, "mtil_dag": 1, "mtdagmt": 2, "w_mult": 3, "w_mult_dag": 4, "w_dagger_w": 5}

    def op_dev(self, which, hout, hin, para, rho=None):
        """hout = op(hin) on resident fields, op one of OPS (m_tilde.F90, w_mult.F90)."""
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_op_dev(self.h, self.OPS[which], hout, hin, C.byref(prm)), "op_dev")

    def cg_dev(self, hx, hb, para, rest, maxiter=1000, log=0, rho=None):
        """cg.F90 on resident fields (x: initial guess in, solution out);
        returns (iterations, info)."""
        it = C.c_int()
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        cp = CgPara(rest, maxiter, log)
        _check(lib().bqcdg_cg_dev(self.h, hx, hb, C.byref(prm), C.byref(cp), C.byref(it), C.byref(info)), "cg_dev")
        return it.value, info

    # ---- resident HMC pieces (momenta, gauge update and force) ----
    def mom_gauss(self):
        _check(lib().bqcdg_mom_gauss(self.h), "mom_gauss")

    def mom_set(self, p):
        _check(lib().bqcdg_mom_set(self.h, _ptr(p, np.float64)), "mom_set")

    def mom_get(self):
        p = np.zeros((4, 2, self.volh, 8), np.float64)
        _check(lib().bqcdg_mom_get(self.h, p.ctypes.data), "mom_get")
        return p

    def mom_action(self):
        v = C.c_double()
        _check(lib().bqcdg_mom_action(self.h, C.byref(v)), "mom_action")
        return v.value

    def mom_mark(self):
        _check(lib().bqcdg_mom_mark(self.h), "mom_mark")

    def mom_change(self):
        v = C.c_double()
        _check(lib().bqcdg_mom_change(self.h, C.byref(v)), "mom_change")
        return v.value

    def dsg_dev(self, step, beta):
        _check(lib().bqcdg_dsg_dev(self.h, step, beta), "dsg_dev")

    def hmc_u_dev(self, step, csw_kappa):
        _check(lib().bqcdg_hmc_u_dev(self.h, step, csw_kappa), "hmc_u_dev")

    def dsf_dev(self, step, para, ha, hb):
        prm = para.params() if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_dsf_dev(self.h, step, C.byref(prm), ha, hb), "dsf_dev")

    def dsd_dev(self, step, para):
        prm = para.params() if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_dsd_dev(self.h, step, C.byref(prm)), "dsd_dev")

    def gauge_save(self):
        _check(lib().bqcdg_gauge_save(self.h), "gauge_save")

    def gauge_restore(self, csw_kappa):
        _check(lib().bqcdg_gauge_restore(self.h, csw_kappa), "gauge_restore")

    def ranf(self):
        v = C.c_double()
        _check(lib().bqcdg_ranf(self.h, C.byref(v)), "ranf")
        return v.value

    def solve_dev(self, hx, hb, para, precision=PREC_HALF, tol=1e-10, relative=True, maxiter=100000, delta=0.1,
                  time_kernels=False, rho=None):
        o = SolverOpts(precision, maxiter, int(relative), tol, delta, 1, int(time_kernels))
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        st = lib().bqcdg_solve_dev(self.h, hx, hb, C.byref(prm), C.byref(o), C.byref(info))
        if st not in (OK, ENOCONV):
            _check(st, "solve_dev")
        return info

    def solve_batch(self, hxs, hbs, para, precision=PREC_HALF, tol=1e-10, relative=True, maxiter=100000,
                    delta=0.1, block=0, rho=None, rhs_per_thread=0):
        """Batched mixed-precision solve of len(hxs) resident systems; block =
        right-hand sides per launch (0: autotuned).  Returns the per-RHS infos."""
        n = len(hxs)
        o = SolverOpts(precision, maxiter, int(relative), tol, delta, 1, 0, rhs_per_thread)
        infos = (SolveInfo * n)()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        st = lib().bqcdg_solve_batch(self.h, n, (C.c_int * n)(*hxs), (C.c_int * n)(*hbs), C.byref(prm),
                                     C.byref(o), block, infos)
        if st not in (OK, ENOCONV):
            _check(st, "solve_batch")
        return list(infos)

    def solve_batch_shifted(self, hxs, hbs, para, rhos, precision=PREC_HALF, tol=1e-10, relative=True,
                            maxiter=100000, delta=0.1, block=0, rhs_per_thread=0):
        """solve_batch with the shift rho of system k given by rhos[k]
        (W = M~ + rho_k); the links and clover are shared.  tol: one number
        for all systems, or one per system."""
        n = len(hxs)
        if len(rhos) != n or len(hbs) != n:
            raise ValueError("solve_batch_shifted: one b and one rho per x")
        tols = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, dtype=np.float64), (n,)))
        o = SolverOpts(precision, maxiter, int(relative), float(tols[0]), delta, 1, 0, rhs_per_thread)
        infos = (SolveInfo * n)()
        prm = para.params(0.0) if isinstance(para, HmcPara) else para
        r = np.ascontiguousarray(rhos, dtype=np.float64)
        st = lib().bqcdg_solve_batch_shifted(self.h, n, (C.c_int * n)(*hxs), (C.c_int * n)(*hbs), C.byref(prm),
                                             r.ctypes.data, tols.ctypes.data, C.byref(o), block, infos)
        if st not in (OK, ENOCONV):
            _check(st, "solve_batch_shifted")
        return list(infos)

    def solve_block(self, hxs, hbs, para, tol=1e-10, relative=True, maxiter=100000, delta=0.1, rho=None):
        """Block CG over the resident systems (W^+W) x_k = b_k (up to 16)
        sharing one Krylov space: FP32 blocks, FP64 restarts.  Returns the
        infos (niter = block iterations until the system left)."""
        n = len(hxs)
        if len(hbs) != n:
            raise ValueError("solve_block: one b per x")
        o = SolverOpts(PREC_SINGLE, maxiter, int(relative), tol, delta, 1, 0, 1)
        infos = (SolveInfo * n)()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        st = lib().bqcdg_solve_block(self.h, n, (C.c_int * n)(*hxs), (C.c_int * n)(*hbs), C.byref(prm), C.byref(o),
                                     infos)
        if st not in (OK, ENOCONV):
            _check(st, "solve_block")
        return list(infos)

    def clover_init_t(self, csw):
        """The clover term for any kappa (bqcdg_clover_init_t): operators
        then build A(kappa) = 1 + kappa T at the kappa of their parameters."""
        _check(lib().bqcdg_clover_init_t(self.h, csw), "clover_init_t")

    def solve_batch_kappa(self, hxs, hbs, para, kappas, rhos=None, precision=PREC_HALF, tol=1e-10, relative=True,
                          maxiter=100000, delta=0.1, block=0):
        """Batched solve of (W_k^+W_k) x_k = b_k, W_k = M~(kappa_k) + rho_k:
        each system its own hopping parameter (and clover term, from
        clover_init_t) and shift; para gives c_sw (nonzero: clover) and h."""
        n = len(hxs)
        if len(kappas) != n or len(hbs) != n or (rhos is not None and len(rhos) != n):
            raise ValueError("solve_batch_kappa: one b, one kappa (and one rho) per x")
        tols = np.ascontiguousarray(np.broadcast_to(np.asarray(tol, dtype=np.float64), (n,)))
        o = SolverOpts(precision, maxiter, int(relative), float(tols[0]), delta, 1, 0, 1)
        infos = (SolveInfo * n)()
        prm = para.params(0.0) if isinstance(para, HmcPara) else para
        k = np.ascontiguousarray(kappas, dtype=np.float64)
        r = None if rhos is None else np.ascontiguousarray(rhos, dtype=np.float64)
        st = lib().bqcdg_solve_batch_kappa(self.h, n, (C.c_int * n)(*hxs), (C.c_int * n)(*hbs), C.byref(prm),
                                           k.ctypes.data, None if r is None else r.ctypes.data, tols.ctypes.data,
                                           C.byref(o), block, infos)
        if st not in (OK, ENOCONV):
            _check(st, "solve_batch_kappa")
        return list(infos)

    def mdagm_dev(self, hout, hin, para, precision, n, rho=None):
        ms = C.c_double()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_mdagm_dev(self.h, hout, hin, C.byref(prm), precision, n, C.byref(ms)), "mdagm_dev")
        return ms.value

    def time_pass(self, hin, para, precision, n, rho=None):
        ms = C.c_double()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_time_pass(self.h, hin, C.byref(prm), precision, n, C.byref(ms)), "time_pass")
        return ms.value

    def time_pass_batch(self, hins, para, precision, n, rho=None, rhs_per_thread=0):
        """Average device ms of one batched first stencil pass over the
        resident fields hins (one launch serves all of them; rhs_per_thread
        per stencil thread, 0 = the solver's timed choice)."""
        ms = C.c_double()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        k = len(hins)
        _check(lib().bqcdg_time_pass_batch(self.h, k, (C.c_int * k)(*hins), C.byref(prm), precision,
                                           rhs_per_thread, n, C.byref(ms)), "time_pass_batch")
        return ms.value


class SlabDecomposition:
    """The lattice cut along t into nranks slabs (bqcdg_dd_* of bqcdg.h): the
    FP64 operators and CG, and the mixed-precision solve (solve).

    SlabDecomposition.local(L, nranks): every slab in this process on one
    device (host arrays are the global ones).  SlabDecomposition.nccl(L,
    nranks, rank, uid): this process's slab, the others in their own
    processes over NCCL (host arrays are the slab's; uid from
    nccl_unique_id() on rank 0, passed to the others by the caller)."""

    OPS = {"mtil": 0, "mtil_dag": 1, "mtdagmt": 2, "w_mult": 3, "w_mult_dag": 4, "w_dagger_w": 5, "d": 6,
           "d_dag": 7}

    def __init__(self, handle, L, nranks):
        self.h = handle
        self.L = tuple(L)
        self.nranks = nranks
        self.volh = lib().bqcdg_dd_volh(self.h)

    @classmethod
    def local(cls, L, nranks, bc=(1, 1, 1, -1), device=0):
        h = C.c_void_p()
        _check(lib().bqcdg_dd_create_local(C.byref(h), (C.c_int * 4)(*L), (C.c_int * 4)(*bc), nranks, device),
               "dd_create_local")
        return cls(h, L, nranks)

    @staticmethod
    def nccl_unique_id():
        buf = C.create_string_buffer(128)
        _check(lib().bqcdg_dd_nccl_unique_id(buf), "dd_nccl_unique_id")
        return buf.raw

    @classmethod
    def nccl(cls, L, nranks, rank, uid, bc=(1, 1, 1, -1), device=0):
        h = C.c_void_p()
        _check(lib().bqcdg_dd_create_nccl(C.byref(h), (C.c_int * 4)(*L), (C.c_int * 4)(*bc), nranks, rank, device,
                                          uid), "dd_create_nccl")
        return cls(h, L, nranks)

    def close(self):
        if self.h:
            lib().bqcdg_dd_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def load_gauge(self, u, flipped):
        _check(lib().bqcdg_dd_load_gauge(self.h, _ptr(u, np.complex128), int(flipped)), "dd_load_gauge")

    def load_clover(self, a, ainv):
        _check(lib().bqcdg_dd_load_clover(self.h, _ptr(a, np.complex128), _ptr(ainv, np.complex128)),
               "dd_load_clover")

    def op(self, name, inp, para):
        out = np.zeros((self.volh, 3, 4), np.complex128)
        prm = para.params() if isinstance(para, HmcPara) else para
        _check(lib().bqcdg_dd_op(self.h, self.OPS[name], out.ctypes.data, _ptr(inp, np.complex128), C.byref(prm)),
               "dd_op")
        return out

    def cg(self, x, b, para, rest, maxiter=1000, log=0, rho=None):
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        it = C.c_int()
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        cp = CgPara(rest, maxiter, log)
        _check(lib().bqcdg_dd_cg(self.h, x.ctypes.data, _ptr(b, np.complex128), C.byref(prm), C.byref(cp),
                                 C.byref(it), C.byref(info)), "dd_cg")
        return x, it.value, info

    def solve(self, x, b, para, tol=1e-10, relative=True, maxiter=100000, delta=0.1, rho=None):
        """bqcdg_dd_solve: int16 iterations with FP64 reliable updates;
        returns (x, info).  No convergence is reported in info, not raised."""
        x = np.array(x, dtype=np.complex128, copy=True, order="C")
        info = SolveInfo()
        prm = para.params(rho) if isinstance(para, HmcPara) else para
        o = SolverOpts(PREC_HALF, maxiter, int(relative), tol, delta, 1, 0)
        st = lib().bqcdg_dd_solve(self.h, x.ctypes.data, _ptr(b, np.complex128), C.byref(prm), C.byref(o),
                                  C.byref(info))
        if st not in (OK, ENOCONV):
            _check(st, "dd_solve")
        return x, info
