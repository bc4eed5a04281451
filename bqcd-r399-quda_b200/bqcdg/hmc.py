"""One HMC trajectory of BQCD on device-resident data.

The flow of hmc.F90:69-216 (test = none) and the routines it calls, driving
the C ABI: the links, the momenta, the pseudofermions phi/phi2 and every
spinor of the solves stay in GPU memory from the momentum draw to the
accept/reject step; only scalars (actions, dot products of the MRE Gram
system, CG statistics) come back to the host.

    hmc_init_p.F90:28-45      momenta                  Lattice.mom_gauss
    hmc_init_phi.F90:28-79    pseudofermions           Hmc._init_phi
    hmc_leap_frog.F90:28-79   nested leapfrog          Hmc._leap_frog
    hmc_integrator.F90:28-85  p_ir / p_uv              Hmc._p_ir / _p_uv
    dsf1.F90, dsf2.F90        fermion forces           Hmc._dsf1 / _dsf2
    dsd.F90, dsg.F90          det and gauge forces     Hmc._dsd / _dsg
    hmc_u.F90                 gauge update             Lattice.hmc_u_dev
    hmc_forces.F90:65-104     force monitor            Hmc._forces_new
    mre.F90:29-279            chronological guess      Mre
    action.F90                Hamiltonian terms        Hmc.trajectory
"""
import math

import numpy as np

from . import HmcPara, ODD


class Mre:
    """Minimal-residual extrapolation of the initial CG guess from the last
    nvec solutions (mre.F90): a ring of resident fields, Gram-Schmidt with
    the real scalar product BQCD uses for its overindexed real vectors, the
    Gram system of the operator images solved on the host."""

    def __init__(self, lat, nvec):
        self.lat = lat
        self.nvec = nvec
        self.rank = 0
        self.vec = [lat.field() for _ in range(nvec)]
        self.mv = [lat.field() for _ in range(nvec)]

    def put(self, h, reset):
        """mre.F90:29-66: remember the solution h (reset: forget all)."""
        if self.nvec == 0:
            return
        if reset:
            self.rank = 0
            return
        self.vec.insert(0, self.vec.pop())
        self.lat.field_copy(self.vec[0], h)
        self.rank = min(self.rank + 1, self.nvec)

    def _gram_schmidt(self):
        """mre.F90:189-213 (real scalar products).  The products of the
        normalised v_k with the later vectors do not depend on one another,
        so each step reads them back in one call."""
        lat = self.lat
        for k in range(self.rank):
            vk = self.vec[k]
            rkk = lat.field_cdot(vk, vk).real
            lat.field_caxpby(vk, 0.0, 1.0 / math.sqrt(rkk), vk)
            later = self.vec[k + 1:self.rank]
            rk = lat.field_cdot_pairs([(vk, vj) for vj in later])
            for vj, rkj in zip(later, rk):
                lat.field_caxpby(vj, 1.0, -rkj.real, vk)

    @staticmethod
    def _gauss_jordan(a, b):
        """mre.F90:215-279: Gauss-Jordan elimination with full pivoting of
        a x = b in place (a: n x n complex, b: n); returns x."""
        n = len(b)
        a = a.copy()
        b = b.copy()
        ipiv = [0] * n
        irow = icol = 0
        for _ in range(n):
            big = 0.0
            for j in range(n):
                if ipiv[j] != 1:
                    for k in range(n):
                        if ipiv[k] == 0:
                            if abs(a[j, k]) >= big:
                                big = abs(a[j, k])
                                irow, icol = j, k
                        elif ipiv[k] > 1:
                            raise ArithmeticError("mre: singular Gram matrix")
            ipiv[icol] += 1
            if irow != icol:
                a[[irow, icol], :] = a[[icol, irow], :]
                b[irow], b[icol] = b[icol], b[irow]
            if a[icol, icol] == 0:
                raise ArithmeticError("mre: singular Gram matrix")
            pivinv = 1.0 / a[icol, icol]
            a[icol, :] = a[icol, :] * pivinv
            b[icol] = b[icol] * pivinv
            for ll in range(n):
                if ll != icol:
                    dum = a[ll, icol]
                    a[ll, icol] = 0
                    a[ll, :] = a[ll, :] - a[icol, :] * dum
                    b[ll] = b[ll] - b[icol] * dum
        return b

    def get(self, op, trial, phi, para, rho=None):
        """mre.F90:68-146: trial = the combination of the stored solutions
        that minimises |op(trial) - phi| (phi itself with none stored)."""
        lat = self.lat
        if self.nvec == 0 or self.rank == 0:
            lat.field_copy(trial, phi)
            return
        if self.rank == 1:
            lat.field_copy(trial, self.vec[0])
            return
        self._gram_schmidt()
        r = self.rank
        for i in range(r):
            lat.op_dev(op, self.mv[i], self.vec[i], para, rho=rho)
        bb = np.array(lat.field_cdot_pairs([(self.vec[i], phi) for i in range(r)]), complex)
        upper = [(i, j) for i in range(r) for j in range(i, r)]
        dots = lat.field_cdot_pairs([(self.mv[i], self.mv[j]) for i, j in upper])
        ga = np.zeros((r, r), complex)
        for (i, j), v in zip(upper, dots):
            if i == j:
                ga[i, i] = v.real
            else:
                ga[i, j] = v
                ga[j, i] = np.conj(v)
        x = self._gauss_jordan(ga, bb)
        lat.field_caxpby(trial, 0.0, x[0], self.vec[0])
        for i in range(1, r):
            lat.field_caxpby(trial, 1.0, x[i], self.vec[i])


I_SG, I_SD, I_SF1, I_SF2 = 0, 1, 2, 3   # force monitor slots (hmc_forces.F90)


class Hmc:
    """HMC for N_f = 2 clover-Wilson fermions (BQCD models A, B, C: one
    pseudofermion, or two with Hasenbusch's W = M~ + rho) on one Lattice.

    beta, kappa, csw, rho, traj_length, ntau, m_scale, model as in BQCD's
    input (tau = traj_length / ntau, bqcd.F90:175).  Solves stop on BQCD's
    absolute rule rtr <= rest.  solver = "cg" is the FP64 CG of cg.F90;
    "mixed" is the path of BQCD's QUDA hook (invert_quda.F90): int16 sloppy
    iterations with FP64 reliable updates, the stop checked on the true FP64
    residual.  A solver that does not converge raises, as cg.F90 dies,
    unless cg_log == 2 (solver_ignore_no_convergence 2 of BQCD's input: the
    FP64 CG then stops after maxiter iterations and the trajectory goes on,
    as in the reference's benchmark inputs)."""

    def __init__(self, lat, beta, kappa, csw, rho, traj_length, ntau, m_scale, model="C", rest=1e-5,
                 maxiter=1000, mre_n_vec=7, solver="cg", cg_log=0):
        self.lat = lat
        self.beta = beta
        self.para = HmcPara(kappa=kappa, csw=csw, rho=rho)
        self.csw_kappa = self.para.csw_kappa
        self.tau = traj_length / ntau
        self.ntau = ntau
        self.m_scale = m_scale
        self.model = model
        self.hasenbusch = model != "A"
        self.rest = rest
        self.maxiter = maxiter
        self.cg_log = cg_log
        if solver not in ("cg", "mixed"):
            raise ValueError("solver must be 'cg' or 'mixed'")
        self.solver = solver
        self.phi = lat.field()
        self.phi2 = lat.field()
        self.phi_bck = lat.field()
        self.tmp = lat.field()
        self.a = lat.field()
        self.b = lat.field()
        self.mre1 = Mre(lat, mre_n_vec)
        self.mre2 = Mre(lat, mre_n_vec)
        self.volume = 2 * lat.volh
        if self.csw_kappa != 0.0:
            lat.clover_init(self.csw_kappa)

    # ---- solver and monitors ----
    def _solve(self, op, hx, hb):
        rho = self.para.rho if op == "w_dagger_w" else 0.0
        if self.solver == "cg":
            it, info = self.lat.cg_dev(hx, hb, self.para, self.rest, maxiter=self.maxiter, log=self.cg_log, rho=rho)
        else:
            from . import PREC_HALF
            info = self.lat.solve_dev(hx, hb, self.para, precision=PREC_HALF, tol=self.rest, relative=False,
                                      maxiter=self.maxiter, rho=rho)
            if not info.converged:
                raise RuntimeError("mixed-precision solve did not converge: %s" % info.as_dict())
            it = info.niter
        self.cg_seconds += info.seconds
        self.cg_ncall += 1
        self.cg_niter_tot += it
        self.cg_niter_max = max(self.cg_niter_max, it)
        return it

    def _forces_old(self):
        if self.hasenbusch:
            self.lat.mom_mark()

    def _forces_new(self, step, which):
        """hmc_forces.F90:65-104: rms change of p per link generator / |step|."""
        if not self.hasenbusch:
            return
        f = self.lat.mom_change() / (8.0 * self.volume * 4.0)
        f = math.sqrt(f) / abs(step)
        self.f_count[which] += 1.0
        self.f_avg[which] += f
        self.f_max[which] = max(self.f_max[which], f)

    # ---- pseudofermions and forces ----
    def _init_phi(self):
        """hmc_init_phi.F90:28-79."""
        lat = self.lat
        lat.field_gauss(self.tmp, 0.5)
        sf1 = lat.field_cdot(self.tmp, self.tmp).real
        lat.op_dev("w_mult_dag", self.phi, self.tmp, self.para)
        sf2 = 0.0
        if self.hasenbusch:
            lat.field_gauss(self.tmp, 0.5)
            sf2 = lat.field_cdot(self.tmp, self.tmp).real
            lat.op_dev("mtil_dag", self.phi2, self.tmp, self.para)
            self._solve("w_dagger_w", self.tmp, self.phi2)
            lat.op_dev("w_mult", self.phi2, self.tmp, self.para)
        return sf1, sf2

    def _dsf1(self, step, calc_sf):
        """dsf1.F90:28-82: S_f1 = phi^+ (W^+W)^-1 phi."""
        lat = self.lat
        self.mre1.get("w_mult", self.a, self.phi, self.para)
        self.it_f1 += self._solve("w_dagger_w", self.a, self.phi)
        self.mre1.put(self.a, calc_sf)
        lat.op_dev("w_mult", self.b, self.a, self.para)
        sf = lat.field_cdot(self.b, self.b).real if calc_sf else 0.0
        self._forces_old()
        lat.dsf_dev(step, self.para, self.a, self.b)
        self._forces_new(step, I_SF1)
        return sf

    def _dsf2(self, step, calc_sf):
        """dsf2.F90:28-80: S_f2 = phi2^+ W (M~^+M~)^-1 W^+ phi2."""
        if not self.hasenbusch:
            return 0.0
        lat = self.lat
        lat.op_dev("w_mult_dag", self.b, self.phi2, self.para)
        self.mre2.get("mtil", self.a, self.b, self.para, rho=0.0)
        self.it_f2 += self._solve("mtdagmt", self.a, self.b)
        self.mre2.put(self.a, calc_sf)
        lat.op_dev("mtil", self.b, self.a, self.para)
        sf = lat.field_cdot(self.b, self.b).real if calc_sf else 0.0
        lat.field_caxpby(self.b, 1.0, -1.0, self.phi2)
        self._forces_old()
        lat.dsf_dev(step, self.para, self.a, self.b)
        self._forces_new(step, I_SF2)
        return sf

    def _dsd(self, step):
        """dsd.F90:28-49: the clover determinant force."""
        if self.csw_kappa != 0.0:
            self._forces_old()
            self.lat.dsd_dev(step, self.para)
            self._forces_new(step, I_SD)

    def _dsg(self, step):
        """dsg.F90:28-53: the gauge force."""
        if self.beta != 0.0:
            self._forces_old()
            self.lat.dsg_dev(step, self.beta)
            self._forces_new(step, I_SG)

    # ---- integrator ----
    def _p_ir(self, step, calc_sf):
        """hmc_integrator.F90: the outer (infrared) time scale."""
        if self.model == "A":
            self.sf1 = self._dsf1(step, calc_sf)
            self._dsd(step)
        elif self.model == "B":
            self.sf1 = self._dsf1(step, calc_sf)
            self.sf2 = self._dsf2(step, calc_sf)
            self._dsd(step)
        else:
            self.sf2 = self._dsf2(step, calc_sf)

    def _p_uv(self, step, calc_sf):
        """hmc_integrator.F90: the inner (ultraviolet) time scale."""
        self._dsg(step)
        if self.model not in ("A", "B"):
            self.sf1 = self._dsf1(step, calc_sf)
            self._dsd(step)

    def _leap_frog(self):
        """hmc_leap_frog.F90:28-79: nested leapfrog, m_scale inner steps."""
        calc_sf = False
        step_ir, step_uv = 0.5 * self.tau, 0.5 * self.tau / self.m_scale
        self._p_ir(step_ir, calc_sf)
        self._p_uv(step_uv, calc_sf)
        step_ir, step_uv = self.tau, self.tau / self.m_scale
        for itau in range(1, self.ntau + 1):
            for is_ in range(1, self.m_scale + 1):
                self.lat.hmc_u_dev(step_uv, self.csw_kappa)
                if itau == self.ntau and is_ == self.m_scale:
                    step_ir *= 0.5
                    step_uv *= 0.5
                    calc_sf = True
                self._p_uv(step_uv, calc_sf)
            self._p_ir(step_ir, calc_sf)

    def _hamiltonian(self, sf1, sf2):
        lat = self.lat
        sd = lat.clover_action(ODD) if self.csw_kappa != 0.0 else 0.0
        sg = lat.sg()
        return sd + lat.mom_action() + sg * self.beta + sf1 + sf2, sg

    def _reset_stats(self):
        self.cg_ncall = self.cg_niter_tot = self.cg_niter_max = 0
        self.cg_seconds = 0.0
        self.it_f1 = self.it_f2 = 0
        self.f_count = [0.0] * 4
        self.f_avg = [0.0] * 4
        self.f_max = [0.0] * 4

    def init_phi(self):
        """New pseudofermions on the current links (hmc_init_phi.F90);
        returns their actions (S_f1, S_f2)."""
        self._reset_stats()
        return self._init_phi()

    def md_evolve(self):
        """The molecular-dynamics part of a trajectory alone: the nested
        leapfrog from the current links and momenta with the pseudofermions
        fixed; returns the fermion actions (S_f1, S_f2) at the end."""
        self._reset_stats()
        self.sf1 = self.sf2 = 0.0
        self._leap_frog()
        return self.sf1, self.sf2

    def trajectory(self, force_accept=False):
        """hmc.F90:69-216: one trajectory; returns its record as a dict."""
        lat = self.lat
        self._reset_stats()
        lat.gauge_save()
        lat.field_copy(self.phi_bck, self.phi)
        lat.mom_gauss()
        sf1_old, sf2_old = self._init_phi()
        h_old, _ = self._hamiltonian(sf1_old, sf2_old)
        self.sf1 = self.sf2 = 0.0
        self._leap_frog()
        h_new, sg_new = self._hamiltonian(self.sf1, self.sf2)
        exp_dh = math.exp(h_old - h_new)
        accepted = True if force_accept else lat.ranf() < exp_dh
        if not accepted:
            lat.gauge_restore(self.csw_kappa)
            lat.field_copy(self.phi, self.phi_bck)
        return {
            "accepted": accepted, "exp_dh": exp_dh, "dh": h_new - h_old,
            "plaq_energy": (sg_new if accepted else lat.sg()) / (6.0 * self.volume),
            "it_f1": self.it_f1, "it_f2": self.it_f2,
            "cg_calls": self.cg_ncall, "cg_it_tot": self.cg_niter_tot, "cg_it_max": self.cg_niter_max,
            "cg_seconds": self.cg_seconds,
            "f_avg": [a / c if c else a for a, c in zip(self.f_avg, self.f_count)],
            "f_max": list(self.f_max),
        }


def quenched_trajectory(lat, beta, traj_length, nsteps, force_accept=False):
    """One pure-gauge HMC trajectory (BQCD with no fermions: the gauge force
    of dsg.F90 in a plain leapfrog of nsteps, hmc_u.F90 updates), for
    bringing a synthetic start configuration to equilibrium at beta before
    dynamical trajectories.  Returns (accepted, dH, plaquette <Re Tr P>/3)."""
    dt = traj_length / nsteps
    lat.gauge_save()
    lat.mom_gauss()
    h_old = lat.mom_action() + beta * lat.sg()
    lat.dsg_dev(0.5 * dt, beta)
    for k in range(nsteps):
        lat.hmc_u_dev(dt, 0.0)
        lat.dsg_dev(dt if k < nsteps - 1 else 0.5 * dt, beta)
    sg = lat.sg()
    dh = lat.mom_action() + beta * sg - h_old
    accepted = force_accept or lat.ranf() < math.exp(-dh)
    if not accepted:
        lat.gauge_restore(0.0)
        sg = lat.sg()
    return accepted, dh, 1.0 - sg / (6.0 * 2 * lat.volh)
