/*
 * bqcdg.h -- C ABI of the B200 (sm_100a) implementation of BQCD's fermion hot
 * path: the even-odd preconditioned clover-Wilson operator, the M^+M
 * conjugate-gradient solver and the pseudofermion force.
 *
 * Every entry point takes plain host pointers in BQCD's own Fortran layouts
 * (defs.h:64-78), so BQCD's HMC driver can reach it through iso_c_binding:
 *
 *   SPINCOL_FIELD   complex(4,3,volh)        double[volh][3][4][2]   (one parity)
 *   GAUGE_FIELD     complex(3,3,volh,0:1,4)  double[4][2][volh][3][3][2]
 *   CLOVER_FIELD_A  type_clover_a(2,volh,0:1) double[2][volh][2][36]  (18 complex,
 *   CLOVER_FIELD_B  type_clover_b(2,volh,0:1)  packed as clover/clover.h:28-82)
 *   GENERATOR_FIELD real(8,volh,0:1,4)       double[4][2][volh][8]
 *
 * Site indices are BQCD's even/odd index i = ilex(x,y,z,t)/2 with parity
 * (x+y+z+t) mod 2 (index.F90:26-76) on a single process (volh_tot = volh).
 * Parities: 0 = EVEN, 1 = ODD.
 *
 * Boundary conditions: inside BQCD every fermion operation runs on links
 * bracketed by flip_bc() (flip_bc.F90:97-121).  bqcdg_load_gauge() takes a
 * flag saying whether the array passed carries that sign; the device keeps
 * periodic links and applies the fermion boundary sign inside the kernels, so
 * every operator below equals BQCD's on the flipped links in either case.
 *
 * All calls return BQCDG_OK (0) or a BQCDG_E* status; none aborts the
 * process (the reference calls die(), misc.F90:28-37; a Fortran shim maps the
 * status back).  A context is single-caller: like the reference's routines
 * (which keep save-scratch, cg.F90:69) it is not reentrant.
 */
#ifndef BQCDG_H
#define BQCDG_H

#ifdef __cplusplus
extern "C" {
#endif

#define BQCDG_OK 0
#define BQCDG_EINVAL 1       /* bad argument */
#define BQCDG_ECUDA 2        /* CUDA runtime error (context is left usable) */
#define BQCDG_ENOCONV 3      /* solver did not converge (cg.F90:121-124) */
#define BQCDG_ENAN 4         /* residual became NaN/Inf */
#define BQCDG_ENOGAUGE 5     /* no gauge field loaded */
#define BQCDG_ENOCLOVER 6    /* clover term requested but not loaded/built */
#define BQCDG_ENOMEM 7       /* device allocation failed */
#define BQCDG_EUNSUPPORTED 8 /* e.g. h != 0 in the QUDA hook (invert_quda.F90:298-301) */
#define BQCDG_ENOTSU3 9      /* links not SU(3): 12-real sloppy storage impossible */
#define BQCDG_ENODEVICE 10   /* no CUDA device */
#define BQCDG_ECHECKSUM 11   /* a configuration file disagrees with the check sum of its info file */
#define BQCDG_EIO 12         /* a file could not be opened, read or written, or is not in the expected form */

typedef struct bqcdg_ctx bqcdg_ctx;

/* the operator parameters of type(hmc_para) (modules/typedef_hmc.F90:32-44)
 * that the hot path reads: M~ = A_ee - kappa^2/(1+h^2) D_eo A_oo^-1 D_oe
 * (m_tilde.F90:43-77), W = M~ + rho (w_mult.F90:28-44) */
typedef struct {
  double kappa;
  double csw_kappa; /* c_sw * kappa; 0 selects the Wilson operator */
  double h;         /* external field of h_mult.F90 */
  double rho;       /* Hasenbusch shift; 0 gives M~^+M~ (mtdagmt) */
} bqcdg_params;

/* type(type_cg_para) (cg.F90:30-34) */
typedef struct {
  float rest;   /* ABSOLUTE stop: |r|^2 <= rest, FP32 like the reference (cg.F90:111) */
  int maxiter;
  int log;      /* 2: no convergence is not an error (cg.F90:121) */
} bqcdg_cg_para;

/* precision of the inner CG iterations */
#define BQCDG_PREC_DOUBLE 0 /* all FP64 */
#define BQCDG_PREC_SINGLE 1 /* FP32 fields, FP64 reliable updates */
#define BQCDG_PREC_HALF 2   /* int16 fields with norms, FP32 r/x, FP64 reliable updates */

typedef struct {
  int precision;      /* BQCDG_PREC_* */
  int maxiter;
  int relative;       /* 1: stop on |r|^2 <= tol^2 |b|^2, 0: |r|^2 <= tol (absolute) */
  double tol;
  double delta;       /* reliable update when |r| < delta * max|r| since the last one */
  int check_true_residual; /* 1: recompute |b - A x|^2 in FP64 at the end */
  int time_kernels;   /* 1: time the first-half stencil launches of the second
                         iteration of every batch of queued iterations with
                         CUDA events (FP64 and single-RHS sloppy solves) */
  int rhs_per_thread; /* batched solves: right-hand sides each stencil thread serves
                         (1, 2, 4; 0 = the fastest, timed once per context) */
} bqcdg_solver_opts;

typedef struct {
  int niter;              /* inner iterations */
  int reliable_updates;   /* FP64 residual recomputations */
  double rtr;             /* final iterated |r|^2 */
  double true_rtr;        /* final |b - A x|^2 in FP64 (if checked) */
  double b2;              /* |b|^2 */
  double seconds;         /* device time of the solve (CUDA events) */
  double stencil_ms;      /* summed device time of the timed launches of the
                             dominant stencil kernel (time_kernels) */
  int stencil_launches;   /* how many launches were timed */
  int converged;
  int kernel_launches;    /* all kernels this solve launched */
} bqcdg_solve_info;

/* ---- context ---------------------------------------------------------- */
/* L: lattice extents (x,y,z,t), all even; bc: fermion boundary conditions
 * (+1/-1, boundary_conditions_fermions of the input file) */
int bqcdg_create(bqcdg_ctx **ctx, const int L[4], const int bc[4], int device);
int bqcdg_destroy(bqcdg_ctx *ctx);
const char *bqcdg_error_string(int status);
/* volh of the context */
int bqcdg_volh(const bqcdg_ctx *ctx);
/* device memory held by the context, bytes */
long long bqcdg_device_bytes(const bqcdg_ctx *ctx);
/* free device memory that later calls re-create on demand, for lattices that
 * fill the GPU.  BQCDG_SCRATCH_SOLVER: the solver's work vectors, the batch
 * buffers and the Fortran-layout staging buffer.  BQCDG_SCRATCH_HMC: the
 * resident momenta (until bqcdg_mom_gauss or bqcdg_mom_set makes new ones
 * the momentum entry points return BQCDG_EINVAL), the saved links of
 * bqcdg_gauge_save and the force work buffers.  Links, clover, the sloppy
 * copies of both and the resident fields are kept. */
#define BQCDG_SCRATCH_SOLVER 1
#define BQCDG_SCRATCH_HMC 2
int bqcdg_release_scratch(bqcdg_ctx *ctx, int what);

/* ---- fields ----------------------------------------------------------- */
/* conf%u; flipped = 1 if flip_bc() has been applied to the array.
 * Replaces load_gauge_quda (invert_quda.F90:134). */
int bqcdg_load_gauge(bqcdg_ctx *ctx, const double *u, int flipped);
int bqcdg_get_gauge(bqcdg_ctx *ctx, double *u, int flipped);
/* conf%a, conf%i, conf%b (both parities, any may be NULL).  Replaces
 * load_clover_quda (invert_quda.F90:138). */
int bqcdg_load_clover(bqcdg_ctx *ctx, const double *a, const double *ainv, const double *b);
int bqcdg_get_clover(bqcdg_ctx *ctx, double *a, double *ainv, double *b);
/* load_clover for the solver only: from the same arrays, A of the even
 * sites and A^-1 of the odd ones, the two parts M~ and W read; a third of
 * the bytes of bqcdg_load_clover(a, ainv, b).  The other parts are released
 * (entry points that need them then return BQCDG_ENOCLOVER). */
int bqcdg_load_clover_solver(bqcdg_ctx *ctx, const double *a, const double *ainv);
/* clover_init(a, i, b, u, csw_kappa) (clover/clover_init.F90:28) on the
 * device, from the loaded links */
int bqcdg_clover_init(bqcdg_ctx *ctx, double csw_kappa);
/* clover_init for the even-odd solver only: A of the even sites and A^-1 of
 * the odd sites (clover_init.F90:28 + clover_inv.F90:29), the two fields that
 * M~ and W use; the other four (A odd, A^-1 even, the B factors) are released.
 * A third of the memory of bqcdg_clover_init, for lattices where all six do
 * not fit; entry points that need the others then return BQCDG_ENOCLOVER. */
int bqcdg_clover_init_solver(bqcdg_ctx *ctx, double csw_kappa);
/* the clover term for any hopping parameter: clover_init.F90:46-77 builds
 * each chiral block as 1 + (-c_sw kappa / 8)(p +- q) from field strengths
 * that do not depend on kappa.  This stores T = (-c_sw / 8)(p +- q) of the
 * even and the odd sites from the loaded links; the operators then form
 * A(kappa) = 1 + kappa T and the LDL^+ solve of A(kappa) per site, at the
 * kappa of their parameters (p->csw_kappa only has to be nonzero).  It is
 * what bqcdg_solve_batch_kappa needs for systems with different kappa.
 * Entry points that read BQCD's clover blocks themselves (clover_mult_*,
 * get_clover, the forces) return BQCDG_EUNSUPPORTED until a clover_init or
 * load_clover replaces T. */
int bqcdg_clover_init_t(bqcdg_ctx *ctx, double csw);
/* clover_action(b(1,1,ODD)) (clover/clover_action.F90:29) */
int bqcdg_clover_action(bqcdg_ctx *ctx, int eo, double *action);

/* ---- operators on host spinor fields ----------------------------------- */
/* d(e,o,out,in,u) / d_dag (d/D21.F90:29): out(parity e) = D_eo in(parity o) */
int bqcdg_d(bqcdg_ctx *ctx, int e, int o, double *out, const double *in);
int bqcdg_d_dag(bqcdg_ctx *ctx, int e, int o, double *out, const double *in);
/* clover_mult_a(out, a(eo), in) (clover/clover_mult_a.F90:30) */
int bqcdg_clover_mult_a(bqcdg_ctx *ctx, int eo, double *out, const double *in);
/* clover_mult_ao(i(eo), x) (clover/clover_mult_ao.F90:30): x = A^-1 x */
int bqcdg_clover_mult_ao(bqcdg_ctx *ctx, int eo, double *x);
/* clover_mult_b(b(eo), x) (clover/clover_mult_b.F90:30): x = B^-1 x (LDL^+) */
int bqcdg_clover_mult_b(bqcdg_ctx *ctx, int eo, double *x);
/* mtil / mtil_dag (m_tilde.F90:43,80), mtdagmt (mtdagmt.F90:28),
 * w_mult / w_mult_dag / w_dagger_w (w_mult.F90:28,46,64) */
int bqcdg_mtil(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);
int bqcdg_mtil_dag(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);
int bqcdg_mtdagmt(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);
int bqcdg_w_mult(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);
int bqcdg_w_mult_dag(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);
int bqcdg_w_dagger_w(bqcdg_ctx *ctx, double *out, const double *in, const bqcdg_params *p);

/* ---- solvers ------------------------------------------------------------ */
/* cg(matrix_mult, x, b, para, conf, iterations) (cg.F90:51) with
 * matrix_mult = w_dagger_w (rho = p->rho) or mtdagmt (rho = 0): FP64 CG, x is
 * the initial guess on input, absolute stop |r|^2 <= cgp->rest.  Returns
 * BQCDG_ENOCONV on no convergence unless cgp->log == 2 (then BQCDG_OK). */
int bqcdg_cg(bqcdg_ctx *ctx, double *x, const double *b, const bqcdg_params *p, const bqcdg_cg_para *cgp,
             int *iterations, bqcdg_solve_info *info);
/* quda_solver(matrix_mult, x, b, para, conf, iterations, rho)
 * (invert_quda.F90:96): mixed-precision CG (int16 sloppy, FP64 reliable
 * updates) to the same absolute criterion, then the FP64 true residual
 * |b - W^+W x|^2 <= rest is re-checked on the device as invert_quda.F90:155-168
 * does on the host.  Gauge and clover must be loaded (the reference uploads
 * them on every call; here they stay resident until reloaded). */
int bqcdg_quda_solver(bqcdg_ctx *ctx, double *x, const double *b, const bqcdg_params *p,
                      const bqcdg_cg_para *cgp, int *iterations, bqcdg_solve_info *info);
/* general entry: any precision, relative or absolute tolerance */
int bqcdg_solve(bqcdg_ctx *ctx, double *x, const double *b, const bqcdg_params *p, const bqcdg_solver_opts *o,
                bqcdg_solve_info *info);
void bqcdg_solver_opts_default(bqcdg_solver_opts *o);

/* ---- forces ------------------------------------------------------------- */
/* dsf(p, conf, step, para, a, b) (dsf.F90:28): p += hopping + clover part of
 * the pseudofermion force for the even fields a, b.  The gauge field must be
 * loaded; the clover part needs conf%b/conf%i of the odd sites. */
int bqcdg_dsf(bqcdg_ctx *ctx, double *p, double step, const bqcdg_params *par, const double *a, const double *b);
/* clover_dsf(eo, p, b, a, s, u) (clover/clover_d.F90:78) */
int bqcdg_clover_dsf(bqcdg_ctx *ctx, int eo, double *p, const double *b, const double *a, double s);
/* clover_dsd(eo, p, b, s, u) (clover/clover_d.F90:40): determinant force */
int bqcdg_clover_dsd(bqcdg_ctx *ctx, int eo, double *p, double s);

/* ---- seeded synthetic inputs on the device ------------------------------ */
/* the context's copy of the 48-bit LCG state of ranf.F90: ranset(seed, skip)
 * (ranf.F90:87-121; seed 0 = the default seed) and ranget */
int bqcdg_ranset(bqcdg_ctx *ctx, long long seed, long long skip);
int bqcdg_ranget(bqcdg_ctx *ctx, long long *seed);
/* conf_hot / conf_cold (conf.F90:172-217) into the context's links, drawing
 * from the context's RNG stream exactly as ran_gauss_volh (ran.F90:28-110) */
int bqcdg_conf_hot(bqcdg_ctx *ctx);
int bqcdg_conf_cold(bqcdg_ctx *ctx);
/* n sweeps of conf_relax (cooling.F90:131-193) on the context's links */
int bqcdg_conf_relax(bqcdg_ctx *ctx, int n);
/* sg(u) (action.F90:70-123): 6 V - sum Re Tr(plaquettes) / 3 */
int bqcdg_sg(bqcdg_ctx *ctx, double *sg);

/* ---- device-resident fields (benchmarks, repeated solves) ---------------- */
/* spinor fields kept on the device between calls, addressed by handle */
int bqcdg_field_create(bqcdg_ctx *ctx, int *handle);
int bqcdg_field_upload(bqcdg_ctx *ctx, int handle, const double *host);
int bqcdg_field_download(bqcdg_ctx *ctx, int handle, double *host);
int bqcdg_field_destroy(bqcdg_ctx *ctx, int handle);
/* fill a resident field with ran_gauss_volh(12, field, var, eo) from the
 * context's RNG stream (var = 1/2 gives unit-variance complex entries) */
int bqcdg_field_gauss(bqcdg_ctx *ctx, int handle, double var);
/* solve with x, b resident (x: initial guess in, solution out) */
int bqcdg_solve_dev(bqcdg_ctx *ctx, int hx, int hb, const bqcdg_params *p, const bqcdg_solver_opts *o,
                    bqcdg_solve_info *info);
/* batched solve of nrhs systems (W^+W) x_k = b_k sharing one operator: every
 * sloppy iteration of all unconverged right-hand sides runs in the same five
 * launches, so each link and clover block is read from HBM once per site for
 * the whole batch; converged right-hand sides retire inside the kernels and
 * each gets its own FP64 reliable updates.  block = right-hand sides per
 * launch (1..16; 0 = choose by timing 1, 4, 8 and 16).  infos: nrhs entries. */
int bqcdg_solve_batch(bqcdg_ctx *ctx, int nrhs, const int *hx, const int *hb, const bqcdg_params *p,
                      const bqcdg_solver_opts *o, int block, bqcdg_solve_info *infos);
/* bqcdg_solve_batch with a shift per right-hand side: system k is
 * (W^+W) x_k = b_k with W = M~ + rho[k] (m_tilde.F90:63-73), the links and
 * clover shared.  These are the solves of the pseudofermion levels of
 * mass-preconditioned HMC, which differ only in rho (dsf1.F90:66 with
 * para%rho, dsf2.F90:64 with rho = 0); p->rho is ignored.  tol: one
 * tolerance per system in the sense of o->relative (NULL: o->tol for all). */
int bqcdg_solve_batch_shifted(bqcdg_ctx *ctx, int nrhs, const int *hx, const int *hb, const bqcdg_params *p,
                              const double *rho, const double *tol, const bqcdg_solver_opts *o, int block,
                              bqcdg_solve_info *infos);
/* bqcdg_solve_batch_shifted with a hopping parameter per right-hand side:
 * system k is (W_k^+W_k) x_k = b_k with W_k = M~(kappa[k]) + rho[k] (rho NULL:
 * p->rho for all), its own clover term from bqcdg_clover_init_t when
 * p->csw_kappa != 0 (BQCDG_ENOCLOVER otherwise) and its own hopping
 * coefficient -kappa[k]^2 / (1 + h^2) (m_tilde.F90:67).  These are the
 * systems of a spectrum of quark masses on one gauge field; their FP64
 * reliable updates and true residuals use their own operators. */
int bqcdg_solve_batch_kappa(bqcdg_ctx *ctx, int nrhs, const int *hx, const int *hb, const bqcdg_params *p,
                            const double *kappa, const double *rho, const double *tol, const bqcdg_solver_opts *o,
                            int block, bqcdg_solve_info *infos);
/* block CG over nrhs <= 16 resident systems (W^+W) x_k = b_k that share W
 * (W = M~ + p->rho), e.g. the point sources of a propagator: one Krylov
 * space for all of them (O'Leary's block CG in the residual-QR form of
 * Dubrulle, 2001), searched along nrhs directions per iteration, so the
 * systems need fewer iterations than alone.  FP32 blocks
 * (o->precision = BQCDG_PREC_SINGLE), restarted from FP64 residuals when the
 * largest residual has dropped by o->delta; a system that reaches its
 * tolerance at a restart leaves the block.  infos[k].niter: block
 * iterations until system k left; reliable_updates: restarts; true_rtr: its
 * last FP64 |b - A x|^2.  The reference solves its systems one at a time
 * (cg.F90:51). */
int bqcdg_solve_block(bqcdg_ctx *ctx, int nrhs, const int *hx, const int *hb, const bqcdg_params *p,
                      const bqcdg_solver_opts *o, bqcdg_solve_info *infos);
/* out = (W^+W) in with both resident, repeated n times; *ms = average device
 * time of one application (CUDA events on the context stream) */
int bqcdg_mdagm_dev(bqcdg_ctx *ctx, int hout, int hin, const bqcdg_params *p, int precision, int n, double *ms);
/* average device time of one even-odd stencil pass (pass 1 of mtil: D_oe,
 * Ainv_oo) at the given precision, n launches */
int bqcdg_time_pass(bqcdg_ctx *ctx, int hin, const bqcdg_params *p, int precision, int n, double *ms);
/* the same for the batched pass over nrhs right-hand sides hin[0..nrhs-1]
 * (1..16; FP32 or int16), rhs_per_thread of them per stencil thread (1, 2, 4;
 * 0 = the batched solver's timed choice): average device time of one launch
 * serving all */
int bqcdg_time_pass_batch(bqcdg_ctx *ctx, int nrhs, const int *hin, const bqcdg_params *p, int precision,
                          int rhs_per_thread, int n, double *ms);

/* ---- configuration files (conf.F90:219-470) ---------------------------- */
/* BQCD's gauge configuration format: one binary file per time slice t,
 * <base>.<tt>.u (tt: t with at least two digits, files.F90:219-234), holding
 * NZ records (one per z) of the sites of that slice in y, x order, each site
 * the first two columns of its four links as 24 big-endian REAL(8) complex
 * numbers, rows fastest, then columns, then mu (conf_seq, conf.F90:219-259;
 * field_io, comm/field_io_mpi.F90; swap_endian8, misc.F90:197-240); and an
 * info file <base>.info with the ConfInfoHeader block (conf_info.F90:28-63)
 * and one line per slice file with its POSIX cksum and byte count
 * (write_cksum, conf_info.F90:165-190; cksum.c).  On the device each slice
 * is reordered, byte-swapped and check-summed in one pass. */
typedef struct {
  int run, traj;          /* Run, Traj */
  int ensemble[2];        /* ensemble, former_ensemble */
  double beta[2], kappa[2], csw[2], csw_kappa[2], h[2];
  double plaq_energy;     /* PlaqEnergy = sg / (6 V); written: computed from the links */
  int L[4], bc[4];        /* L, bc_fermions; written: the context's */
} bqcdg_conf_meta;
/* conf_write: the resident links to the slice files and the info file */
int bqcdg_conf_write(bqcdg_ctx *ctx, const char *base, bqcdg_conf_meta *meta);
/* conf_read: the configuration named by an info file becomes the resident
 * links (the third columns rebuilt by u_complete, su3.F90:301-310).  Slice
 * file names are taken relative to the info file's directory.  A lattice
 * other than the context's gives BQCDG_EINVAL, a check-sum mismatch
 * BQCDG_ECHECKSUM (conf.F90 dies in both cases); afterwards no gauge field
 * is loaded.  meta receives the header. */
int bqcdg_conf_read(bqcdg_ctx *ctx, const char *info_file, bqcdg_conf_meta *meta);

/* ---- resident HMC pieces ------------------------------------------------ */
/* With these a trajectory keeps the links, the momenta and its spinor fields
 * in device memory: nothing crosses PCIe between the start and the
 * accept/reject step.  Momenta are one device field per context in BQCD's
 * GENERATOR_FIELD layout, real(8, volh, 0:1, 4) (defs.h:71); spinor fields
 * are the resident handles above. */
/* hmc_init_p.F90:28-45: momenta from ran_gauss_volh(4, p(:,:,eo,mu), 1, eo),
 * mu outer, eo inner, from the context's RNG stream */
int bqcdg_mom_gauss(bqcdg_ctx *ctx);
int bqcdg_mom_set(bqcdg_ctx *ctx, const double *p);
int bqcdg_mom_get(bqcdg_ctx *ctx, double *p);
/* kinetic term of the Hamiltonian, sp = 1/2 sum p^2 (action.F90) */
int bqcdg_mom_action(bqcdg_ctx *ctx, double *sp);
/* force monitor (hmc_forces.F90:65-104): mark saves p, change returns
 * sum (p_marked - p)^2 */
int bqcdg_mom_mark(bqcdg_ctx *ctx);
int bqcdg_mom_change(bqcdg_ctx *ctx, double *d2);
/* dsg.F90:28-53: gauge force p += (-step beta / 3) Im Tr(lambda_j U staples) */
int bqcdg_dsg_dev(bqcdg_ctx *ctx, double step, double beta);
/* hmc_u.F90:28-69: U <- exp(i step p) U (gen2u, su3.F90:28-193), u_normalize,
 * then clover_init of the new links when csw_kappa != 0 */
int bqcdg_hmc_u_dev(bqcdg_ctx *ctx, double step, double csw_kappa);
/* dsf.F90:28-110 into the resident momenta from resident fields a, b */
int bqcdg_dsf_dev(bqcdg_ctx *ctx, double step, const bqcdg_params *p, int ha, int hb);
/* dsd.F90:28-49: det-term force clover_dsd(ODD, p, b, -2 step csw_kappa/8) */
int bqcdg_dsd_dev(bqcdg_ctx *ctx, double step, const bqcdg_params *p);
/* links saved on the device and restored on a rejected trajectory
 * (hmc.F90:195-199); restore rebuilds the clover when csw_kappa != 0 */
int bqcdg_gauge_save(bqcdg_ctx *ctx);
int bqcdg_gauge_restore(bqcdg_ctx *ctx, double csw_kappa);
/* the next ranf() of the context's stream (ranf.F90), for the Metropolis step */
int bqcdg_ranf(bqcdg_ctx *ctx, double *r);
/* operators on resident fields: which = 0 mtil, 1 mtil_dag, 2 mtdagmt,
 * 3 w_mult, 4 w_mult_dag, 5 w_dagger_w (m_tilde.F90:43-114, mtdagmt.F90:28,
 * w_mult.F90:28-84) */
int bqcdg_op_dev(bqcdg_ctx *ctx, int which, int hout, int hin, const bqcdg_params *p);
/* cg(matrix_mult, x, b, para, conf, iterations) (cg.F90:51-137) on resident
 * fields: FP64, the operator fixed by p->rho as in bqcdg_cg */
int bqcdg_cg_dev(bqcdg_ctx *ctx, int hx, int hb, const bqcdg_params *p, const bqcdg_cg_para *cgp, int *iterations,
                 bqcdg_solve_info *info);
/* <a, b> = sum conj(a) b (sc_cdotc, sc.F90:224-286) and y = ay y + a x with
 * complex a (the linear combinations of mre.F90:68-213) on resident fields */
int bqcdg_field_cdot(bqcdg_ctx *ctx, int ha, int hb, double *re, double *im);
int bqcdg_field_caxpby(bqcdg_ctx *ctx, int hy, double ay, double are, double aim, int hx);
/* re[j] + i im[j] = <ha[j], hb[j]> for j < n <= BQCDG_MAX_DOT_PAIRS, in one
 * pass and one read-back: each value equals bqcdg_field_cdot's bit for bit.
 * The scalar products of one mre.F90 step (Gram-Schmidt, mre.F90:189-213,
 * and the Gram system, mre.F90:68-146) come in a few such calls. */
#define BQCDG_MAX_DOT_PAIRS 8
int bqcdg_field_cdot_pairs(bqcdg_ctx *ctx, int n, const int *ha, const int *hb, double *re, double *im);

/* ---- domain decomposition in time ---------------------------------------- */
/* The global lattice L is cut along t into nranks slabs of L[3]/nranks time
 * slices (an even number, so a slab's parity is the global one).  Slab r
 * holds the contiguous range [r V3h Lt, (r+1) V3h Lt) of BQCD's even/odd site
 * index (V3h = L[0] L[1] L[2] / 2, Lt = L[3]/nranks).  Before each stencil
 * pass every slab sends the two-spin half spinors that the t hop keeps
 * (12 reals per site) of its first slice to rank-1 and of its last slice to
 * rank+1, and the CG takes the global sums of its three scalars, as the
 * reference's MPI build does (d/D21.F90:53-72, comm/xbound_mpi.F90:418-461,
 * cg.F90:91,97,109).  U_t of each slab's last slice is sent to rank+1 once per
 * gauge field.  The operators and bqcdg_dd_cg are FP64; bqcdg_dd_solve runs
 * int16 iterations with FP32 faces and FP64 reliable updates.  The faces go
 * on a second stream while the slab interior computes.
 *
 * Two ways to run it:
 *  - bqcdg_dd_create_local: all nranks slabs in this process on one device,
 *    the faces copied between them on the device and the global sums added
 *    on the host in rank order.  Host arrays are the GLOBAL ones.
 *  - bqcdg_dd_create_nccl: one slab per process (rank `rank`, one GPU each),
 *    faces by ncclSend/ncclRecv and sums by ncclAllReduce on the slab's
 *    stream.  Rank 0 makes the id with bqcdg_dd_nccl_unique_id and hands its
 *    128 bytes to the others (any side channel).  Host arrays are the slab's
 *    own (volh = V3h Lt sites per parity).  libnccl.so.2 is opened at run
 *    time; without it both calls return BQCDG_EUNSUPPORTED.  Every call
 *    that exchanges or sums (load_gauge, op, cg, solve) is collective: all
 *    ranks make it, in the same order and with the same parameters. */
typedef struct bqcdg_dd bqcdg_dd;
int bqcdg_dd_create_local(bqcdg_dd **dd, const int L[4], const int bc[4], int nranks, int device);
int bqcdg_dd_nccl_unique_id(char *id128);
int bqcdg_dd_create_nccl(bqcdg_dd **dd, const int L[4], const int bc[4], int nranks, int rank, int device,
                         const char *id128);
int bqcdg_dd_destroy(bqcdg_dd *dd);
/* sites per parity of the host spinors this process passes */
int bqcdg_dd_volh(const bqcdg_dd *dd);
/* conf%u (flipped = 1: flip_bc applied, whose sign is on the global last
 * slice only) and conf%a, conf%i of both parities (CLOVER_FIELD_A layout) */
int bqcdg_dd_load_gauge(bqcdg_dd *dd, const double *u, int flipped);
int bqcdg_dd_load_clover(bqcdg_dd *dd, const double *a, const double *ainv);
/* out = op(in) on even-site spinors: which = 0 mtil, 1 mtil_dag, 2 mtdagmt,
 * 3 w_mult, 4 w_mult_dag, 5 w_dagger_w (as bqcdg_op_dev), 6 d(EVEN, ODD) and
 * 7 d_dag(EVEN, ODD) (in: odd sites) */
int bqcdg_dd_op(bqcdg_dd *dd, int which, double *out, const double *in, const bqcdg_params *p);
/* cg(matrix_mult, x, b, ...) (cg.F90:51-137) on the decomposed lattice:
 * FP64, x the initial guess, |r|^2 <= cgp->rest, W = M~ + p->rho */
int bqcdg_dd_cg(bqcdg_dd *dd, double *x, const double *b, const bqcdg_params *p, const bqcdg_cg_para *cgp,
                int *iterations, bqcdg_solve_info *info);
/* (W^+W) x = b on the decomposed lattice with the mixed-precision scheme of
 * bqcdg_solve (o->precision must be BQCDG_PREC_HALF: int16 iterations, FP32
 * r and x_s, FP64 reliable updates), x the initial guess; stop as in
 * bqcdg_solve (o->relative: |r|/|b| <= o->tol, else |r|^2 <= o->tol), the
 * last residual recomputed in FP64.  The CG scalars stay on the device: the
 * two reductions of an iteration are summed over the slabs of the process in
 * slab order and over the ranks by ncclAllReduce.  BQCDG_ENOCONV when the
 * int16 iterations stop making progress or maxiter is reached. */
int bqcdg_dd_solve(bqcdg_dd *dd, double *x, const double *b, const bqcdg_params *p, const bqcdg_solver_opts *o,
                   bqcdg_solve_info *info);

/* ---- allocation-free operator ------------------------------------------- */
/* This entry point has no counterpart in the reference.  It is for callers
 * that cannot let the library allocate device memory: a framework whose pool
 * or arena allocator owns every buffer, or code that must not call cudaMalloc
 * (which may synchronise the device) in a latency-critical region.  It needs
 * no context.
 *
 * out = (W^+W) in with W = M~ + p->rho (p->rho = 0: mtdagmt), in FP64.  All
 * arrays are caller-owned DEVICE memory in the library's device layout, with
 * stride = volh rounded up to a multiple of 64:
 *   gauge     double2[4][2][9][stride]  periodic links, u(row,col) at k = col*3+row
 *   a_even    double2[36][stride]       conf%a of the even sites (chi*18 + slot)
 *   ainv_odd  double2[36][stride]       conf%i of the odd sites (may be NULL for csw = 0)
 *   in, out   double2[12][stride]       even-site spinors, k = colour*4+spin
 * The fermion boundary signs bc are applied inside the kernels.  stream is a
 * cudaStream_t (NULL: the default stream); the call only enqueues work.
 *
 * Its two intermediate fields live in one static device array sized for
 * volh <= BQCDG_NOALLOC_MAX_VOLH (6.3 MB per device, held until the process
 * exits); larger lattices are rejected with BQCDG_EINVAL.  The first call on
 * a device looks up that array's device address (cudaGetSymbolAddress) with
 * the device current.  Under CUDA's lazy module loading that look-up is also
 * what loads the library's kernels on the device and allocates the array, so
 * the first call is the one that may allocate and synchronise: make it before
 * any stream capture, before a latency-critical region and before a pool or
 * arena takes over the device's memory, and from one host thread at a time
 * (the look-up is not locked).  The address is kept per device ordinal for
 * the rest of the process: after a cudaDeviceReset, or under another CUDA
 * context than the one current at the first call, it is stale and the entry
 * point must not be called again.  All calls on a device share the array and
 * it keeps the last call's contents: calls that overlap on the GPU race.
 * Nothing in it needs to start at zero, since each call writes every site it
 * later reads. */
#define BQCDG_NOALLOC_MAX_VOLH 16384
int bqcdg_mdagm_noalloc(const int L[4], const int bc[4], const double *gauge, const double *a_even,
                        const double *ainv_odd, const bqcdg_params *p, const double *in, double *out,
                        void *stream);

#ifdef __cplusplus
}
#endif
#endif
