/*
 * pot3d_gpu.h -- C-ABI of libpot3d_gpu.so, the B200 (sm_100a) PCG hot path
 * of POT3D.
 *
 * Two groups of entry points:
 *
 * 1. The three legacy symbols of POT3D's external LU solver
 *    (module external_lu_solver_interface, src/pot3d.F90:581-609), with the
 *    same signatures and semantics as src/lusol_cusparse.c:64,309,374, so a
 *    -DCUSPARSE build of the Fortran host links against this library instead
 *    of the cuSPARSE shim.  Like the shim they take DEVICE pointers, keep a
 *    single global instance, print "ERROR! ..." and exit(1) on failure.
 *
 * 2. pot3d_gpu_* : a whole-solve offload that replaces the body of
 *    cgsolve (src/pot3d.F90:4231-4369) and the pieces of potfld around it
 *    (RHS, phi finalisation, energies).  They return a status code
 *    (POT3D_OK = 0) and never exit; pot3d_gpu_last_error() describes the
 *    most recent failure on the calling thread.
 *
 * Layout conventions follow the reference exactly:
 *  - 1-D mesh arrays are the local_mesh arrays of one rank (Fortran element
 *    k is C element k-1): r,dr (nr-1); rh,drh (nr); t,dt,st (nt-1);
 *    th,dth,sth (nt); p,dp,ph,dph (np).
 *  - CG vectors are the packed interior vectors of potfld, length
 *    N = (nr-2)*(nt-2)*(np-2), index (k-2)*(nt-2)*(nr-2)+(j-2)*(nr-2)+(i-2)
 *    (src/pot3d.F90:3917,4930).
 *  - 2-D/3-D fields (br0, phi) are Fortran column-major: br0(nt,np),
 *    phi(nr,nt,np).
 */
#ifndef POT3D_GPU_H
#define POT3D_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Legacy external LU solver (drop-in for src/lusol_cusparse.c)            */
/* ---------------------------------------------------------------------- */

/* Replaces load_external_lu_solver, src/lusol_cusparse.c:64-302
 * (Fortran interface src/pot3d.F90:587-593).  CSR_LU/CSR_I/CSR_J are DEVICE
 * pointers to the 1-based CSR built by diacsr (src/pot3d.F90:4870-5018);
 * N rows, M = CSR_I[N] as returned by getM.  Factorises CSR_LU in place into
 * ILU(0) L\U (unit lower L, upper U), FP32, with the row operations of ilu0
 * (src/pot3d.F90:4717-4813).  Keeps the pointers for external_lu_solver. */
void load_external_lu_solver(float *CSR_LU, int *CSR_I, int *CSR_J, int N, int M);

/* Replaces external_lu_solver, src/lusol_cusparse.c:309-367
 * (src/pot3d.F90:595-600).  In place on the DEVICE FP64 vector x of length
 * N: x <- (double)(U^-1 L^-1 (float)x), the sweeps of lusol
 * (src/pot3d.F90:5227-5302) in FP32. */
void external_lu_solver(double *x);

/* Replaces unload_external_lu_solver, src/lusol_cusparse.c:374-391
 * (src/pot3d.F90:602-604).  Frees what load_external_lu_solver allocated. */
void unload_external_lu_solver(void);

/* ---------------------------------------------------------------------- */
/* Whole-solve offload                                                    */
/* ---------------------------------------------------------------------- */

enum {
  POT3D_OK = 0,
  POT3D_ERR_ARG = 1,        /* invalid argument or size */
  POT3D_ERR_CUDA = 2,       /* CUDA runtime failure */
  POT3D_ERR_NOMEM = 3,      /* device allocation failed */
  POT3D_ERR_PIVOT = 4,      /* zero pivot in the ILU(0) factorisation */
  POT3D_ERR_NOT_CONVERGED = 5,
  POT3D_ERR_TIMEOUT = 6,    /* a bounded device wait ran out */
  POT3D_ERR_BREAKDOWN = 7   /* non-finite or zero curvature in PCG */
};

/* Preconditioner choice, as the namelist's ifprec (src/pot3d.F90:428). */
enum { POT3D_PREC_NONE = 0, POT3D_PREC_DIAG = 1, POT3D_PREC_ILU0 = 2 };

/* Arithmetic of the solve. */
enum {
  POT3D_FP64 = 0,          /* the reference's classical FP64 PCG */
  POT3D_FP32_REFINED = 1   /* FP32-stored inner iterations (p, q, r, the
                              ILU(0) sweeps; products formed in FP64)
                              inside FP64 reliable updates of r = b - A x */
};

typedef struct {
  int nr, nt, np;
  const double *r, *dr;           /* nr-1 */
  const double *rh, *drh;         /* nr   */
  const double *t, *dt, *st;      /* nt-1 */
  const double *th, *dth, *sth;   /* nt   */
  const double *p, *dp;           /* np   */
  const double *ph, *dph;         /* np   */
} pot3d_mesh_t;

typedef struct pot3d_gpu_solver pot3d_gpu_solver;

typedef struct {
  int ncg;           /* iterations (FP64 PCG) or total inner iterations */
  int n_refine;      /* FP64 residual replacements (refined mode) */
  double epsn;       /* final epsn as ernorm defines it (src/pot3d.F90:4432) */
  double true_resid; /* ||b - A x||_2 / ||b||_2 of the returned x, FP64 */
  double seconds;    /* device time of the iteration (CUDA events) */
  long long kernel_launches; /* kernels this library launched for the solve */
} pot3d_solve_info_t;

/* Set up a solve: copies the mesh and br0 (host pointers) to the device,
 * forms the matrix-free operator of load_matrix_pot3d_solve
 * (src/pot3d.F90:4565-4613) and the preconditioner of
 * load_preconditioner_pot3d_solve (src/pot3d.F90:4615-4715).  pm_r1 is the
 * r=R1 switch of check_input (src/pot3d.F90:1250-1285).  br1 may be NULL; if
 * given, the validation-run Neumann condition at r=R1 is used
 * (src/pot3d.F90:5420-5423) and pm_r1 is ignored.  device < 0 means the
 * current device. */
int pot3d_gpu_create(const pot3d_mesh_t *mesh, const double *br0, const double *br1,
                     double pm_r1, int ifprec, int precision, int device,
                     pot3d_gpu_solver **out);
int pot3d_gpu_destroy(pot3d_gpu_solver *s);

/* Number of unknowns N. */
long pot3d_gpu_size(const pot3d_gpu_solver *s);

/* Replace br0 (host, (nt,np) column-major) of a set-up solve, as set_flux
 * would for a new boundary map (src/pot3d.F90:3754-3864), keeping the mesh,
 * operator and preconditioner.  No counterpart in the reference, which
 * solves one map per run. */
int pot3d_gpu_set_br0(pot3d_gpu_solver *s, const double *br0);

/* readbr after the file read (src/pot3d.F90:6751-6829) and set_flux's |Br|
 * for 'open' (src/pot3d.F90:3832), on the device: the map fi(ntn,npn)
 * (host, column-major) with its increasing scales tn (theta, ntn) and pn
 * (phi, npn) is interpolated bilinearly onto th(2:ntm1) x ph(2:npm1), copied
 * periodically, given the m=0 pole rows and flux-balanced unless
 * do_not_balance_flux ('ss'/'open'); option 0 'potential', 1 'open', 2 'ss'.
 * The result replaces the solve's br0 (and its RHS, as pot3d_gpu_set_br0);
 * br0_out (host, (nt,np)) receives it when non-NULL.  Bit for bit the host
 * readbr of include/pot3d_host.h.  Returns POT3D_ERR_ARG for scales that do
 * not increase or a mesh point outside them. */
int pot3d_gpu_br0_from_map(pot3d_gpu_solver *s, int ntn, int npn, const double *tn, const double *pn,
                           const double *fi, int option, int do_not_balance_flux, double *br0_out);

/* RHS by potfld's boundary trick, src/pot3d.F90:3937-3950 (host output). */
int pot3d_gpu_rhs(pot3d_gpu_solver *s, double *rhs);

/* cgsolve(x, r, N, ierr), src/pot3d.F90:4231-4369, host pointers.  On entry
 * x is the guess and r the RHS; on exit x is the solution and r the
 * residual.  *ierr = 0 converged, 1 ncgmax exceeded (as the reference).
 * info may be NULL. */
int pot3d_gpu_cgsolve(pot3d_gpu_solver *s, double *x, double *r, long N, int ncgmax,
                      double epscg, int *ierr, pot3d_solve_info_t *info);
/* Same with DEVICE pointers (the Fortran host's use_device_addr arrays). */
int pot3d_gpu_cgsolve_dev(pot3d_gpu_solver *s, double *x, double *r, long N, int ncgmax,
                          double epscg, int *ierr, pot3d_solve_info_t *info);

/* Controls of the FP32-inner / FP64-refined solve (precision
 * POT3D_FP32_REFINED).  A reliable update (r = b - A x in FP64, its
 * preconditioned norm replacing the FP32 recurrence's) is made once the
 * recurrence's r.M^-1 r has fallen by refine_ratio (default 1e-4) since the
 * last one, and whenever the recurrence reports convergence or ncgmax.  An
 * update whose FP64 r.M^-1 r fell by less than the factor stall_drop
 * (default 0.5) is stagnant; stall_limit (default 2) stagnant updates in a
 * row finish the solve with FP64 PCG (same preconditioner) from the current
 * x.  No counterpart in the reference, whose cgsolve is FP64 throughout
 * (src/pot3d.F90:4231-4369). */
int pot3d_gpu_set_refine(pot3d_gpu_solver *s, double refine_ratio, double stall_drop, int stall_limit);
/* Reliable updates of the last refined solve and the FP64 PCG iterations
 * after a switch to FP64 (0: the solve finished in the refined mode). */
int pot3d_gpu_refine_info(const pot3d_gpu_solver *s, int *n_refine, int *fallback_iterations);

/* Residual history of the last solve: epsn after iterations 0..n-1
 * (ernorm's value, src/pot3d.F90:4432-4433).  Returns how many were
 * written (at most cap). */
int pot3d_gpu_history(const pot3d_gpu_solver *s, double *eps, int cap);

/* unpack_scalar + set_boundary_points(phi,1) + seam_hhh, the phi
 * finalisation of potfld (src/pot3d.F90:3966-3969).  x: host, N.
 * phi: host, (nr,nt,np) column-major. */
int pot3d_gpu_finalize_phi(pot3d_gpu_solver *s, const double *x, double *phi);

/* getb + magnetic_energy (src/pot3d.F90:6187-6321) from a host phi with
 * ghosts; w = {W_r, W_t, W_p}. */
int pot3d_gpu_energy(pot3d_gpu_solver *s, const double *phi, double w[3]);

/* The post-solve passes of the reference's main program in one device
 * call: potfld's phi finalisation (src/pot3d.F90:3966-3969), getb
 * (:6187-6233) and magnetic_energy (:6235-6321), from the interior solution
 * x (host, N).  phi (nr,nt,np), br (nrm1,nt,np), bt (nr,ntm1,np),
 * bp (nr,nt,npm1): host, column-major, each written when non-NULL; w gets
 * {W_r, W_t, W_p} when non-NULL.  The B fields go through one transient
 * device buffer, freed before the call returns. */
int pot3d_gpu_fields(pot3d_gpu_solver *s, const double *x, double *phi, double *br, double *bt, double *bp,
                     double w[3]);

/* Kernel-level entry points for parity checks, DEVICE pointers, length N.
 * ax: y = A x as ax (src/pot3d.F90:5102-5150), homogeneous boundaries.
 * prec: x <- M^-1 x as prec_inv (src/pot3d.F90:5152-5225). */
int pot3d_gpu_ax_dev(pot3d_gpu_solver *s, const double *x, double *y);
int pot3d_gpu_prec_dev(pot3d_gpu_solver *s, double *x);
/* The FP32 diagonal preconditioner a_i (src/pot3d.F90:4653-4661) or, for
 * ifprec=2, the FP32 U diagonal of ILU(0) and its inverse a_csr_d
 * (src/pot3d.F90:4706-4708); host outputs of length N (dinv may be NULL). */
int pot3d_gpu_precond_diag(pot3d_gpu_solver *s, float *d, float *dinv);

/* Times the two kernels of one FP64 PCG iteration with CUDA events on the
 * solver's stream: reps iterations from a fresh start (r = b, p = 0), the
 * stencil+dot kernel and the update+dot kernel timed separately.
 * ms[0], ms[1] = average milliseconds per launch; bytes[0], bytes[1] = the
 * algorithmic DRAM bytes per launch (stencil: r, p read, p, Ap written;
 * update: x, p, r, Ap read, x, r written; 8 B each per unknown). */
int pot3d_gpu_time_kernels(pot3d_gpu_solver *s, int reps, double ms[2], double bytes[2]);
/* Average device milliseconds of the ILU(0) forward (ms[0]) and backward
 * (ms[1]) wavefront sweeps over `reps` applications (ifprec = 2 only), in
 * the form the solver iterates with: the plain sweeps for FP64 PCG, the
 * sweeps fused with the inner update's residual half and with rho for the
 * refined mode.  No counterpart in the reference (its timers cover whole
 * preconditioner calls, src/pot3d.F90 timing.out "PC"). */
int pot3d_gpu_time_sweeps(pot3d_gpu_solver *s, int reps, double ms[2]);

/* Failure-detection check of the ILU(0) wavefront sweeps (ifprec = 2): runs
 * the forward sweep with one tile left undone, so the waits of the tiles
 * that consume its faces cannot be satisfied and must give up after
 * spin_limit polls (the library's own limit is 2^22).  Returns
 * POT3D_ERR_TIMEOUT when they did; the device context stays usable and the
 * next solve on the handle proceeds normally.  Nothing faults or hangs.  No
 * counterpart in the reference, whose sweeps are sequential. */
int pot3d_gpu_test_sweep_stall(pot3d_gpu_solver *s, unsigned spin_limit);

/* Magnetic energies like pot3d_gpu_energy, for callers that cannot allocate
 * device memory (their memory is owned by another allocator or pool, or
 * their device footprint is fixed at start-up).  No counterpart in the
 * reference.  All arrays are caller-owned DEVICE arrays, 0-based, with the
 * lengths of pot3d_mesh_t; phi is (nr,nt,np) column-major; w receives
 * {W_r, W_t, W_p} on the device, asynchronously on `stream` (a cudaStream_t,
 * NULL for the default stream).  Scratch is a fixed file-scope device array
 * of 8192 phi planes (3 doubles each): np-2 > 8192 is rejected with
 * POT3D_ERR_ARG.  The library calls no cudaMalloc for it; the first call on
 * a device looks up the array's device address and keeps it, so make it
 * before any stream capture, and do not call again after cudaDeviceReset.
 * Calls share that scratch: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int pot3d_gpu_energy_noalloc(int nr, int nt, int np, const double *rh, const double *dr,
                             const double *drh, const double *dt, const double *dth,
                             const double *sth, const double *dp, const double *dph,
                             const double *phi, double *w, void *stream);

/* Batched solves: n independent cases (own mesh, br0 and pm_r1; FP64 PCG
 * with the diagonal preconditioner, or ILU(0) through
 * pot3d_gpu_batch_create_ex), each tiled kernel launch covering the tiles of every unfinished
 * case, with per-case convergence.  No counterpart in the reference, which
 * solves one case per run.  tk: stencil planes per block (0 = the per-case
 * default; see pot3d_gpu_batch_tune). */
typedef struct pot3d_gpu_batch pot3d_gpu_batch;
int pot3d_gpu_batch_create(int n, const pot3d_mesh_t *meshes, const double *const *br0s,
                           const double *pm_r1s, int tk, pot3d_gpu_batch **out);
/* The same with the preconditioner chosen: ifprec = 1 (diagonal, as above)
 * or 2 (ILU(0) of every case, its two triangular sweeps run for all running
 * cases by one wavefront kernel per direction). */
int pot3d_gpu_batch_create_ex(int n, const pot3d_mesh_t *meshes, const double *const *br0s,
                              const double *pm_r1s, int tk, int ifprec, pot3d_gpu_batch **out);
/* The same with the arithmetic chosen as well: precision POT3D_FP32_REFINED
 * runs every case's inner iterations in FP32 storage (the batched forms of
 * the single solve's refined kernels) with per-case FP64 reliable updates,
 * per-case stagnation switches to FP64 PCG and per-case convergence on the
 * FP64 residual, as pot3d_gpu_set_refine describes for one case. */
int pot3d_gpu_batch_create_mode(int n, const pot3d_mesh_t *meshes, const double *const *br0s,
                                const double *pm_r1s, int tk, int ifprec, int precision,
                                pot3d_gpu_batch **out);
/* Initial guess of case i for the following pot3d_gpu_batch_solve calls
 * (host, packed layout of length N_i, copied; NULL returns to x = 0), as
 * potfld's x_cg = 0 (src/pot3d.F90:3924) replaced by, e.g., a learned
 * prediction.  PCG from the guess decides convergence as from zero. */
int pot3d_gpu_batch_set_guess(pot3d_gpu_batch *b, int i, const double *x);
/* Autotuner: times `iters` batched iterations for each candidate planes per
 * block, keeps the fastest (*best_tk; ms_out[c] = time of candidate c). */
int pot3d_gpu_batch_tune(pot3d_gpu_batch *b, const int *candidates, int ncand, int iters, int *best_tk,
                         float *ms_out);
/* Autotuner over two tile parameters: the stencil's planes per block
 * (cand_tk, 8..512) and the update kernels' planes per block (cand_tku, >=
 * 8); times every pair, keeps the fastest; ms_out[c * n_tku + d] = time of
 * (cand_tk[c], cand_tku[d]). */
int pot3d_gpu_batch_tune2(pot3d_gpu_batch *b, const int *cand_tk, int n_tk, const int *cand_tku, int n_tku,
                          int iters, int *best_tk, int *best_tku, float *ms_out);
/* Solve all cases from their guesses (x = 0 unless set) to epscg (ernorm's
 * rule per case; with FP32_REFINED, info[i].n_refine the case's reliable
 * updates); ierr[i],
 * info[i] per case; *seconds = device time of the whole batch. */
int pot3d_gpu_batch_solve(pot3d_gpu_batch *b, int ncgmax, double epscg, int *ierr,
                          pot3d_solve_info_t *info, double *seconds);
/* Solution of case i (host, packed layout of length N_i). */
int pot3d_gpu_batch_solution(pot3d_gpu_batch *b, int i, double *x);
int pot3d_gpu_batch_destroy(pot3d_gpu_batch *b);

/* Message for the most recent failing call on this thread. */
const char *pot3d_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* POT3D_GPU_H */
