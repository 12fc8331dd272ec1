// Host-side solver object behind the pot3d_gpu_* C-ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <utility>
#include <vector>

#include "pot3d_internal.cuh"

namespace pot3d {

struct DiluState;   // ILU(0) preconditioner (dilu.cu)

struct Solver {
  Geo g{};
  DevMesh m{};
  int ifprec = 1, precision = 0;
  double pm_r1 = -1.0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<void *> allocs;

  SolveState *d_state = nullptr;
  SolveState *h_state = nullptr;
  double *d_partials = nullptr;
  size_t nblk_tiled = 0;
  int tk_default = 0, nkc_default = 0;  // stencil k-chunking chosen at setup
  int tku_default = 0, nkcu_default = 0;  // the update kernels' k-chunking
  double *d_s1z = nullptr, *d_s1p = nullptr, *d_s1 = nullptr;
  double *d_scalar = nullptr, *d_sums = nullptr, *d_hist = nullptr;
  int hist_cap = 0;
  // padded FP64 vectors
  double *d_x = nullptr, *d_r = nullptr, *d_p = nullptr, *d_p2 = nullptr, *d_q = nullptr, *d_b = nullptr;
  double *d_tmp = nullptr;      // scratch (API packing, residual)
  double *d_ref = nullptr;      // scratch in the reference packed layout (N)
  double *d_phi = nullptr;      // (nr,nt,np) scratch for finalize/energy
  float *d_ai = nullptr;        // diagonal preconditioner (FP32, padded)
  double *p_cur = nullptr, *p_nxt = nullptr;

  // FP32-inner / FP64-refined mode (both preconditioners)
  float *m_p32a = nullptr, *m_p32b = nullptr, *m_r32 = nullptr, *m_q32 = nullptr;
  // ILU(0): four directions in rotation (a, b and two more), so the solution
  // update is applied once per four iterations
  float *m_p32q[X_GROUP] = {};  // refined ILU(0): the directions of X_GROUP consecutive iterations
  float *p32_cur = nullptr, *p32_nxt = nullptr;
  cudaGraphExec_t graph32_exec = nullptr;
  int graph32_U = 0;
  int xblocks = 0;  // grid of the refined ILU(0) iterations' grouped solution update
  cudaEvent_t evm0 = nullptr, evm1 = nullptr;
  double refine_ratio = 1e-4;  // reliable update once the recurrence's r.z fell by this factor
  double stall_drop = 0.5;     // an update whose FP64 r.z fell by less than this factor is stagnant
  int stall_limit = 2;         // consecutive stagnant updates that switch the solve to FP64 PCG
  int last_fallback_iters = 0; // FP64 iterations after a switch in the last solve (0: none)
  float *r32_inner();          // the FP32 recurrence residual (the sweeps' input with ILU(0))
  int launch_iteration32(int u);  // u: position in the captured graph (pairs of iterations)
  int reliable_update();
  int mixed_solve(bool zero_guess, int ncgmax, double epscg, int *ierr, pot3d_solve_info_t *info);

  cudaGraphExec_t graph_exec = nullptr;
  int graph_U = 0, graph_kind = -1;

  long long launches = 0;  // kernel launches of the last solve
  int last_ncg = 0, last_refine = 0;
  double last_epsn = 0.0, last_seconds = 0.0;

  // TMA descriptors of padded vectors, keyed by (address, is_fp64).
  std::map<std::pair<const void *, int>, CUtensorMap> tmaps;
  int tensor_map(const void *ptr, bool fp64, CUtensorMap *out);

  DiluState *dilu = nullptr;

  ~Solver();
  int alloc(void **p, size_t bytes);
  int setup(const pot3d_mesh_t *mesh, const double *br0, const double *br1, double pm_r1, int ifprec,
            int precision);
  int pack(const double *ref_dev, double *pad_dev);
  int unpack(const double *pad_dev, double *ref_dev);
  int ax_padded(const double *x, double *y);
  int prec_padded(double *x);  // x <- M^-1 x
  int rhs_padded(double *b);
  int dot_padded(const double *x, const double *y, double *out_dev);
  int launch_iteration();
  // FP64 PCG on d_x (guess) / d_b (RHS).  d_r holds the residual on exit.
  int cgsolve_padded(bool zero_guess, int ncgmax, double epscg, int *ierr, pot3d_solve_info_t *info);
  int true_residual(double *out);  // ||b - A x|| / ||b|| of d_x, d_b
  int finalize_phi_dev(const double *xpad, double *phi_dev);
  int time_kernels(int reps, double ms[2], double bytes[2]);
  int sweep_launches() const;  // kernels per ILU(0) application
  // getb (src/pot3d.F90:6187-6233) from a device phi into device B fields.
  int getb_dev(const double *phi_dev, double *br, double *bt, double *bp);
  int energy_dev(const double *phi_dev, double w[3]);
};

// ILU(0) preconditioner hooks (dilu.cu).
int dilu_setup(Solver *s);
void dilu_destroy(Solver *s);
float *dilu_r32(Solver *s);   // FP32 input of the sweeps (padded layout)
float *dilu_z32(Solver *s);   // FP32 output z = (LU)^-1 r32
// Forward + backward sweeps r32 -> z32 on s->stream; with check_status the
// kernels return at once when the PCG state is no longer running.
int dilu_sweeps(Solver *s, bool check_status);
// The refined mode's inner iteration: the sweeps fused with the residual
// half of the update (forward, on the residual stream) and with rho, beta,
// ncg and ernorm (backward); q32 = A p of the iteration.
int dilu_sweeps_fused(Solver *s, const float *q32);
// Refresh the fused sweeps' residual stream from r32 (after r32 was formed
// from an FP64 residual).
int dilu_r_stream(Solver *s);
int encode_padded_map(const Geo &g, const void *ptr, bool fp64, int bx, int by, int bz, CUtensorMap *out,
                      bool interior_only = false);
int dilu_reset(Solver *s);
int dilu_status(Solver *s);  // POT3D_ERR_TIMEOUT if a sweep gave up waiting
int dilu_test_stall(Solver *s, unsigned spin_limit);  // a sweep whose waits must run out
// Sweeps for a factored 1-based CSR with the 7-point pattern of s->g's grid.
int dilu_setup_csr(Solver *s, const int *ia, const int *ja, const int *dptr, const float *a, const float *dinv);
int dilu_time(Solver *s, int reps, double ms[2]);
int dilu_diag(Solver *s, float *d_host, float *dinv_host);
int dilu_sweep_launches(Solver *s);
// Batched sweeps over many cases (dilu.cu): one kernel per direction covers
// the tiles of every running case.
struct DiluBatch;
int dilu_batch_setup(Solver *const *cases, int n, cudaStream_t stream, DiluBatch **out);
int dilu_batch_sweeps(DiluBatch *b, cudaStream_t stream);
int dilu_batch_sweeps_fused(DiluBatch *b, cudaStream_t stream);  // refined mode (dilu_sweeps_fused per case)
bool dilu_batch_fused(const DiluBatch *b);
int dilu_batch_reset(DiluBatch *b, cudaStream_t stream);
void dilu_batch_destroy(DiluBatch *b);


// Kernel launch helpers shared between translation units.
int grid1d(long long n);

}  // namespace pot3d
