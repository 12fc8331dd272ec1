// Internal definitions shared by the pot3d_gpu CUDA sources.
//
// Data layout in HBM: every CG vector lives in a padded interior layout
//   idx = (kk * ntm2 + jj) * NRP + e
// with e = i-2, jj = j-2, kk = k-2 the interior offsets of Fortran (i,j,k)
// and NRP = nrm2 rounded up to a multiple of 16 doubles (128 B), so every
// radial line starts on a 128-byte boundary and the double2/float2 loads of
// the kernels are aligned.  Pad lanes hold zeros and are never written with
// anything else.  The reference's packed layout (src/pot3d.F90:4930) is the
// same with NRP = nrm2; pack/unpack kernels convert at the API boundary.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/pot3d_gpu.h"

namespace pot3d {

constexpr int TI = 64;      // radial points per tile (32 lanes x 2)
constexpr int TJ = 8;       // theta rows per tile (one warp each)
constexpr int NTHR = 256;   // threads per tile block
constexpr int X_GROUP = 8;  // refined ILU(0) single solve: iterations per solution update
constexpr int SROW = TI + 4;  // shared-memory row: [pad, halo-, 64 own, halo+, pad]

// Mesh arrays on the device, 1-based Fortran indexing: arr[k] is Fortran
// element k (one spare slot at 0 and at the end).
struct DevMesh {
  const double *drh, *dth, *sth_i, *dp_i, *dph, *st, *dt_i, *sth, *r2, *dr_i;
  const double *dr, *rh, *dt, *dp;
  const double *th, *ph;    // half-mesh coordinates (readbr's interpolation points)
  const double *br0, *br1;  // (nt,np) column-major, 0-based
  double dr1, drn, pm_r1, pl_i;
};

struct Geo {
  int nr, nt, np;
  int nrm2, ntm2, npm2;
  int NRP;      // padded radial line length
  int tk;       // k-planes per block of the stencil kernel
  int nkc;      // number of k chunks of the stencil kernel (gridDim.z)
  int tk_u;     // k-planes per block of the update kernels
  int nkc_u;    // number of k chunks of the update kernels
  int nit;      // number of i tiles (gridDim.x)
  int njt;      // number of j tiles (gridDim.y)
  long long Np; // padded vector length
  long long N;  // packed vector length
  __host__ __device__ long long idx(int e, int jj, int kk) const {
    return ((long long)kk * ntm2 + jj) * NRP + e;
  }
};

// Scalars of one PCG solve, resident on the device so the iteration never
// waits on the host.
struct SolveState {
  double rho, rho_old, alpha, beta, bdotb, epsn, pq, epscg;
  double rho_true;  // refined mode: preconditioned FP64 residual norm^2
  double xa[X_GROUP];  // refined ILU(0): alphas of the x updates applied in groups (0: none)
  int ncg, ncgmax, status, par;
  unsigned int cnt_a, cnt_b, cnt_c, pad0;
  int hist_cap, n_refine, inner, pad1;
  double *hist;
};

enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXIT = 2, ST_BREAKDOWN = 3, ST_TIMEOUT = 4 };

// ---- deterministic block reduction --------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block in a fixed order; result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NT / 32; q++) s += sh[q];
  }
  return s;
}

// Kinds of the r.z reductions of a PCG solve.  UPD_ITER: the update of an
// iteration with the diagonal preconditioner; UPD_INIT: the initial
// residual; UPD_BDOTB: b.M^-1 b; UPD_ZDOT: r.z after the ILU(0) sweeps;
// UPD_RU: r.z of a fresh FP64 residual (reliable update of the refined mode).
enum { UPD_ITER = 0, UPD_INIT = 1, UPD_BDOTB = 2, UPD_ZDOT = 3, UPD_RU = 4 };

// What follows a new r.z = total (one thread, KIND != UPD_BDOTB): rho and
// beta (src/pot3d.F90:4352-4356), ncg and ernorm's epsn and stopping rule
// (src/pot3d.F90:4430-4483).  UPD_RU replaces the recurrence's rho and
// decides the status on this residual whatever the recurrence said; a
// reliable update that finds the recurrence far off (its r.z more than 10x
// the recurrence's) restarts the direction (beta = 0: p = z).
template <int KIND>
__device__ __forceinline__ void rz_epilogue(SolveState *s, double total) {
  const double rho_it = s->rho;  // UPD_RU: the recurrence's value it replaces
  if (KIND != UPD_RU) s->rho_old = s->rho;
  s->rho = total;
  if (KIND == UPD_ITER || KIND == UPD_ZDOT) s->ncg = s->ncg + 1;
  const double epssq = total / s->bdotb;
  const double epsn = (epssq >= 0.0 ? 1.0 : -1.0) * sqrt(fabs(epssq));
  s->epsn = epsn;
  if (s->hist && s->ncg < s->hist_cap) s->hist[s->ncg] = epsn;
  if (KIND == UPD_RU) s->status = ST_RUNNING;
  if (epsn < s->epscg) {
    s->status = ST_CONVERGED;
  } else if (s->ncg >= s->ncgmax) {
    s->status = ST_MAXIT;
  } else if (!isfinite(epsn)) {
    s->status = ST_BREAKDOWN;
  }
  if (KIND == UPD_RU) s->rho_true = total;
  const bool restart = KIND == UPD_RU && (!(s->rho_old > 0.0) || total > 10.0 * rho_it);
  s->beta = (KIND == UPD_INIT || restart) ? 0.0 : total / s->rho_old;
}

// Last-block pattern: every block stores its partial at slot b, the block
// that arrives last sums all partials in index order (deterministic for a
// fixed grid) and returns true in all its threads with the total in *total.
template <int NT>
__device__ bool last_block_sum_at(double part, double *partials, unsigned int *counter, unsigned int nblocks,
                                  unsigned int b, double *total, double *sh) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    partials[b] = part;
    __threadfence();
    unsigned int prev = atomicAdd(counter, 1u);
    is_last = (prev == nblocks - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double s = 0.0;
  for (unsigned int q = threadIdx.x; q < nblocks; q += NT) s += __ldcg(partials + q);
  s = block_sum<NT>(s, sh);
  if (threadIdx.x == 0) {
    *total = s;
    *counter = 0u;
  }
  return true;
}
template <int NT>
__device__ bool last_block_sum(double part, double *partials, unsigned int *counter, unsigned int nblocks,
                               double *total, double *sh) {
  const unsigned int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  return last_block_sum_at<NT>(part, partials, counter, nblocks, b, total, sh);
}

}  // namespace pot3d

// Error reporting shared by the C-ABI entry points.
void pot3d_set_error(const std::string &msg);

// Return the library status of a failing CUDA runtime call.
#define CK(call)                                                  \
  do {                                                            \
    int _st = pot3d_cuda_status((call), #call);                   \
    if (_st != POT3D_OK) return _st;                              \
  } while (0)

int pot3d_cuda_status(cudaError_t e, const char *where);
