// ILU(0) preconditioner (ifprec = 2) of the whole-solve path.
//
// For POT3D's 7-point pattern with np >= 6 the row-wise ILU(0) of ilu0
// (src/pot3d.F90:4717-4813) changes only the diagonal: with the boundary
// couplings dropped as diacsr does (src/pot3d.F90:4940-4967),
//   d_i = a_ii - sum_{k in L(i), ascending column} (a_ik / d_k) * a_ki ,
// the stored L entries are a_ik/d_k and the U entries are the unchanged
// a_ij, all in FP32.  lusol (src/pot3d.F90:5227-5302) then solves
//   y_i = r_i - sum_{k in L(i)} l_ik y_k          (rows ascending)
//   z_i = (y_i - sum_{j in U(i)} a_ij z_j) * dinv_i  (rows descending)
// with dinv_i = real(1/d_i in FP64, REAL32) (src/pot3d.F90:4706-4708).
//
// Nothing is stored but d and dinv: the FP32 couplings are the FP64
// coefficients of load_matrix_pot3d_solve, formed on the fly in the
// reference's operand order and rounded to FP32 as diacsr rounds them.
// Every FP32 operation is an explicit __fdiv_rn/__fmul_rn/__fsub_rn so the
// factor and both sweeps are bit-identical to the oracle.
//
// Rows depend on their lower neighbours i-1, j-1, k-1 and, on the last phi
// plane, on the first plane through the periodic seam; all of them lie on
// earlier hyperplanes e+jj+kk, so one kernel per hyperplane (level) runs
// each recurrence.  Column order inside a row, as diacsr builds it:
//   lower: [seam from plane 1 (last plane only)], k-1, j-1, i-1
//   upper: i+1, j+1, k+1, [seam to the last plane (first plane only)]
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "pot3d_internal.cuh"
#include "pot3d_solver.h"

namespace pot3d {

// FP64 coefficients of one row in the reference's operand order.
struct Row7 {
  double a1, a2, a3, a4, a5, a6, a7;
};
__device__ __forceinline__ Row7 row7(const DevMesh &m, int i, int j, int k) {
  Row7 a;
  const double drh = m.drh[i];
  const double c17 = __dmul_rn(__dmul_rn(drh, m.dth[j]), m.sth_i[j]);
  a.a1 = -__dmul_rn(c17, m.dp_i[k - 1]);
  a.a7 = -__dmul_rn(c17, m.dp_i[k]);
  const double u = __dmul_rn(drh, m.dph[k]);
  a.a2 = -__dmul_rn(__dmul_rn(u, m.st[j - 1]), m.dt_i[j - 1]);
  a.a6 = -__dmul_rn(__dmul_rn(u, m.st[j]), m.dt_i[j]);
  const double v = __dmul_rn(__dmul_rn(m.sth[j], m.dth[j]), m.dph[k]);
  a.a3 = -__dmul_rn(__dmul_rn(v, m.r2[i - 1]), m.dr_i[i - 1]);
  a.a5 = -__dmul_rn(__dmul_rn(v, m.r2[i]), m.dr_i[i]);
  a.a4 = -__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(a.a1, a.a2), a.a3), a.a5), a.a6), a.a7);
  return a;
}

struct LevelArgs {
  Geo g;
  DevMesh m;
  int level;
  int kk_lo;
  float *d, *dinv;          // factor (padded layout)
  const float *r32;         // sweep input
  float *y32;               // forward result
  float *z32;               // backward result
  const SolveState *st;     // optional early exit
  int *pivot;               // first zero pivot (packed row index + 1), 0 if none
};

// Point of level l handled by this thread; false if out of range.
__device__ __forceinline__ bool level_point(const LevelArgs &a, int *e, int *jj, int *kk) {
  const Geo &g = a.g;
  *kk = a.kk_lo + blockIdx.y;
  const int rest = a.level - *kk;  // e + jj
  const int jlo = max(0, rest - (g.nrm2 - 1));
  *jj = jlo + blockIdx.x * blockDim.x + threadIdx.x;
  if (*jj >= g.ntm2 || *jj > rest) return false;
  *e = rest - *jj;
  return *e >= 0 && *e < g.nrm2 && *kk < g.npm2;
}

__global__ void k_dilu_factor(LevelArgs a) {
  int e, jj, kk;
  if (!level_point(a, &e, &jj, &kk)) return;
  const Geo &g = a.g;
  const Row7 c = row7(a.m, e + 2, jj + 2, kk + 2);
  float d = (float)c.a4;
  if (kk == g.npm2 - 1) {  // seam: a7 couples to plane 1, the smallest column
    const float aik = (float)c.a7;
    const float l = __fdiv_rn(aik, a.d[g.idx(e, jj, 0)]);
    d = __fsub_rn(d, __fmul_rn(l, aik));
  }
  if (kk > 0) {
    const float aik = (float)c.a1;
    const float l = __fdiv_rn(aik, a.d[g.idx(e, jj, kk - 1)]);
    d = __fsub_rn(d, __fmul_rn(l, aik));
  }
  if (jj > 0) {
    const float aik = (float)c.a2;
    const float l = __fdiv_rn(aik, a.d[g.idx(e, jj - 1, kk)]);
    d = __fsub_rn(d, __fmul_rn(l, aik));
  }
  if (e > 0) {
    const float aik = (float)c.a3;
    const float l = __fdiv_rn(aik, a.d[g.idx(e - 1, jj, kk)]);
    d = __fsub_rn(d, __fmul_rn(l, aik));
  }
  const long long id = g.idx(e, jj, kk);
  a.d[id] = d;
  a.dinv[id] = __double2float_rn(__ddiv_rn(1.0, (double)d));
  if (d == 0.0f) {
    const long long packed = ((long long)kk * g.ntm2 + jj) * g.nrm2 + e + 1;
    atomicMin(a.pivot, (int)min(packed, (long long)0x7fffffff));
  }
}

__global__ void k_dilu_forward(LevelArgs a) {
  if (a.st && a.st->status != ST_RUNNING) return;
  int e, jj, kk;
  if (!level_point(a, &e, &jj, &kk)) return;
  const Geo &g = a.g;
  const Row7 c = row7(a.m, e + 2, jj + 2, kk + 2);
  const long long id = g.idx(e, jj, kk);
  float y = a.r32[id];
  if (kk == g.npm2 - 1) {
    const long long k = g.idx(e, jj, 0);
    y = __fsub_rn(y, __fmul_rn(__fdiv_rn((float)c.a7, a.d[k]), a.y32[k]));
  }
  if (kk > 0) {
    const long long k = g.idx(e, jj, kk - 1);
    y = __fsub_rn(y, __fmul_rn(__fdiv_rn((float)c.a1, a.d[k]), a.y32[k]));
  }
  if (jj > 0) {
    const long long k = g.idx(e, jj - 1, kk);
    y = __fsub_rn(y, __fmul_rn(__fdiv_rn((float)c.a2, a.d[k]), a.y32[k]));
  }
  if (e > 0) {
    const long long k = g.idx(e - 1, jj, kk);
    y = __fsub_rn(y, __fmul_rn(__fdiv_rn((float)c.a3, a.d[k]), a.y32[k]));
  }
  a.y32[id] = y;
}

__global__ void k_dilu_backward(LevelArgs a) {
  if (a.st && a.st->status != ST_RUNNING) return;
  int e, jj, kk;
  if (!level_point(a, &e, &jj, &kk)) return;
  const Geo &g = a.g;
  const Row7 c = row7(a.m, e + 2, jj + 2, kk + 2);
  const long long id = g.idx(e, jj, kk);
  float z = a.y32[id];
  if (e < g.nrm2 - 1) z = __fsub_rn(z, __fmul_rn((float)c.a5, a.z32[g.idx(e + 1, jj, kk)]));
  if (jj < g.ntm2 - 1) z = __fsub_rn(z, __fmul_rn((float)c.a6, a.z32[g.idx(e, jj + 1, kk)]));
  if (kk < g.npm2 - 1) z = __fsub_rn(z, __fmul_rn((float)c.a7, a.z32[g.idx(e, jj, kk + 1)]));
  if (kk == 0) z = __fsub_rn(z, __fmul_rn((float)c.a1, a.z32[g.idx(e, jj, g.npm2 - 1)]));
  a.z32[id] = __fmul_rn(z, a.dinv[id]);
}

struct DiluState {
  float *d = nullptr, *dinv = nullptr, *r32 = nullptr, *y32 = nullptr, *z32 = nullptr;
  int *pivot = nullptr;
  int nlev = 0;
  std::vector<int> kk_lo, nkk, nblk;  // per level launch shape
};

static void level_shape(const Geo &g, int l, int *kk_lo, int *nkk, int *nblk) {
  const int lo = std::max(0, l - (g.nrm2 - 1) - (g.ntm2 - 1));
  const int hi = std::min(g.npm2 - 1, l);
  *kk_lo = lo;
  *nkk = hi - lo + 1;
  const int span = std::min(g.nrm2, g.ntm2);  // valid jj per kk
  *nblk = (span + 127) / 128;
}

static void launch_level(Solver *s, int which, int l, bool check) {
  DiluState *D = s->dilu;
  LevelArgs a{};
  a.g = s->g;
  a.m = s->m;
  a.level = l;
  a.kk_lo = D->kk_lo[l];
  a.d = D->d;
  a.dinv = D->dinv;
  a.r32 = D->r32;
  a.y32 = D->y32;
  a.z32 = D->z32;
  a.st = check ? s->d_state : nullptr;
  a.pivot = D->pivot;
  dim3 grid(D->nblk[l], D->nkk[l]);
  if (which == 0)
    k_dilu_factor<<<grid, 128, 0, s->stream>>>(a);
  else if (which == 1)
    k_dilu_forward<<<grid, 128, 0, s->stream>>>(a);
  else
    k_dilu_backward<<<grid, 128, 0, s->stream>>>(a);
}

int dilu_setup(Solver *s) {
  const Geo &g = s->g;
  if (g.nrm2 < 3 || g.ntm2 < 3 || g.npm2 < 4) {
    pot3d_set_error("ifprec=2 needs nr>=5, nt>=5, np>=6 (ILU(0) without fill)");
    return POT3D_ERR_ARG;
  }
  s->dilu = new DiluState();
  DiluState *D = s->dilu;
  int st;
  const size_t fb = sizeof(float) * (size_t)g.Np;
  if ((st = s->alloc((void **)&D->d, fb)) || (st = s->alloc((void **)&D->dinv, fb)) ||
      (st = s->alloc((void **)&D->r32, fb)) || (st = s->alloc((void **)&D->y32, fb)) ||
      (st = s->alloc((void **)&D->z32, fb)) || (st = s->alloc((void **)&D->pivot, sizeof(int))))
    return st;
  D->nlev = g.nrm2 + g.ntm2 + g.npm2 - 2;
  D->kk_lo.resize(D->nlev);
  D->nkk.resize(D->nlev);
  D->nblk.resize(D->nlev);
  for (int l = 0; l < D->nlev; l++) level_shape(g, l, &D->kk_lo[l], &D->nkk[l], &D->nblk[l]);
  const int big = 0x7fffffff;
  if ((st = pot3d_cuda_status(cudaMemcpyAsync(D->pivot, &big, sizeof(int), cudaMemcpyHostToDevice, s->stream),
                              "cudaMemcpy(pivot)")))
    return st;
  for (int l = 0; l < D->nlev; l++) launch_level(s, 0, l, false);
  if ((st = pot3d_cuda_status(cudaGetLastError(), "k_dilu_factor"))) return st;
  int piv = big;
  if ((st = pot3d_cuda_status(cudaMemcpyAsync(&piv, D->pivot, sizeof(int), cudaMemcpyDeviceToHost, s->stream),
                              "cudaMemcpy(pivot)")))
    return st;
  if ((st = pot3d_cuda_status(cudaStreamSynchronize(s->stream), "ILU(0) factorisation"))) return st;
  if (piv != big) {
    pot3d_set_error("zero pivot in the ILU(0) factorisation at row " + std::to_string(piv));
    return POT3D_ERR_PIVOT;
  }
  return POT3D_OK;
}

void dilu_destroy(Solver *s) {
  delete s->dilu;
  s->dilu = nullptr;
}

float *dilu_r32(Solver *s) { return s->dilu->r32; }
float *dilu_z32(Solver *s) { return s->dilu->z32; }
int dilu_sweep_launches(Solver *s) { return s->dilu ? 2 * s->dilu->nlev : 0; }

int dilu_sweeps(Solver *s, bool check_status) {
  DiluState *D = s->dilu;
  for (int l = 0; l < D->nlev; l++) launch_level(s, 1, l, check_status);
  for (int l = D->nlev - 1; l >= 0; l--) launch_level(s, 2, l, check_status);
  return pot3d_cuda_status(cudaGetLastError(), "ILU(0) sweeps");
}

__global__ static void k_unpack_f32(Geo g, const float *__restrict__ src, float *__restrict__ dst) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.N;
       t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t % g.nrm2);
    const long long line = t / g.nrm2;
    dst[t] = src[line * g.NRP + e];
  }
}

int dilu_diag(Solver *s, float *d_host, float *dinv_host) {
  DiluState *D = s->dilu;
  const Geo &g = s->g;
  int st;
  for (int w = 0; w < 2; w++) {
    float *h = w == 0 ? d_host : dinv_host;
    if (!h) continue;
    k_unpack_f32<<<grid1d(g.N), NTHR, 0, s->stream>>>(g, w == 0 ? D->d : D->dinv, D->y32);
    if ((st = pot3d_cuda_status(cudaMemcpyAsync(h, D->y32, sizeof(float) * g.N, cudaMemcpyDeviceToHost, s->stream),
                                "cudaMemcpy(diag)")))
      return st;
  }
  return pot3d_cuda_status(cudaStreamSynchronize(s->stream), "dilu_diag");
}

}  // namespace pot3d
