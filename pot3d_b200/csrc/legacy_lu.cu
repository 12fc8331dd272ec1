// The three symbols of POT3D's external LU solver (src/lusol_cusparse.c),
// reimplemented on our own kernels: ILU(0) of a general 1-based CSR matrix
// and its forward/backward sweeps, level-scheduled on the GPU.
//
//   load_external_lu_solver   src/lusol_cusparse.c:64-302
//   external_lu_solver        src/lusol_cusparse.c:309-367
//   unload_external_lu_solver src/lusol_cusparse.c:374-391
//
// Semantics follow the shim: device pointers from the Fortran host, one
// global instance, the CSR values factorised in place into L\U (unit lower
// L), x <- (double)(U^-1 L^-1 (float)x) per call, and "ERROR! ..." plus
// exit(1) on any failure.  The arithmetic follows the reference's CPU
// routines ilu0 (src/pot3d.F90:4717-4813) and lusol (src/pot3d.F90:5227-5302)
// operation for operation in FP32 (no fused multiply-adds), with the
// upper-triangular solve multiplying by dinv = real(1/d in FP64, REAL32)
// (src/pot3d.F90:4706-4708).
//
// The sparsity analysis (row levels of L and of U) runs once on the host
// from the integer structure and the factorisation is one kernel per level.
// When the matrix has the 7-point pattern diacsr builds for a
// nrm2 x ntm2 x npm2 interior (src/pot3d.F90:4870-5018: boundary couplings
// dropped, the periodic phi seam kept) -- recognised from the columns alone --
// each call runs the two wavefront sweeps of the whole-solve path, their
// coefficient streams formed from the factored CSR; any other pattern runs
// level-scheduled sweeps (one kernel per level) replayed as a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "pot3d_internal.cuh"
#include "pot3d_solver.h"

namespace {

struct LegacyLU {
  int N = 0, nnz = 0;
  float *val = nullptr;       // caller's CSR values (factorised in place)
  const int *ia = nullptr;    // caller's 1-based row pointers
  const int *ja = nullptr;    // caller's 1-based columns
  int *dptr = nullptr;        // 0-based position of each diagonal
  float *dinv = nullptr;
  float *x32 = nullptr;
  int *rows_f = nullptr, *rows_b = nullptr;  // rows ordered by level
  std::vector<int> lev_f, lev_b;             // level offsets into rows_*
  cudaStream_t stream = nullptr;
  cudaGraphExec_t sweeps = nullptr;   // level-scheduled route
  pot3d::Solver *wave = nullptr;      // wavefront route (7-point pattern): grid, stream, sweeps
  bool loaded = false;
};
LegacyLU g_lu;

// The grid of a CSR with diacsr's 7-point pattern, or false.  Row 0 gives
// the column offsets nrm2 (j+1) and nrm2*ntm2 (k+1); every row must then hold
// exactly the columns diacsr writes for its (e, j, k), in ascending order.
bool seven_point(int N, const std::vector<int> &ia, const std::vector<int> &ja, int *nrm2_, int *ntm2_,
                 int *npm2_) {
  if (N < 36 || ia[1] - ia[0] != 5) return false;
  const int c1 = ja[ia[0]], cj = ja[ia[0] + 1] - 1, ck = ja[ia[0] + 2] - 1;
  if (ja[ia[0] - 1] != 1 || c1 != 2 || cj < 3 || ck <= cj || ck % cj != 0 || N % ck != 0) return false;
  const long long nrm2 = cj, P = ck, ntm2 = P / nrm2, npm2 = N / P;
  if (nrm2 < 3 || ntm2 < 3 || npm2 < 4) return false;
  const long long W = (npm2 - 1) * P;
  std::vector<long long> want;
  for (long long i = 0; i < N; i++) {
    const long long e = i % nrm2, j = (i / nrm2) % ntm2, k = i / P;
    want.clear();
    if (k == npm2 - 1) want.push_back(i - W);
    if (k > 0) want.push_back(i - P);
    if (j > 0) want.push_back(i - nrm2);
    if (e > 0) want.push_back(i - 1);
    want.push_back(i);
    if (e < nrm2 - 1) want.push_back(i + 1);
    if (j < ntm2 - 1) want.push_back(i + nrm2);
    if (k < npm2 - 1) want.push_back(i + P);
    if (k == 0) want.push_back(i + W);
    if (ia[i + 1] - ia[i] != (int)want.size()) return false;
    for (size_t q = 0; q < want.size(); q++)
      if (ja[ia[i] - 1 + q] - 1 != want[q]) return false;
  }
  *nrm2_ = (int)nrm2;
  *ntm2_ = (int)ntm2;
  *npm2_ = (int)npm2;
  return true;
}

// Packed FP64 vector -> padded FP32 sweep input, and back.
__global__ void k_lu_narrow_pad(pot3d::Geo g, const double *__restrict__ x, float *__restrict__ r32) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.N;
       t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t % g.nrm2);
    const long long line = t / g.nrm2;
    r32[line * g.NRP + e] = (float)x[t];
  }
}
__global__ void k_lu_widen_pad(pot3d::Geo g, const float *__restrict__ z32, double *__restrict__ x) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.N;
       t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t % g.nrm2);
    const long long line = t / g.nrm2;
    x[t] = (double)z32[line * g.NRP + e];
  }
}

[[noreturn]] void die(const char *what, const char *detail) {
  printf(" ERROR! %s %s \n", what, detail ? detail : "");
  fflush(stdout);
  exit(1);
}
void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(what, cudaGetErrorString(e));
}

// ilu0's row step for one row: L entries divided by the pivots of earlier
// rows, then the updates of the row's entries whose column appears in the
// earlier row's upper part.
__global__ void k_lu_factor(const int *__restrict__ rows, int n, const int *__restrict__ ia,
                            const int *__restrict__ ja, const int *__restrict__ dptr, float *__restrict__ a,
                            int *__restrict__ pivot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = rows[t];  // 0-based row
  const int lo = ia[i] - 1, hi = ia[i + 1] - 1, di = dptr[i];
  for (int ik = lo; ik < di; ik++) {
    const int k = ja[ik] - 1;
    const float aik = __fdiv_rn(a[ik], a[dptr[k]]);
    a[ik] = aik;
    for (int kj = dptr[k] + 1; kj < ia[k + 1] - 1; kj++) {
      const int col = ja[kj];
      for (int ij = lo; ij < hi; ij++)
        if (ja[ij] == col) {
          a[ij] = __fsub_rn(a[ij], __fmul_rn(aik, a[kj]));
          break;
        }
    }
  }
  if (a[di] == 0.0f) atomicMin(pivot, i + 1);
}

__global__ void k_lu_dinv(int n, const int *__restrict__ dptr, const float *__restrict__ a, float *__restrict__ dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dinv[i] = __double2float_rn(__ddiv_rn(1.0, (double)a[dptr[i]]));
}

__global__ void k_lu_forward(const int *__restrict__ rows, int n, const int *__restrict__ ia, const int *__restrict__ ja,
                             const int *__restrict__ dptr, const float *__restrict__ a, float *__restrict__ x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = rows[t];
  float v = x[i];
  for (int k = ia[i] - 1; k < dptr[i]; k++) v = __fsub_rn(v, __fmul_rn(a[k], x[ja[k] - 1]));
  x[i] = v;
}

__global__ void k_lu_backward(const int *__restrict__ rows, int n, const int *__restrict__ ia,
                              const int *__restrict__ ja, const int *__restrict__ dptr, const float *__restrict__ a,
                              const float *__restrict__ dinv, float *__restrict__ x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = rows[t];
  float v = x[i];
  for (int k = dptr[i] + 1; k < ia[i + 1] - 1; k++) v = __fsub_rn(v, __fmul_rn(a[k], x[ja[k] - 1]));
  x[i] = __fmul_rn(v, dinv[i]);
}

__global__ void k_lu_narrow(int n, const double *__restrict__ x, float *__restrict__ x32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x32[i] = (float)x[i];
}
__global__ void k_lu_widen(int n, const float *__restrict__ x32, double *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = (double)x32[i];
}

// Rows grouped by dependency level: lev[i] = 1 + max lev over the rows this
// row reads (lower part for L, upper part for U).
void levels(int N, const std::vector<int> &ia, const std::vector<int> &ja, const std::vector<int> &dptr, bool lower,
            std::vector<int> &order, std::vector<int> &offs) {
  std::vector<int> lev(N, 0);
  int maxl = 0;
  if (lower) {
    for (int i = 0; i < N; i++) {
      int l = 0;
      for (int k = ia[i] - 1; k < dptr[i]; k++) l = std::max(l, lev[ja[k] - 1] + 1);
      lev[i] = l;
      maxl = std::max(maxl, l);
    }
  } else {
    for (int i = N - 1; i >= 0; i--) {
      int l = 0;
      for (int k = dptr[i] + 1; k < ia[i + 1] - 1; k++) l = std::max(l, lev[ja[k] - 1] + 1);
      lev[i] = l;
      maxl = std::max(maxl, l);
    }
  }
  offs.assign(maxl + 2, 0);
  for (int i = 0; i < N; i++) offs[lev[i] + 1]++;
  for (int l = 0; l <= maxl; l++) offs[l + 1] += offs[l];
  order.assign(N, 0);
  std::vector<int> pos(offs.begin(), offs.end() - 1);
  for (int i = 0; i < N; i++) order[pos[lev[i]]++] = i;  // ascending rows within a level
}

}  // namespace

extern "C" void load_external_lu_solver(float *CSR_LU, int *CSR_I, int *CSR_J, int N, int M) {
  LegacyLU &L = g_lu;
  if (L.loaded) die("ILU0 solver already loaded:", "call unload_external_lu_solver first");
  if (N <= 0 || !CSR_LU || !CSR_I || !CSR_J) die("ILU0 Info Error =", "invalid arguments");
  (void)M;
  L.N = N;
  L.val = CSR_LU;
  L.ia = CSR_I;
  L.ja = CSR_J;
  std::vector<int> ia(N + 1);
  ck(cudaMemcpy(ia.data(), CSR_I, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost), "ILU0 Buffer Size Error =");
  L.nnz = ia[N] - 1;
  if (L.nnz <= 0) die("ILU0 Buffer Size Error =", "empty matrix");
  std::vector<int> ja(L.nnz);
  ck(cudaMemcpy(ja.data(), CSR_J, sizeof(int) * L.nnz, cudaMemcpyDeviceToHost), "ILU0 Buffer Size Error =");
  std::vector<int> dptr(N, -1);
  for (int i = 0; i < N; i++)
    for (int k = ia[i] - 1; k < ia[i + 1] - 1; k++)
      if (ja[k] == i + 1) dptr[i] = k;
  for (int i = 0; i < N; i++)
    if (dptr[i] < 0) die("ILU0 Structural Zero Pivot at row", std::to_string(i + 1).c_str());
  std::vector<int> of, ob;
  levels(N, ia, ja, dptr, true, of, L.lev_f);
  levels(N, ia, ja, dptr, false, ob, L.lev_b);
  ck(cudaStreamCreate(&L.stream), "ILU0 Setup Error =");  // blocking: ordered after the legacy default stream
  ck(cudaMalloc(&L.dptr, sizeof(int) * N), "ILU0 Buffer Error =");
  ck(cudaMalloc(&L.dinv, sizeof(float) * N), "ILU0 Buffer Error =");
  ck(cudaMalloc(&L.x32, sizeof(float) * N), "ILU0 Buffer Error =");
  ck(cudaMalloc(&L.rows_f, sizeof(int) * N), "ILU0 Buffer Error =");
  ck(cudaMalloc(&L.rows_b, sizeof(int) * N), "ILU0 Buffer Error =");
  int *d_piv = nullptr;
  ck(cudaMalloc(&d_piv, sizeof(int)), "ILU0 Buffer Error =");
  ck(cudaMemcpy(L.dptr, dptr.data(), sizeof(int) * N, cudaMemcpyHostToDevice), "ILU0 Setup Error =");
  ck(cudaMemcpy(L.rows_f, of.data(), sizeof(int) * N, cudaMemcpyHostToDevice), "ILU0 Setup Error =");
  ck(cudaMemcpy(L.rows_b, ob.data(), sizeof(int) * N, cudaMemcpyHostToDevice), "ILU0 Setup Error =");
  const int big = 0x7fffffff;
  ck(cudaMemcpy(d_piv, &big, sizeof(int), cudaMemcpyHostToDevice), "ILU0 Setup Error =");
  // Factorise level by level (rows of one level are independent).
  for (size_t l = 0; l + 1 < L.lev_f.size(); l++) {
    const int n = L.lev_f[l + 1] - L.lev_f[l];
    if (n > 0)
      k_lu_factor<<<(n + 127) / 128, 128, 0, L.stream>>>(L.rows_f + L.lev_f[l], n, L.ia, L.ja, L.dptr, L.val, d_piv);
  }
  k_lu_dinv<<<(N + 255) / 256, 256, 0, L.stream>>>(N, L.dptr, L.val, L.dinv);
  ck(cudaGetLastError(), "ILU0 Factorization Error =");
  int piv = big;
  ck(cudaMemcpyAsync(&piv, d_piv, sizeof(int), cudaMemcpyDeviceToHost, L.stream), "ILU0 Factorization Error =");
  ck(cudaStreamSynchronize(L.stream), "ILU0 Factorization Error =");
  cudaFree(d_piv);
  if (piv != big) die("ILU0 Zero Pivot at row", std::to_string(piv).c_str());
  int nrm2 = 0, ntm2 = 0, npm2 = 0;
  if (seven_point(N, ia, ja, &nrm2, &ntm2, &npm2)) {
    // the wavefront route: a solver object holding only the grid and a stream
    pot3d::Solver *w = new pot3d::Solver();
    pot3d::Geo &g = w->g;
    g.nrm2 = nrm2;
    g.ntm2 = ntm2;
    g.npm2 = npm2;
    g.nr = nrm2 + 2;
    g.nt = ntm2 + 2;
    g.np = npm2 + 2;
    g.NRP = (nrm2 + 15) / 16 * 16;
    g.N = (long long)nrm2 * ntm2 * npm2;
    g.Np = (long long)g.NRP * ntm2 * npm2;
    L.wave = w;
    ck(cudaStreamCreate(&w->stream), "ILU0 Setup Error =");
    if (pot3d::dilu_setup_csr(w, L.ia, L.ja, L.dptr, L.val, L.dinv) != POT3D_OK)
      die("ILU0 Setup Error =", pot3d_gpu_last_error());
    ck(cudaStreamSynchronize(w->stream), "ILU0 Setup Error =");
    L.loaded = true;
    return;
  }
  // The per-call sweeps, captured once.
  cudaGraph_t graph;
  ck(cudaStreamBeginCapture(L.stream, cudaStreamCaptureModeThreadLocal), "Forward Solve Error =");
  for (size_t l = 0; l + 1 < L.lev_f.size(); l++) {
    const int n = L.lev_f[l + 1] - L.lev_f[l];
    if (n > 0)
      k_lu_forward<<<(n + 127) / 128, 128, 0, L.stream>>>(L.rows_f + L.lev_f[l], n, L.ia, L.ja, L.dptr, L.val, L.x32);
  }
  for (size_t l = 0; l + 1 < L.lev_b.size(); l++) {
    const int n = L.lev_b[l + 1] - L.lev_b[l];
    if (n > 0)
      k_lu_backward<<<(n + 127) / 128, 128, 0, L.stream>>>(L.rows_b + L.lev_b[l], n, L.ia, L.ja, L.dptr, L.val,
                                                            L.dinv, L.x32);
  }
  ck(cudaStreamEndCapture(L.stream, &graph), "Backward Solve Error =");
  ck(cudaGraphInstantiate(&L.sweeps, graph, 0), "Backward Solve Error =");
  cudaGraphDestroy(graph);
  ck(cudaDeviceSynchronize(), "ILU0 Setup Error =");
  L.loaded = true;
}

extern "C" void external_lu_solver(double *x) {
  LegacyLU &L = g_lu;
  if (!L.loaded) die("Forward Solve Error =", "load_external_lu_solver was not called");
  const int nb = std::min((L.N + 255) / 256, 148 * 8);
  if (L.wave) {
    pot3d::Solver *w = L.wave;
    k_lu_narrow_pad<<<nb, 256, 0, w->stream>>>(w->g, x, pot3d::dilu_r32(w));
    ck(cudaGetLastError(), "Forward Solve Error =");
    if (pot3d::dilu_sweeps(w, false) != POT3D_OK) die("Forward Solve Error =", pot3d_gpu_last_error());
    k_lu_widen_pad<<<nb, 256, 0, w->stream>>>(w->g, pot3d::dilu_z32(w), x);
    ck(cudaGetLastError(), "Backward Solve Error =");
    if (pot3d::dilu_status(w) != POT3D_OK) die("Backward Solve Error =", pot3d_gpu_last_error());
    return;
  }
  k_lu_narrow<<<nb, 256, 0, L.stream>>>(L.N, x, L.x32);
  ck(cudaGetLastError(), "Forward Solve Error =");
  ck(cudaGraphLaunch(L.sweeps, L.stream), "Forward Solve Error =");
  k_lu_widen<<<nb, 256, 0, L.stream>>>(L.N, L.x32, x);
  ck(cudaGetLastError(), "Backward Solve Error =");
  ck(cudaStreamSynchronize(L.stream), "Backward Solve Error =");
}

extern "C" void unload_external_lu_solver(void) {
  LegacyLU &L = g_lu;
  if (!L.loaded) return;
  cudaStreamSynchronize(L.stream);
  delete L.wave;  // its stream, sweeps and buffers
  if (L.sweeps) cudaGraphExecDestroy(L.sweeps);
  cudaFree(L.dptr);
  cudaFree(L.dinv);
  cudaFree(L.x32);
  cudaFree(L.rows_f);
  cudaFree(L.rows_b);
  cudaStreamDestroy(L.stream);
  L = LegacyLU();
  cudaDeviceSynchronize();
}
