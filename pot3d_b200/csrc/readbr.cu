// readbr's work after the file read (src/pot3d.F90:6751-6829) and set_flux's
// |Br| for option 'open' (src/pot3d.F90:3832), on the device: the map
// fi(ntn, npn) with its scales is interpolated bilinearly onto the half-mesh
// points th(2:ntm1) x ph(2:npm1) (intrp2d, src/pot3d.F90:6833-6932, with
// interp's interval search, :7028-7072), copied periodically in phi, given
// the m=0 pole values, and flux-balanced.  Every operation rounds
// separately and the sums run in the reference's loop order (one thread),
// so br0 is bit for bit the host's (and the oracle's) readbr.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pot3d_internal.cuh"
#include "pot3d_solver.h"

namespace pot3d {

// interp's bracket: the first interval [x[q], x[q+1]] holding v, and its
// weight; -1 and an error flag when v lies outside the table.
__global__ void k_bracket(const double *__restrict__ x, int n, const double *__restrict__ v, int lo, int hi,
                          int *__restrict__ idx, double *__restrict__ w, int *__restrict__ err) {
  const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i > hi) return;
  const double vi = v[i];
  for (int q = 0; q + 1 < n; q++)
    if (vi >= x[q] && vi <= x[q + 1]) {
      idx[i] = q;
      w[i] = __ddiv_rn(__dsub_rn(vi, x[q]), __dsub_rn(x[q + 1], x[q]));
      return;
    }
  idx[i] = -1;
  atomicExch(err, 1);
}

// intrp2d at the interior points (j, k) (1-based 2..ntm1, 2..npm1).
__global__ void k_br0_interp(int nt, int np, int ntn, const double *__restrict__ fi, const int *__restrict__ jb,
                             const double *__restrict__ ax, const int *__restrict__ kb, const double *__restrict__ ay,
                             double *__restrict__ br0) {
  const long long n = (long long)(nt - 2) * (np - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % (nt - 2)) + 2, k = (int)(t / (nt - 2)) + 2;
    const int a = jb[j], b = kb[k];
    const double wx = ax[j], wy = ay[k];
    const double f00 = fi[a + (size_t)ntn * b], f01 = fi[a + (size_t)ntn * (b + 1)];
    const double f10 = fi[a + 1 + (size_t)ntn * b], f11 = fi[a + 1 + (size_t)ntn * (b + 1)];
    const double cy = __dsub_rn(1.0, wy), cx = __dsub_rn(1.0, wx);
    const double t0 = __dadd_rn(__dmul_rn(cy, f00), __dmul_rn(wy, f01));
    const double t1 = __dadd_rn(__dmul_rn(cy, f10), __dmul_rn(wy, f11));
    br0[(j - 1) + (size_t)nt * (k - 1)] = __dadd_rn(__dmul_rn(cx, t0), __dmul_rn(wx, t1));
  }
}

// Periodic copy, pole values from the ring sums, and the flux balance's
// sums, in the reference's order (one thread); out[0] = the offset.
__global__ void k_br0_rings_flux(int nt, int np, DevMesh m, double *__restrict__ br0, double *__restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  auto B = [&](int j, int k) -> double & { return br0[(j - 1) + (size_t)nt * (k - 1)]; };  // 1-based
  for (int j = 1; j <= nt; j++) {
    B(j, 1) = B(j, np - 1);
    B(j, np) = B(j, 2);
  }
  const double pl_i = __ddiv_rn(1.0, 2.0 * 3.1415926535897932);
  double n0 = 0.0, n1 = 0.0;
  for (int k = 2; k <= np - 1; k++) n0 = __dadd_rn(n0, __dmul_rn(B(2, k), m.dph[k]));
  for (int k = 2; k <= np - 1; k++) n1 = __dadd_rn(n1, __dmul_rn(B(nt - 1, k), m.dph[k]));
  n0 = __dmul_rn(n0, pl_i);
  n1 = __dmul_rn(n1, pl_i);
  for (int k = 1; k <= np; k++) {
    B(1, k) = __dsub_rn(__dmul_rn(2.0, n0), B(2, k));
    B(nt, k) = __dsub_rn(__dmul_rn(2.0, n1), B(nt - 1, k));
  }
  double area = 0.0, fp = 0.0, fm = 0.0;
  for (int j = 2; j <= nt - 1; j++)
    for (int k = 2; k <= np - 1; k++) {
      const double da = __dmul_rn(__dmul_rn(m.sth[j], m.dth[j]), m.dph[k]);
      const double v = B(j, k);
      if (v > 0.)
        fp = __dadd_rn(fp, __dmul_rn(v, da));
      else
        fm = __dadd_rn(fm, __dmul_rn(v, da));
      area = __dadd_rn(area, da);
    }
  out[0] = __ddiv_rn(__dadd_rn(fp, fm), area);
}

__global__ void k_br0_offset(long long n, const double *__restrict__ off, int balance, int absolute,
                             double *__restrict__ br0) {
  const double o = balance ? off[0] : 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    double v = balance ? __dsub_rn(br0[t], o) : br0[t];
    br0[t] = absolute ? fabs(v) : v;
  }
}

}  // namespace pot3d

struct pot3d_gpu_solver;  // api.cu: holds the Solver as its first member
namespace pot3d {
Solver *solver_of(pot3d_gpu_solver *h);
}

extern "C" int pot3d_gpu_br0_from_map(pot3d_gpu_solver *h, int ntn, int npn, const double *tn, const double *pn,
                                      const double *fi, int option, int do_not_balance_flux, double *br0_out) {
  using namespace pot3d;
  if (!h || ntn < 2 || npn < 2 || !tn || !pn || !fi || option < 0 || option > 2) {
    pot3d_set_error("pot3d_gpu_br0_from_map: invalid arguments");
    return POT3D_ERR_ARG;
  }
  // flint's monotonicity check of the scales (src/pot3d.F90:6934-7026)
  for (int q = 1; q < ntn; q++)
    if (!(tn[q] > tn[q - 1])) {
      pot3d_set_error("pot3d_gpu_br0_from_map: the theta scale is not increasing");
      return POT3D_ERR_ARG;
    }
  for (int q = 1; q < npn; q++)
    if (!(pn[q] > pn[q - 1])) {
      pot3d_set_error("pot3d_gpu_br0_from_map: the phi scale is not increasing");
      return POT3D_ERR_ARG;
    }
  Solver &s = *solver_of(h);
  const Geo &g = s.g;
  const int nt = g.nt, np = g.np;
  const size_t nfi = (size_t)ntn * npn;
  // one transient block: tn, pn, fi, the brackets and weights, the offset, the error flag
  const size_t doubles = ntn + npn + nfi + (nt + 2) + (np + 2) + 2;
  const size_t bytes = sizeof(double) * doubles + sizeof(int) * (nt + np + 8);
  unsigned char *d = nullptr;
  if (cudaMallocAsync((void **)&d, bytes, s.stream) != cudaSuccess) {
    cudaGetLastError();
    pot3d_set_error("pot3d_gpu_br0_from_map: device allocation failed");
    return POT3D_ERR_NOMEM;
  }
  double *d_tn = reinterpret_cast<double *>(d), *d_pn = d_tn + ntn, *d_fi = d_pn + npn;
  double *d_ax = d_fi + nfi, *d_ay = d_ax + (nt + 2), *d_off = d_ay + (np + 2);
  int *d_jb = reinterpret_cast<int *>(d_off + 2), *d_kb = d_jb + (nt + 2), *d_err = d_kb + (np + 2);
  double *br0 = const_cast<double *>(s.m.br0);
  int st = POT3D_OK, err = 0;
  auto ok = [&](cudaError_t e, const char *w) { return st == POT3D_OK && (st = pot3d_cuda_status(e, w)) == POT3D_OK; };
  ok(cudaMemcpyAsync(d_tn, tn, sizeof(double) * ntn, cudaMemcpyHostToDevice, s.stream), "br0: tn");
  ok(cudaMemcpyAsync(d_pn, pn, sizeof(double) * npn, cudaMemcpyHostToDevice, s.stream), "br0: pn");
  ok(cudaMemcpyAsync(d_fi, fi, sizeof(double) * nfi, cudaMemcpyHostToDevice, s.stream), "br0: fi");
  ok(cudaMemsetAsync(d_err, 0, sizeof(int), s.stream), "br0: flag");
  if (st == POT3D_OK) {
    // interp brackets of th(2:ntm1) in tn and of ph(2:npm1) in pn (1-based mesh indices)
    k_bracket<<<(nt + 127) / 128, 128, 0, s.stream>>>(d_tn, ntn, s.m.th, 2, nt - 1, d_jb, d_ax, d_err);
    k_bracket<<<(np + 127) / 128, 128, 0, s.stream>>>(d_pn, npn, s.m.ph, 2, np - 1, d_kb, d_ay, d_err);
    ok(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s.stream), "br0: flag");
    ok(cudaStreamSynchronize(s.stream), "br0: brackets");
  }
  if (st == POT3D_OK && err) {
    pot3d_set_error("pot3d_gpu_br0_from_map: a mesh point lies outside the map's scales");
    st = POT3D_ERR_ARG;
  }
  if (st == POT3D_OK) {
    k_br0_interp<<<grid1d((long long)(nt - 2) * (np - 2)), NTHR, 0, s.stream>>>(nt, np, ntn, d_fi, d_jb, d_ax, d_kb,
                                                                                d_ay, br0);
    k_br0_rings_flux<<<1, 32, 0, s.stream>>>(nt, np, s.m, br0, d_off);
    const int balance = !((option == 1 || option == 2) && do_not_balance_flux);
    k_br0_offset<<<grid1d((long long)nt * np), NTHR, 0, s.stream>>>((long long)nt * np, d_off, balance, option == 1,
                                                                     br0);
    ok(cudaGetLastError(), "br0 kernels");
  }
  if (st == POT3D_OK) st = s.rhs_padded(s.d_b);  // the RHS follows the new map (as pot3d_gpu_set_br0)
  if (st == POT3D_OK && br0_out)
    ok(cudaMemcpyAsync(br0_out, br0, sizeof(double) * nt * np, cudaMemcpyDeviceToHost, s.stream), "br0: out");
  const int fst = pot3d_cuda_status(cudaFreeAsync(d, s.stream), "br0: free");
  if (st == POT3D_OK) ok(cudaStreamSynchronize(s.stream), "br0");
  return st != POT3D_OK ? st : fst;
}
