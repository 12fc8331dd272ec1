// extern "C" entry points of libpot3d_gpu.so (declared in include/pot3d_gpu.h).
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "pot3d_internal.cuh"
#include "pot3d_solver.h"

using pot3d::Solver;

struct pot3d_gpu_solver {
  Solver s;
  double *d_io = nullptr;  // device staging buffer, reference packed layout (N)
  double *d_io2 = nullptr;
};

#define CKS(call)                                                 \
  do {                                                            \
    int _st = pot3d_cuda_status((call), #call);                   \
    if (_st != POT3D_OK) return _st;                              \
  } while (0)

static int check_solver(const pot3d_gpu_solver *h) {
  if (!h) {
    pot3d_set_error("null solver handle");
    return POT3D_ERR_ARG;
  }
  return POT3D_OK;
}

extern "C" int pot3d_gpu_create(const pot3d_mesh_t *mesh, const double *br0, const double *br1, double pm_r1,
                                int ifprec, int precision, int device, pot3d_gpu_solver **out) {
  if (!mesh || !br0 || !out) {
    pot3d_set_error("pot3d_gpu_create: null argument");
    return POT3D_ERR_ARG;
  }
  *out = nullptr;
  if (device >= 0) CKS(cudaSetDevice(device));
  pot3d_gpu_solver *h = new (std::nothrow) pot3d_gpu_solver();
  if (!h) {
    pot3d_set_error("host allocation failed");
    return POT3D_ERR_NOMEM;
  }
  int st = h->s.setup(mesh, br0, br1, pm_r1, ifprec, precision);
  if (st == POT3D_OK) st = h->s.alloc((void **)&h->d_io, sizeof(double) * (size_t)h->s.g.N);
  if (st == POT3D_OK) st = h->s.alloc((void **)&h->d_io2, sizeof(double) * (size_t)h->s.g.N);
  if (st != POT3D_OK) {
    delete h;
    return st;
  }
  *out = h;
  return POT3D_OK;
}

extern "C" int pot3d_gpu_destroy(pot3d_gpu_solver *h) {
  delete h;
  return POT3D_OK;
}

extern "C" long pot3d_gpu_size(const pot3d_gpu_solver *h) { return h ? (long)h->s.g.N : 0; }

extern "C" int pot3d_gpu_rhs(pot3d_gpu_solver *h, double *rhs) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  if ((st = s.rhs_padded(s.d_tmp))) return st;
  if ((st = s.unpack(s.d_tmp, h->d_io))) return st;
  CKS(cudaMemcpyAsync(rhs, h->d_io, sizeof(double) * s.g.N, cudaMemcpyDeviceToHost, s.stream));
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

static int solve_common(pot3d_gpu_solver *h, const double *x_dev, const double *r_dev, long N, int ncgmax,
                        double epscg, int *ierr, pot3d_solve_info_t *info, double *x_out, double *r_out) {
  int st;
  Solver &s = h->s;
  if (N != (long)s.g.N) {
    pot3d_set_error("cgsolve: N does not match the mesh");
    return POT3D_ERR_ARG;
  }
  if ((st = s.pack(x_dev, s.d_x))) return st;
  if ((st = s.pack(r_dev, s.d_b))) return st;
  // A zero guess skips the first operator application, as ax(0) = 0.
  bool zero_guess = false;
  {
    if ((st = s.dot_padded(s.d_x, s.d_x, s.d_scalar))) return st;
    double xx = 0;
    CKS(cudaMemcpyAsync(&xx, s.d_scalar, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    CKS(cudaStreamSynchronize(s.stream));
    zero_guess = (xx == 0.0);
  }
  int ie = 1;
  pot3d_solve_info_t inf{};
  if (s.precision == POT3D_FP32_REFINED)
    st = s.mixed_solve(zero_guess, ncgmax, epscg, &ie, &inf);
  else
    st = s.cgsolve_padded(zero_guess, ncgmax, epscg, &ie, &inf);
  if (st) return st;
  double tr = 0.0;
  if ((st = s.true_residual(&tr))) return st;
  inf.true_resid = tr;
  if ((st = s.unpack(s.d_x, x_out))) return st;
  if ((st = s.unpack(s.d_r, r_out))) return st;
  CKS(cudaStreamSynchronize(s.stream));
  if (ierr) *ierr = ie;
  if (info) *info = inf;
  return POT3D_OK;
}

extern "C" int pot3d_gpu_cgsolve_dev(pot3d_gpu_solver *h, double *x, double *r, long N, int ncgmax, double epscg,
                                     int *ierr, pot3d_solve_info_t *info) {
  int st;
  if ((st = check_solver(h))) return st;
  return solve_common(h, x, r, N, ncgmax, epscg, ierr, info, x, r);
}

extern "C" int pot3d_gpu_cgsolve(pot3d_gpu_solver *h, double *x, double *r, long N, int ncgmax, double epscg,
                                 int *ierr, pot3d_solve_info_t *info) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  if (N != (long)s.g.N) {
    pot3d_set_error("cgsolve: N does not match the mesh");
    return POT3D_ERR_ARG;
  }
  const size_t b = sizeof(double) * (size_t)N;
  CKS(cudaMemcpyAsync(h->d_io, x, b, cudaMemcpyHostToDevice, s.stream));
  CKS(cudaMemcpyAsync(h->d_io2, r, b, cudaMemcpyHostToDevice, s.stream));
  if ((st = solve_common(h, h->d_io, h->d_io2, N, ncgmax, epscg, ierr, info, h->d_io, h->d_io2))) return st;
  CKS(cudaMemcpyAsync(x, h->d_io, b, cudaMemcpyDeviceToHost, s.stream));
  CKS(cudaMemcpyAsync(r, h->d_io2, b, cudaMemcpyDeviceToHost, s.stream));
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

extern "C" int pot3d_gpu_history(const pot3d_gpu_solver *h, double *eps, int cap) {
  if (!h || !eps || cap <= 0) return 0;
  const Solver &s = h->s;
  int n = s.last_ncg + 1;
  if (n > cap) n = cap;
  if (n > s.hist_cap) n = s.hist_cap;
  if (cudaMemcpy(eps, s.d_hist, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  return n;
}

extern "C" int pot3d_gpu_finalize_phi(pot3d_gpu_solver *h, const double *x, double *phi) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  const size_t nphi = (size_t)s.g.nr * s.g.nt * s.g.np;
  if (!s.d_phi && (st = s.alloc((void **)&s.d_phi, sizeof(double) * nphi))) return st;
  CKS(cudaMemcpyAsync(h->d_io, x, sizeof(double) * s.g.N, cudaMemcpyHostToDevice, s.stream));
  if ((st = s.pack(h->d_io, s.d_tmp))) return st;
  if ((st = s.finalize_phi_dev(s.d_tmp, s.d_phi))) return st;
  CKS(cudaMemcpyAsync(phi, s.d_phi, sizeof(double) * nphi, cudaMemcpyDeviceToHost, s.stream));
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

extern "C" int pot3d_gpu_energy(pot3d_gpu_solver *h, const double *phi, double w[3]) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  const size_t nphi = (size_t)s.g.nr * s.g.nt * s.g.np;
  if (!s.d_phi && (st = s.alloc((void **)&s.d_phi, sizeof(double) * nphi))) return st;
  CKS(cudaMemcpyAsync(s.d_phi, phi, sizeof(double) * nphi, cudaMemcpyHostToDevice, s.stream));
  return s.energy_dev(s.d_phi, w);
}

extern "C" int pot3d_gpu_fields(pot3d_gpu_solver *h, const double *x, double *phi, double *br, double *bt,
                                double *bp, double w[3]) {
  int st;
  if ((st = check_solver(h))) return st;
  if (!x) {
    pot3d_set_error("pot3d_gpu_fields: null x");
    return POT3D_ERR_ARG;
  }
  Solver &s = h->s;
  const size_t nr = s.g.nr, nt = s.g.nt, np = s.g.np;
  const size_t nphi = nr * nt * np;
  if (!s.d_phi && (st = s.alloc((void **)&s.d_phi, sizeof(double) * nphi))) return st;
  CKS(cudaMemcpyAsync(h->d_io, x, sizeof(double) * s.g.N, cudaMemcpyHostToDevice, s.stream));
  if ((st = s.pack(h->d_io, s.d_tmp))) return st;
  if ((st = s.finalize_phi_dev(s.d_tmp, s.d_phi))) return st;
  if (phi) CKS(cudaMemcpyAsync(phi, s.d_phi, sizeof(double) * nphi, cudaMemcpyDeviceToHost, s.stream));
  if (br || bt || bp) {
    const size_t nbr = (nr - 1) * nt * np, nbt = nr * (nt - 1) * np, nbp = nr * nt * (np - 1);
    double *d_b = nullptr;
    if (cudaMallocAsync((void **)&d_b, sizeof(double) * (nbr + nbt + nbp), s.stream) != cudaSuccess) {
      cudaGetLastError();
      pot3d_set_error("pot3d_gpu_fields: device allocation of the B fields failed");
      return POT3D_ERR_NOMEM;
    }
    st = s.getb_dev(s.d_phi, d_b, d_b + nbr, d_b + nbr + nbt);
    if (!st && br)
      st = pot3d_cuda_status(cudaMemcpyAsync(br, d_b, sizeof(double) * nbr, cudaMemcpyDeviceToHost, s.stream),
                             "fields: br");
    if (!st && bt)
      st = pot3d_cuda_status(
          cudaMemcpyAsync(bt, d_b + nbr, sizeof(double) * nbt, cudaMemcpyDeviceToHost, s.stream), "fields: bt");
    if (!st && bp)
      st = pot3d_cuda_status(
          cudaMemcpyAsync(bp, d_b + nbr + nbt, sizeof(double) * nbp, cudaMemcpyDeviceToHost, s.stream),
          "fields: bp");
    const int fst = pot3d_cuda_status(cudaFreeAsync(d_b, s.stream), "fields: free");
    if (st) return st;
    if (fst) return fst;
  }
  if (w) return s.energy_dev(s.d_phi, w);
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

extern "C" int pot3d_gpu_ax_dev(pot3d_gpu_solver *h, const double *x, double *y) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  if ((st = s.pack(x, s.d_tmp))) return st;
  if ((st = s.ax_padded(s.d_tmp, s.d_q))) return st;
  if ((st = s.unpack(s.d_q, y))) return st;
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

extern "C" int pot3d_gpu_prec_dev(pot3d_gpu_solver *h, double *x) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  if ((st = s.pack(x, s.d_tmp))) return st;
  if ((st = s.prec_padded(s.d_tmp))) return st;
  if ((st = s.unpack(s.d_tmp, x))) return st;
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

// Host copy of a padded FP32 vector in the reference packed layout.
__global__ static void k_unpack_f(pot3d::Geo g, const float *__restrict__ src, float *__restrict__ dst) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.N;
       t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t % g.nrm2);
    const long long line = t / g.nrm2;
    dst[t] = src[line * g.NRP + e];
  }
}

extern "C" int pot3d_gpu_precond_diag(pot3d_gpu_solver *h, float *d, float *dinv) {
  int st;
  if ((st = check_solver(h))) return st;
  Solver &s = h->s;
  if (s.ifprec == 2) return pot3d::dilu_diag(&s, d, dinv);
  float *tmp = reinterpret_cast<float *>(h->d_io);
  k_unpack_f<<<pot3d::grid1d(s.g.N), pot3d::NTHR, 0, s.stream>>>(s.g, s.d_ai, tmp);
  CKS(cudaGetLastError());
  if (d) CKS(cudaMemcpyAsync(d, tmp, sizeof(float) * s.g.N, cudaMemcpyDeviceToHost, s.stream));
  CKS(cudaStreamSynchronize(s.stream));
  if (dinv) memset(dinv, 0, sizeof(float) * s.g.N);
  return POT3D_OK;
}

extern "C" int pot3d_gpu_time_kernels(pot3d_gpu_solver *h, int reps, double ms[2], double bytes[2]) {
  int st;
  if ((st = check_solver(h))) return st;
  if (reps <= 0 || h->s.ifprec == 2) {
    pot3d_set_error("time_kernels: reps must be positive and ifprec 0 or 1");
    return POT3D_ERR_ARG;
  }
  return h->s.time_kernels(reps, ms, bytes);
}

extern "C" int pot3d_gpu_time_sweeps(pot3d_gpu_solver *h, int reps, double ms[2]) {
  int st;
  if ((st = check_solver(h))) return st;
  if (reps <= 0 || h->s.ifprec != 2 || !ms) {
    pot3d_set_error("time_sweeps: reps must be positive and ifprec 2");
    return POT3D_ERR_ARG;
  }
  return pot3d::dilu_time(&h->s, reps, ms);
}

extern "C" int pot3d_gpu_set_br0(pot3d_gpu_solver *h, const double *br0) {
  int st;
  if ((st = check_solver(h))) return st;
  if (!br0) {
    pot3d_set_error("pot3d_gpu_set_br0: null br0");
    return POT3D_ERR_ARG;
  }
  Solver &s = h->s;
  CKS(cudaMemcpyAsync(const_cast<double *>(s.m.br0), br0, sizeof(double) * (size_t)s.g.nt * s.g.np,
                      cudaMemcpyHostToDevice, s.stream));
  if ((st = s.rhs_padded(s.d_b))) return st;
  CKS(cudaStreamSynchronize(s.stream));
  return POT3D_OK;
}

extern "C" int pot3d_gpu_set_refine(pot3d_gpu_solver *h, double refine_ratio, double stall_drop, int stall_limit) {
  int st;
  if ((st = check_solver(h))) return st;
  if (!(refine_ratio > 0.0 && refine_ratio < 1.0) || !(stall_drop > 0.0) || stall_limit < 1) {
    pot3d_set_error("pot3d_gpu_set_refine: need 0 < refine_ratio < 1, stall_drop > 0, stall_limit >= 1");
    return POT3D_ERR_ARG;
  }
  h->s.refine_ratio = refine_ratio;
  h->s.stall_drop = stall_drop;
  h->s.stall_limit = stall_limit;
  return POT3D_OK;
}

extern "C" int pot3d_gpu_refine_info(const pot3d_gpu_solver *h, int *n_refine, int *fallback_iterations) {
  if (!h) {
    pot3d_set_error("null solver handle");
    return POT3D_ERR_ARG;
  }
  if (n_refine) *n_refine = h->s.last_refine;
  if (fallback_iterations) *fallback_iterations = h->s.last_fallback_iters;
  return POT3D_OK;
}

extern "C" int pot3d_gpu_test_sweep_stall(pot3d_gpu_solver *h, unsigned spin_limit) {
  int st;
  if ((st = check_solver(h))) return st;
  if (h->s.ifprec != 2 || spin_limit == 0) {
    pot3d_set_error("pot3d_gpu_test_sweep_stall: needs ifprec 2 and a positive spin limit");
    return POT3D_ERR_ARG;
  }
  return pot3d::dilu_test_stall(&h->s, spin_limit);
}

namespace pot3d {
Solver *solver_of(pot3d_gpu_solver *h) { return &h->s; }
}  // namespace pot3d
