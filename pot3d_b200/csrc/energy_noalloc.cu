// Magnetic-energy diagnostic that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// owned by another allocator or pool (a Fortran/OpenMP runtime that maps all
// arrays itself, a framework that forbids foreign allocations), or a process
// that must not grow its device footprint after start-up.  For them this file
// provides pot3d_gpu_energy_noalloc: the same getb + magnetic_energy
// reduction as pot3d_gpu_energy (src/pot3d.F90:6187-6321), on caller-owned
// device arrays, with its scratch -- one partial sum per phi plane and
// energy component -- in a file-scope __device__ array.
//
// Limits and sharing: the scratch holds ENERGY_NOALLOC_MAX_PLANES planes,
// so np-2 may not exceed it (larger meshes are rejected with
// POT3D_ERR_ARG).  The array lives on every GPU that loads the library until
// the process exits.  All calls share it: a call writes every slot it reads
// before reading it, so nothing has to start at zero, but two calls whose
// kernels overlap on the GPU (different streams, or different host threads)
// race on it and must be serialised by the caller.  The first call on a
// device looks up the array's device address with cudaGetSymbolAddress (the
// host-side name is only a stand-in for it) and keeps it for the life of the
// process; make that first call before any stream capture begins, and do not
// use the entry point again after cudaDeviceReset (the kept address belongs
// to the context that looked it up).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "pot3d_internal.cuh"

namespace {

constexpr int ENERGY_NOALLOC_MAX_PLANES = 8192;
constexpr int ENERGY_NOALLOC_THREADS = 256;
constexpr int ENERGY_NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_energy_scratch[3 * ENERGY_NOALLOC_MAX_PLANES];

std::mutex g_scratch_mutex;
double *g_scratch_ptr[ENERGY_NOALLOC_MAX_DEVICES] = {nullptr};

// One block per interior phi plane k = 2..np-1; 0-based mesh arrays.
__global__ void __launch_bounds__(ENERGY_NOALLOC_THREADS)
    k_energy_plane(int nr, int nt, const double *__restrict__ rh, const double *__restrict__ dr,
                   const double *__restrict__ drh, const double *__restrict__ dt, const double *__restrict__ dth,
                   const double *__restrict__ sth, const double *__restrict__ dp, const double *__restrict__ dph,
                   const double *__restrict__ phi, double *__restrict__ part) {
  __shared__ double red[ENERGY_NOALLOC_THREADS / 32];
  const int k = blockIdx.x + 2;  // Fortran plane index
  const long long nrr = nr, ntr = (long long)nr * nt;
  const int nin = (nr - 2) * (nt - 2);
  double wr = 0.0, wt = 0.0, wp = 0.0;
  for (int t = threadIdx.x; t < nin; t += blockDim.x) {
    const int i = t % (nr - 2) + 2, j = t / (nr - 2) + 2;  // Fortran indices
    const long long c = (i - 1) + nrr * (j - 1) + ntr * (k - 1);
    const double f = phi[c];
    const double rhi = rh[i - 1];
    const double br_p = (phi[c + 1] - f) / dr[i - 1];
    const double br_m = (f - phi[c - 1]) / dr[i - 2];
    const double bt_p = (phi[c + nrr] - f) / (rhi * dt[j - 1]);
    const double bt_m = (f - phi[c - nrr]) / (rhi * dt[j - 2]);
    const double rs = __dmul_rn(rhi, sth[j - 1]);
    const double bp_p = (phi[c + ntr] - f) / (rs * dp[k - 1]);
    const double bp_m = (f - phi[c - ntr]) / (rs * dp[k - 2]);
    const double dv = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(rhi, rhi), drh[i - 1]), dth[j - 1]),
                                          sth[j - 1]),
                                dph[k - 1]);
    const double brav = 0.5 * (br_p + br_m);
    const double btav = 0.5 * (bt_p + bt_m);
    const double bpav = 0.5 * (bp_p + bp_m);
    wr += __dmul_rn(0.5 * __dmul_rn(brav, brav), dv);
    wt += __dmul_rn(0.5 * __dmul_rn(btav, btav), dv);
    wp += __dmul_rn(0.5 * __dmul_rn(bpav, bpav), dv);
  }
  const double s0 = pot3d::block_sum<ENERGY_NOALLOC_THREADS>(wr, red);
  const double s1 = pot3d::block_sum<ENERGY_NOALLOC_THREADS>(wt, red);
  const double s2 = pot3d::block_sum<ENERGY_NOALLOC_THREADS>(wp, red);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = s0;
    part[3 * blockIdx.x + 1] = s1;
    part[3 * blockIdx.x + 2] = s2;
  }
}

// Plane sums added in plane order, as the reference's k-outer loop nest.
__global__ void k_energy_planes_total(const double *__restrict__ part, int nplanes, double *__restrict__ w) {
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int b = 0; b < nplanes; b++) s += part[3 * b + threadIdx.x];
    w[threadIdx.x] = s;
  }
}

// Device address of the scratch array on the current device (set up once).
int scratch_on_current_device(double **out) {
  int dev = 0;
  int st = pot3d_cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (st) return st;
  if (dev < 0 || dev >= ENERGY_NOALLOC_MAX_DEVICES) {
    pot3d_set_error("pot3d_gpu_energy_noalloc: device index out of range");
    return POT3D_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    st = pot3d_cuda_status(cudaGetSymbolAddress(&p, g_energy_scratch), "cudaGetSymbolAddress(g_energy_scratch)");
    if (st) return st;
    g_scratch_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_ptr[dev];
  return POT3D_OK;
}

}  // namespace

extern "C" int pot3d_gpu_energy_noalloc(int nr, int nt, int np, const double *rh, const double *dr,
                                        const double *drh, const double *dt, const double *dth, const double *sth,
                                        const double *dp, const double *dph, const double *phi, double *w,
                                        void *stream) {
  if (nr < 3 || nt < 3 || np < 3 || !rh || !dr || !drh || !dt || !dth || !sth || !dp || !dph || !phi || !w) {
    pot3d_set_error("pot3d_gpu_energy_noalloc: invalid mesh size or null pointer");
    return POT3D_ERR_ARG;
  }
  if (np - 2 > ENERGY_NOALLOC_MAX_PLANES) {
    pot3d_set_error("pot3d_gpu_energy_noalloc: np-2 = " + std::to_string(np - 2) +
                    " exceeds the scratch limit of " + std::to_string(ENERGY_NOALLOC_MAX_PLANES) + " phi planes");
    return POT3D_ERR_ARG;
  }
  double *scratch = nullptr;
  int st = scratch_on_current_device(&scratch);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_energy_plane<<<np - 2, ENERGY_NOALLOC_THREADS, 0, s>>>(nr, nt, rh, dr, drh, dt, dth, sth, dp, dph, phi, scratch);
  k_energy_planes_total<<<1, 32, 0, s>>>(scratch, np - 2, w);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_gpu_energy_noalloc");
}
