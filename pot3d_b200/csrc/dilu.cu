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

// ============================================================================
// Wavefront sweeps.  One persistent kernel per triangular solve.  The (j, k)
// lines of the interior are cut into tiles of 4 x 8 lines; one warp owns a
// tile for the whole radial extent, lane (jl, kl) = (lane & 3, lane >> 2)
// owning one line.  Lanes are skewed by s = jl + kl steps (mirrored in the
// backward sweep), so at its step t a lane handles point e = t - s and the
// lower neighbours it needs, (e, j-1, k) and (e, j, k-1), were produced by
// lanes L-1 and L-4 one step earlier: a warp shuffle.  Across tile faces,
// and through the periodic seam, values travel as 64-bit words holding the
// FP32 value and a sweep tag, written once and polled by the consumer until
// the tag matches (bounded spin; a timeout marks the solve state).  Warps
// take tiles in the order of the tickets of a global counter, sorted so
// every tile's producers hold smaller tickets: a warp only ever waits on a
// tile already owned by a running warp, so the kernel needs no co-residency.
// The last warp to finish resets the counter and advances the sweep tag.
// Every value is computed with the level kernels' operations in the same
// order (the reference's lusol), so the result is bit-identical to them.
// ============================================================================
constexpr int WJ = 4, WK = 8;           // lines per tile in j and k
constexpr int WAVE_THREADS = 128;
constexpr int WAVE_PF = 8;              // prefetch distance (steps) of the point loads
constexpr unsigned WAVE_SPIN_LIMIT = 1u << 22;

struct WaveCtl {
  unsigned ticket, done, epoch;
  int error;
};

struct WaveArgs {
  Geo g;
  DevMesh m;
  const float *in;    // forward: r32 ; backward: y32
  float *out;         // forward: y32 ; backward: z32
  const float *d;     // forward: factor diagonal d ; backward: dinv
  unsigned long long *xj, *xk, *xs;  // tile-face and seam exchange words
  const int2 *order;  // ticket -> tile (tj, tk) in forward order
  WaveCtl *ctl;
  SolveState *st;
  int check;          // skip when the solve state is no longer running
  int ntj, ntk, ntiles;
};

__device__ __forceinline__ void wave_publish(unsigned long long *p, unsigned epoch, float v) {
  const unsigned long long w = ((unsigned long long)epoch << 32) | __float_as_uint(v);
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ bool wave_take(const unsigned long long *p, unsigned epoch, float *v) {
  unsigned long long w;
  for (unsigned it = 0;; it++) {
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    if ((unsigned)(w >> 32) == epoch) break;
    if (it >= WAVE_SPIN_LIMIT) return false;
    if (it >= 16) __nanosleep(64);
  }
  *v = __uint_as_float((unsigned)w);
  return true;
}

// Forward solve of one tile: y = r - sum_{lower} (a/d) y, lusol's row order
// [seam, k-1, j-1, i-1].  Returns false on an exchange timeout.
__device__ __forceinline__ bool wave_tile_forward(const WaveArgs &a, const double *sh, unsigned epoch, int tj,
                                                  int tk, int lane) {
  const Geo &g = a.g;
  const DevMesh &m = a.m;
  const int jl = lane & 3, kl = lane >> 2;
  const int jj = tj * WJ + jl, kk = tk * WK + kl;
  const bool valid = jj < g.ntm2 && kk < g.npm2;
  const int sk = jl + kl;
  const int nr2 = g.nrm2;
  const double *sh_drh = sh, *sh_r2 = sh + nr2, *sh_dri = sh + 2 * nr2;
  double dth_j = 0, sthi_j = 0, dpi_km1 = 0, dpi_k = 0, dph_k = 0, st_jm1 = 0, dti_jm1 = 0, v = 0;
  if (valid) {
    const int j = jj + 2, k = kk + 2;
    dth_j = m.dth[j];
    sthi_j = m.sth_i[j];
    dpi_km1 = m.dp_i[k - 1];
    dpi_k = m.dp_i[k];
    dph_k = m.dph[k];
    st_jm1 = m.st[j - 1];
    dti_jm1 = m.dt_i[j - 1];
    v = __dmul_rn(__dmul_rn(m.sth[j], dth_j), dph_k);
  }
  const long long base = valid ? ((long long)kk * g.ntm2 + jj) * g.NRP : 0;
  const long long plane = (long long)g.ntm2 * g.NRP;
  const bool use_seam = valid && kk == g.npm2 - 1;
  const bool pub_j = valid && jl == WJ - 1 && tj + 1 < a.ntj;
  const bool pub_k = valid && kl == WK - 1 && tk + 1 < a.ntk;
  const bool pub_s = valid && kk == 0;
  const unsigned long long *cj = tj > 0 ? a.xj + ((size_t)(tk * a.ntj + tj - 1) * WK + kl) * nr2 : a.xj;
  const unsigned long long *ck = tk > 0 ? a.xk + ((size_t)((tk - 1) * a.ntj + tj) * WJ + jl) * nr2 : a.xk;
  unsigned long long *pj = a.xj + ((size_t)(tk * a.ntj + tj) * WK + kl) * nr2;
  unsigned long long *pk = a.xk + ((size_t)(tk * a.ntj + tj) * WJ + jl) * nr2;
  unsigned long long *xs = a.xs + (size_t)jj * nr2;
  const float *pin = a.in + base, *pd = a.d + base;
  float *pout = a.out + base;
  float rbuf[WAVE_PF], dbuf[WAVE_PF];
#pragma unroll
  for (int u = 0; u < WAVE_PF; u++) {  // points e = u - sk of the first steps
    const int e = u - sk;
    const bool ld = valid && e >= 0 && e < nr2;
    rbuf[u] = ld ? pin[e] : 0.f;
    dbuf[u] = ld ? pd[e] : 0.f;
  }
  float yprev = 0.f, dprev = 0.f;
  bool ok = true;
  const int nsteps = nr2 + (WJ - 1) + (WK - 1);
  for (int t0 = 0; t0 < nsteps; t0 += WAVE_PF) {
#pragma unroll
    for (int u = 0; u < WAVE_PF; u++) {
      const int t = t0 + u;
      const float yj_in = __shfl_up_sync(0xffffffffu, yprev, 1);
      const float yk_in = __shfl_up_sync(0xffffffffu, yprev, WJ);
      const float dj_in = __shfl_up_sync(0xffffffffu, dprev, 1);
      const float dk_in = __shfl_up_sync(0xffffffffu, dprev, WJ);
      const int e = t - sk;
      const float r_e = rbuf[u], d_e = dbuf[u];
      {  // prefetch the point WAVE_PF steps ahead into the freed slot
        const int ef = e + WAVE_PF;
        const bool ld = valid && ef >= 0 && ef < nr2;
        rbuf[u] = ld ? pin[ef] : 0.f;
        dbuf[u] = ld ? pd[ef] : 0.f;
      }
      if (t < nsteps && valid && e >= 0 && e < nr2) {
        const double drh = sh_drh[e];
        const double c17 = __dmul_rn(__dmul_rn(drh, dth_j), sthi_j);
        float y = r_e;
        if (use_seam) {
          const float aik = __double2float_rn(-__dmul_rn(c17, dpi_k));
          float ys = 0.f;
          ok &= wave_take(a.xs + (size_t)jj * nr2 + e, epoch, &ys);
          const float ds = a.d[(long long)jj * g.NRP + e];
          y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, ds), ys));
        }
        if (kk > 0) {
          const float aik = __double2float_rn(-__dmul_rn(c17, dpi_km1));
          float yk = yk_in, dk = dk_in;
          if (kl == 0) {
            ok &= wave_take(ck + e, epoch, &yk);
            dk = pd[e - plane];
          }
          y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dk), yk));
        }
        if (jj > 0) {
          const double u2 = __dmul_rn(drh, dph_k);
          const float aik = __double2float_rn(-__dmul_rn(__dmul_rn(u2, st_jm1), dti_jm1));
          float yj = yj_in, dj = dj_in;
          if (jl == 0) {
            ok &= wave_take(cj + e, epoch, &yj);
            dj = pd[e - g.NRP];
          }
          y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dj), yj));
        }
        if (e > 0) {
          const float aik = __double2float_rn(-__dmul_rn(__dmul_rn(v, sh_r2[e]), sh_dri[e]));
          y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dprev), yprev));
        }
        pout[e] = y;
        if (pub_j) wave_publish(pj + e, epoch, y);
        if (pub_k) wave_publish(pk + e, epoch, y);
        if (pub_s) wave_publish(xs + e, epoch, y);
        yprev = y;
        dprev = d_e;
      }
    }
    if (__any_sync(0xffffffffu, !ok)) return false;
  }
  return true;
}

// Backward solve of one tile: z = (y - sum_{upper} a z) * dinv, lusol's row
// order [i+1, j+1, k+1, seam].  Mirror image of the forward tile.
__device__ __forceinline__ bool wave_tile_backward(const WaveArgs &a, const double *sh, unsigned epoch, int tj,
                                                   int tk, int lane) {
  const Geo &g = a.g;
  const DevMesh &m = a.m;
  const int jl = lane & 3, kl = lane >> 2;
  const int jj = tj * WJ + jl, kk = tk * WK + kl;
  const bool valid = jj < g.ntm2 && kk < g.npm2;
  const int sk = (WJ - 1 - jl) + (WK - 1 - kl);
  const int nr2 = g.nrm2;
  const double *sh_drh = sh, *sh_r2 = sh + nr2, *sh_dri = sh + 2 * nr2;
  double dth_j = 0, sthi_j = 0, dpi_km1 = 0, dpi_k = 0, dph_k = 0, st_j = 0, dti_j = 0, v = 0;
  if (valid) {
    const int j = jj + 2, k = kk + 2;
    dth_j = m.dth[j];
    sthi_j = m.sth_i[j];
    dpi_km1 = m.dp_i[k - 1];
    dpi_k = m.dp_i[k];
    dph_k = m.dph[k];
    st_j = m.st[j];
    dti_j = m.dt_i[j];
    v = __dmul_rn(__dmul_rn(m.sth[j], dth_j), dph_k);
  }
  const long long base = valid ? ((long long)kk * g.ntm2 + jj) * g.NRP : 0;
  const bool up_j = valid && jj < g.ntm2 - 1, up_k = valid && kk < g.npm2 - 1;
  const bool use_seam = valid && kk == 0;
  const bool pub_j = valid && jl == 0 && tj > 0;
  const bool pub_k = valid && kl == 0 && tk > 0;
  const bool pub_s = valid && kk == g.npm2 - 1;
  const unsigned long long *cj = tj + 1 < a.ntj ? a.xj + ((size_t)(tk * a.ntj + tj + 1) * WK + kl) * nr2 : a.xj;
  const unsigned long long *ck = tk + 1 < a.ntk ? a.xk + ((size_t)((tk + 1) * a.ntj + tj) * WJ + jl) * nr2 : a.xk;
  unsigned long long *pj = a.xj + ((size_t)(tk * a.ntj + tj) * WK + kl) * nr2;
  unsigned long long *pk = a.xk + ((size_t)(tk * a.ntj + tj) * WJ + jl) * nr2;
  unsigned long long *xs = a.xs + (size_t)jj * nr2;
  const float *pin = a.in + base, *pdi = a.d + base;
  float *pout = a.out + base;
  float ybuf[WAVE_PF], dbuf[WAVE_PF];
#pragma unroll
  for (int u = 0; u < WAVE_PF; u++) {
    const int e = nr2 - 1 - (u - sk);
    const bool ld = valid && e >= 0 && e < nr2;
    ybuf[u] = ld ? pin[e] : 0.f;
    dbuf[u] = ld ? pdi[e] : 0.f;
  }
  float zprev = 0.f;
  bool ok = true;
  const int nsteps = nr2 + (WJ - 1) + (WK - 1);
  for (int t0 = 0; t0 < nsteps; t0 += WAVE_PF) {
#pragma unroll
    for (int u = 0; u < WAVE_PF; u++) {
      const int t = t0 + u;
      const float zj_in = __shfl_down_sync(0xffffffffu, zprev, 1);
      const float zk_in = __shfl_down_sync(0xffffffffu, zprev, WJ);
      const int e = nr2 - 1 - (t - sk);
      const float y_e = ybuf[u], di_e = dbuf[u];
      {
        const int ef = e - WAVE_PF;
        const bool ld = valid && ef >= 0 && ef < nr2;
        ybuf[u] = ld ? pin[ef] : 0.f;
        dbuf[u] = ld ? pdi[ef] : 0.f;
      }
      if (t < nsteps && valid && e >= 0 && e < nr2) {
        const double drh = sh_drh[e];
        float z = y_e;
        if (e < nr2 - 1) {
          const float aij = __double2float_rn(-__dmul_rn(__dmul_rn(v, sh_r2[e]), sh_dri[e]));
          z = __fsub_rn(z, __fmul_rn(aij, zprev));
        }
        if (up_j) {
          const double u2 = __dmul_rn(drh, dph_k);
          const float aij = __double2float_rn(-__dmul_rn(__dmul_rn(u2, st_j), dti_j));
          float zj = zj_in;
          if (jl == WJ - 1) ok &= wave_take(cj + e, epoch, &zj);
          z = __fsub_rn(z, __fmul_rn(aij, zj));
        }
        const double c17 = __dmul_rn(__dmul_rn(drh, dth_j), sthi_j);
        if (up_k) {
          const float aij = __double2float_rn(-__dmul_rn(c17, dpi_k));
          float zk = zk_in;
          if (kl == WK - 1) ok &= wave_take(ck + e, epoch, &zk);
          z = __fsub_rn(z, __fmul_rn(aij, zk));
        }
        if (use_seam) {
          const float aij = __double2float_rn(-__dmul_rn(c17, dpi_km1));
          float zs = 0.f;
          ok &= wave_take(a.xs + (size_t)jj * nr2 + e, epoch, &zs);
          z = __fsub_rn(z, __fmul_rn(aij, zs));
        }
        z = __fmul_rn(z, di_e);
        pout[e] = z;
        if (pub_j) wave_publish(pj + e, epoch, z);
        if (pub_k) wave_publish(pk + e, epoch, z);
        if (pub_s) wave_publish(xs + e, epoch, z);
        zprev = z;
      }
    }
    if (__any_sync(0xffffffffu, !ok)) return false;
  }
  return true;
}

template <bool FWD>
__global__ void __launch_bounds__(WAVE_THREADS) k_dilu_wave(WaveArgs a) {
  extern __shared__ double wave_sh[];  // drh(i), r2(i-1|i), dr_i(i-1|i) for the block's radial points
  const Geo &g = a.g;
  for (int e = threadIdx.x; e < g.nrm2; e += blockDim.x) {
    const int i = e + 2;
    wave_sh[e] = a.m.drh[i];
    wave_sh[g.nrm2 + e] = FWD ? a.m.r2[i - 1] : a.m.r2[i];
    wave_sh[2 * g.nrm2 + e] = FWD ? a.m.dr_i[i - 1] : a.m.dr_i[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned epoch = *(volatile unsigned *)&a.ctl->epoch;
  bool run = !(a.check && *(volatile int *)&a.st->status != ST_RUNNING);
  while (run) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(&a.ctl->ticket, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= (unsigned)a.ntiles) break;
    const int2 tile = a.order[FWD ? t : a.ntiles - 1 - t];
    const bool ok = FWD ? wave_tile_forward(a, wave_sh, epoch, tile.x, tile.y, lane)
                        : wave_tile_backward(a, wave_sh, epoch, tile.x, tile.y, lane);
    if (!ok) {
      if (lane == 0) {
        atomicExch(&a.ctl->error, 1);
        if (a.st) atomicExch(&a.st->status, ST_TIMEOUT);
      }
      run = false;
    }
  }
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    const unsigned total = gridDim.x * (blockDim.x / 32);
    if (atomicAdd(&a.ctl->done, 1u) == total - 1) {  // last warp: reset for the next sweep
      atomicExch(&a.ctl->ticket, 0u);
      atomicExch(&a.ctl->done, 0u);
      __threadfence();
      atomicAdd(&a.ctl->epoch, 1u);
    }
  }
}

__global__ void k_wave_reset(WaveCtl *c) {
  c->ticket = 0;
  c->done = 0;
  c->epoch += 1;
  c->error = 0;
}

struct DiluState {
  float *d = nullptr, *dinv = nullptr, *r32 = nullptr, *y32 = nullptr, *z32 = nullptr;
  int *pivot = nullptr;
  int nlev = 0;
  std::vector<int> kk_lo, nkk, nblk;  // per level launch shape (factorisation)
  // wavefront sweeps
  unsigned long long *xj = nullptr, *xk = nullptr, *xs = nullptr;
  int2 *order = nullptr;
  WaveCtl *ctl = nullptr;
  int ntj = 0, ntk = 0, ntiles = 0, wave_blocks = 0;
  size_t wave_smem = 0;
};

static void level_shape(const Geo &g, int l, int *kk_lo, int *nkk, int *nblk) {
  const int lo = std::max(0, l - (g.nrm2 - 1) - (g.ntm2 - 1));
  const int hi = std::min(g.npm2 - 1, l);
  *kk_lo = lo;
  *nkk = hi - lo + 1;
  const int span = std::min(g.nrm2, g.ntm2);  // valid jj per kk
  *nblk = (span + 127) / 128;
}

static void launch_factor_level(Solver *s, int l) {
  DiluState *D = s->dilu;
  LevelArgs a{};
  a.g = s->g;
  a.m = s->m;
  a.level = l;
  a.kk_lo = D->kk_lo[l];
  a.d = D->d;
  a.dinv = D->dinv;
  a.pivot = D->pivot;
  dim3 grid(D->nblk[l], D->nkk[l]);
  k_dilu_factor<<<grid, 128, 0, s->stream>>>(a);
}

// Exchange buffers, tile order and launch shape of the wavefront sweeps.
static int wave_setup(Solver *s) {
  DiluState *D = s->dilu;
  const Geo &g = s->g;
  D->ntj = (g.ntm2 + WJ - 1) / WJ;
  D->ntk = (g.npm2 + WK - 1) / WK;
  D->ntiles = D->ntj * D->ntk;
  const size_t nxj = (size_t)D->ntiles * WK * g.nrm2, nxk = (size_t)D->ntiles * WJ * g.nrm2,
               nxs = (size_t)g.ntm2 * g.nrm2;
  int st;
  if ((st = s->alloc((void **)&D->xj, 8 * nxj)) || (st = s->alloc((void **)&D->xk, 8 * nxk)) ||
      (st = s->alloc((void **)&D->xs, 8 * nxs)) || (st = s->alloc((void **)&D->order, sizeof(int2) * D->ntiles)) ||
      (st = s->alloc((void **)&D->ctl, sizeof(WaveCtl))))
    return st;
  // Tickets in order of the tile's first wavefront step 4 tj + 8 tk (ties by
  // tj): every producer of a tile (tj-1, tk), (tj, tk-1) and, through the
  // seam, (tj, 0) has a smaller key.
  std::vector<int2> ord;
  ord.reserve(D->ntiles);
  for (int tk = 0; tk < D->ntk; tk++)
    for (int tj = 0; tj < D->ntj; tj++) ord.push_back(make_int2(tj, tk));
  std::stable_sort(ord.begin(), ord.end(), [](const int2 &x, const int2 &y) {
    const int kx = WJ * x.x + WK * x.y, ky = WJ * y.x + WK * y.y;
    return kx != ky ? kx < ky : x.x < y.x;
  });
  CK(cudaMemcpyAsync(D->order, ord.data(), sizeof(int2) * D->ntiles, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemsetAsync(D->xj, 0, 8 * nxj, s->stream));
  CK(cudaMemsetAsync(D->xk, 0, 8 * nxk, s->stream));
  CK(cudaMemsetAsync(D->xs, 0, 8 * nxs, s->stream));
  CK(cudaMemsetAsync(D->ctl, 0, sizeof(WaveCtl), s->stream));
  D->wave_smem = sizeof(double) * 3 * g.nrm2;
  if (D->wave_smem > 48 * 1024) {
    CK(cudaFuncSetAttribute(k_dilu_wave<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem));
    CK(cudaFuncSetAttribute(k_dilu_wave<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem));
  }
  int dev = 0, nsm = 0, occ_f = 0, occ_b = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_dilu_wave<true>, WAVE_THREADS, D->wave_smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_dilu_wave<false>, WAVE_THREADS, D->wave_smem));
  const int warps = std::max(1, std::min(occ_f, occ_b)) * nsm * (WAVE_THREADS / 32);
  D->wave_blocks = std::max(1, std::min(warps, D->ntiles) / (WAVE_THREADS / 32));
  return POT3D_OK;
}

static void launch_wave(Solver *s, bool fwd, bool check) {
  DiluState *D = s->dilu;
  WaveArgs a{};
  a.g = s->g;
  a.m = s->m;
  a.in = fwd ? D->r32 : D->y32;
  a.out = fwd ? D->y32 : D->z32;
  a.d = fwd ? D->d : D->dinv;
  a.xj = D->xj;
  a.xk = D->xk;
  a.xs = D->xs;
  a.order = D->order;
  a.ctl = D->ctl;
  a.st = s->d_state;
  a.check = check ? 1 : 0;
  a.ntj = D->ntj;
  a.ntk = D->ntk;
  a.ntiles = D->ntiles;
  if (fwd)
    k_dilu_wave<true><<<D->wave_blocks, WAVE_THREADS, D->wave_smem, s->stream>>>(a);
  else
    k_dilu_wave<false><<<D->wave_blocks, WAVE_THREADS, D->wave_smem, s->stream>>>(a);
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
  if ((st = wave_setup(s))) return st;
  D->nlev = g.nrm2 + g.ntm2 + g.npm2 - 2;
  D->kk_lo.resize(D->nlev);
  D->nkk.resize(D->nlev);
  D->nblk.resize(D->nlev);
  for (int l = 0; l < D->nlev; l++) level_shape(g, l, &D->kk_lo[l], &D->nkk[l], &D->nblk[l]);
  const int big = 0x7fffffff;
  if ((st = pot3d_cuda_status(cudaMemcpyAsync(D->pivot, &big, sizeof(int), cudaMemcpyHostToDevice, s->stream),
                              "cudaMemcpy(pivot)")))
    return st;
  for (int l = 0; l < D->nlev; l++) launch_factor_level(s, l);
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
int dilu_sweep_launches(Solver *s) { return s->dilu ? 2 : 0; }

int dilu_sweeps(Solver *s, bool check_status) {
  launch_wave(s, true, check_status);
  launch_wave(s, false, check_status);
  return pot3d_cuda_status(cudaGetLastError(), "ILU(0) sweeps");
}

// Status of the sweeps issued so far (synchronises the solver stream).
int dilu_status(Solver *s) {
  WaveCtl c{};
  CK(cudaMemcpyAsync(&c, s->dilu->ctl, sizeof(WaveCtl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (c.error) {
    pot3d_set_error("ILU(0) wavefront sweep: a tile exchange wait ran out");
    return POT3D_ERR_TIMEOUT;
  }
  return POT3D_OK;
}

// Clear the sweeps' ticket counter and advance their tag (start of a solve;
// also recovers the counters after an aborted sweep).
int dilu_reset(Solver *s) {
  k_wave_reset<<<1, 1, 0, s->stream>>>(s->dilu->ctl);
  return pot3d_cuda_status(cudaGetLastError(), "k_wave_reset");
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
