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
// Wavefront sweeps.  One persistent kernel per triangular solve.
//
// Each thread owns one radial-latitude line (e, j) and walks it along phi
// (k), so the periodic seam coupling between the first and the last phi
// plane stays in the thread's registers.  A block owns a tile of 16 x 16
// lines; thread (el, jl) is skewed by s = el + jl steps (mirrored in the
// backward sweep), so at step t it handles plane k = t - s and its
// neighbours (e-1, j, k) and (e, j-1, k) were produced by the threads
// (el-1, jl) and (el, jl-1) one step earlier: the block runs in lockstep,
// one barrier per step, and exchanges them through shared memory.
//
// Across tile faces values travel as 64-bit words holding the FP32 value
// and a sweep tag.  A word is indexed by the step at which its consumer
// needs it, so the words of one face for 8 consecutive steps are one
// contiguous block; the whole block fetches the next 8 steps' words (and,
// forward, the neighbour pivots) one chunk ahead, checks their tags when
// the chunk starts and polls again (bounded) only for words not yet
// written.  Tiles are taken in the order of the tickets of a global
// counter, sorted so that every tile's producers (e-1 and j-1 faces)
// hold smaller tickets: a block only ever waits for a tile already owned
// by a running block, and the kernel needs no co-residency.  The last
// block to finish resets the counter and advances the tag.
//
// Every value is computed with the operations, and in the order, of the
// reference's lusol (src/pot3d.F90:5227-5302), so the sweeps are
// bit-identical to it.
// ============================================================================
constexpr int WE = 16, WJT = 16;        // lines per tile in e and j
constexpr int WAVE_THREADS = WE * WJT;  // one thread per line
constexpr int WCH = 8;                  // steps per exchange chunk
constexpr int WPF = 4;                  // prefetch distance of the point loads (steps)
constexpr int WSK = (WE - 1) + (WJT - 1);
constexpr unsigned WAVE_SPIN_LIMIT = 1u << 22;
static_assert(2 * WCH * 16 == WAVE_THREADS, "one exchange word per thread and chunk");
static_assert(WCH % WPF == 0, "chunk is a whole number of prefetch rounds");

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
  const float *dfac;  // factor diagonal d (forward neighbour pivots)
  unsigned long long *xe, *xj;  // e-face and j-face exchange words
  const int2 *order;  // ticket -> tile (te, tj) in forward order
  WaveCtl *ctl;
  SolveState *st;
  int check;          // skip when the solve state is no longer running
  int nte, ntj, ntiles, ndiag;
};

__device__ __forceinline__ void wave_publish(unsigned long long *p, unsigned epoch, float v) {
  const unsigned long long w = ((unsigned long long)epoch << 32) | __float_as_uint(v);
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long wave_load(const unsigned long long *p) {
  unsigned long long w;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}

struct WaveSmem {
  float y[2][WJT][WE + 1];           // step parity, line values
  float dv[2][WJT][WE + 1];          // forward: the lines' pivots d at their current point
  float ring[2][2][WCH][16];         // chunk parity, face (0: e, 1: j), step in chunk, line
  float dring[2][2][WCH][16];        // forward: pivots of the neighbours across the faces
  int2 tile;
  int abort;
};

// Exchange slot (face, step s of chunk, line) of thread T.
__device__ __forceinline__ void wave_slot(int T, int *f, int *s, int *line) {
  *f = T >> 7;
  *s = (T >> 4) & (WCH - 1);
  *line = T & 15;
}

template <bool FWD>
__device__ __forceinline__ bool wave_tile(const WaveArgs &a, WaveSmem &S, const double *kdph, const double *kdpi,
                                          unsigned epoch, int te, int tj) {
  const Geo &g = a.g;
  const DevMesh &m = a.m;
  const int T = threadIdx.x;
  const int el = T & (WE - 1), jl = T / WE;
  const int e = te * WE + el, jj = tj * WJT + jl;
  const bool valid = e < g.nrm2 && jj < g.ntm2;
  const int sk = FWD ? el + jl : (WE - 1 - el) + (WJT - 1 - jl);
  const int npm2 = g.npm2;
  const long long plane = (long long)g.ntm2 * g.NRP;
  const long long row = (long long)(valid ? jj : 0) * g.NRP + (valid ? e : 0);
  // neighbour tiles across the faces this tile consumes and produces
  const int te_in = FWD ? te - 1 : te + 1, tj_in = FWD ? tj - 1 : tj + 1;
  const int te_out = FWD ? te + 1 : te - 1, tj_out = FWD ? tj + 1 : tj - 1;
  const bool has_in_e = te_in >= 0 && te_in < a.nte, has_in_j = tj_in >= 0 && tj_in < a.ntj;
  const bool pub_e = valid && (FWD ? el == WE - 1 : el == 0) && te_out >= 0 && te_out < a.nte;
  const bool pub_j = valid && (FWD ? jl == WJT - 1 : jl == 0) && tj_out >= 0 && tj_out < a.ntj;
  const bool ext_e = FWD ? el == 0 : el == WE - 1;    // e-neighbour across the face
  const bool ext_j = FWD ? jl == 0 : jl == WJT - 1;   // j-neighbour across the face
  const bool cpl_e = valid && (FWD ? e > 0 : e < g.nrm2 - 1);
  const bool cpl_j = valid && (FWD ? jj > 0 : jj < g.ntm2 - 1);
  unsigned long long *xe_out = a.xe + (size_t)(tj * a.nte + te) * a.ndiag * 16;
  unsigned long long *xj_out = a.xj + (size_t)(tj * a.nte + te) * a.ndiag * 16;
  // per-line constants of the coefficients (load_matrix_pot3d_solve's operand order)
  double drh = 0, c17 = 0, sd = 0, stj = 0, dtij = 0, r2i = 0, drii = 0;
  if (valid) {
    const int i = e + 2, j = jj + 2;
    drh = m.drh[i];
    c17 = __dmul_rn(__dmul_rn(drh, m.dth[j]), m.sth_i[j]);
    sd = __dmul_rn(m.sth[j], m.dth[j]);
    stj = FWD ? m.st[j - 1] : m.st[j];
    dtij = FWD ? m.dt_i[j - 1] : m.dt_i[j];
    r2i = FWD ? m.r2[i - 1] : m.r2[i];
    drii = FWD ? m.dr_i[i - 1] : m.dr_i[i];
  }
  // exchange slot of this thread: who consumes it, which word it is
  int xf, xs, xl;
  wave_slot(T, &xf, &xs, &xl);
  const bool x_tile = xf == 0 ? has_in_e : has_in_j;
  const unsigned long long *x_src =
      xf == 0 ? a.xe + (size_t)(tj * a.nte + (x_tile ? te_in : te)) * a.ndiag * 16
              : a.xj + (size_t)((x_tile ? tj_in : tj) * a.nte + te) * a.ndiag * 16;
  // the consumer of slot (xf, *, xl): thread (el_c, jl_c) of this tile
  const int el_c = xf == 0 ? (FWD ? 0 : WE - 1) : xl, jl_c = xf == 0 ? xl : (FWD ? 0 : WJT - 1);
  const int e_c = te * WE + el_c, jj_c = tj * WJT + jl_c;
  const int sk_c = FWD ? el_c + jl_c : (WE - 1 - el_c) + (WJT - 1 - jl_c);
  const bool x_line = x_tile && e_c < g.nrm2 && jj_c < g.ntm2;
  // the neighbour point across the face (forward: its pivot is needed)
  const int e_n = xf == 0 ? e_c + (FWD ? -1 : 1) : e_c, jj_n = xf == 1 ? jj_c + (FWD ? -1 : 1) : jj_c;
  auto x_needed = [&](int t) {
    const int q = t - sk_c;
    return x_line && t < a.ndiag && q >= 0 && q < npm2;
  };
  auto x_kk = [&](int t) { return FWD ? t - sk_c : npm2 - 1 - (t - sk_c); };
  unsigned long long xw = 0;  // word of the next chunk
  float xd = 0.f;             // forward: neighbour pivot of the next chunk
  auto x_fetch = [&](int c) {
    const int t = c * WCH + xs;
    if (x_needed(t)) {
      xw = wave_load(x_src + (size_t)t * 16 + xl);
      if (FWD) xd = a.dfac[(long long)x_kk(t) * plane + (long long)jj_n * g.NRP + e_n];
    }
  };
  // Commit the fetched chunk c into ring slot c & 1; false on a timeout.
  auto x_commit = [&](int c) {
    const int t = c * WCH + xs;
    bool ok = true;
    if (x_needed(t)) {
      unsigned it = 0;
      while ((unsigned)(xw >> 32) != epoch) {
        if (++it > WAVE_SPIN_LIMIT) {
          ok = false;
          break;
        }
        if (it > 8) __nanosleep(32);
        xw = wave_load(x_src + (size_t)t * 16 + xl);
      }
      S.ring[c & 1][xf][xs][xl] = __uint_as_float((unsigned)xw);
      if (FWD) S.dring[c & 1][xf][xs][xl] = xd;
    }
    return ok;
  };

  const float *pin = a.in + row, *pdd = a.d + row;
  float *pout = a.out + row;
  auto kk_of = [&](int t) { return FWD ? t - sk : npm2 - 1 - (t - sk); };
  auto active = [&](int t) { return valid && t - sk >= 0 && t - sk < npm2; };
  float ib[WPF], db[WPF];
#pragma unroll
  for (int u = 0; u < WPF; u++) {
    const bool ld = active(u);
    ib[u] = ld ? pin[kk_of(u) * plane] : 0.f;
    db[u] = ld ? pdd[kk_of(u) * plane] : 0.f;
  }
  float seam_y = 0.f, seam_d = 0.f;  // value (and pivot) at the line's first plane of the sweep
  float prev = 0.f, dprev = 0.f;     // own value and pivot at the previous step
  const int nsteps = npm2 + WSK;
  const int nch = (nsteps + WCH - 1) / WCH;
  x_fetch(0);
  bool ok = x_commit(0);
  x_fetch(1);
  if (!ok) S.abort = 1;
  __syncthreads();
  if (S.abort) return false;
  for (int c = 0; c < nch; c++) {
    if (c > 0) {
      ok = x_commit(c);
      x_fetch(c + 1);
      if (!ok) S.abort = 1;
      __syncthreads();
      if (S.abort) return false;
    }
#pragma unroll
    for (int u = 0; u < WCH; u++) {
      const int t = c * WCH + u;
      const int p = (t + 1) & 1;  // buffer of step t-1
      const float v_in = ib[u % WPF], d_own = db[u % WPF];
      {  // prefetch the point WPF steps ahead
        const int tf = t + WPF;
        const bool ld = active(tf);
        ib[u % WPF] = ld ? pin[kk_of(tf) * plane] : 0.f;
        db[u % WPF] = ld ? pdd[kk_of(tf) * plane] : 0.f;
      }
      if (active(t)) {
        const int kk = kk_of(t);
        const int K = kk + 2;
        float ne, nj, dne = 0.f, dnj = 0.f;
        if (ext_e) {
          ne = S.ring[c & 1][0][u][jl];
          if (FWD) dne = S.dring[c & 1][0][u][jl];
        } else {
          ne = S.y[p][jl][FWD ? el - 1 : el + 1];
          if (FWD) dne = S.dv[p][jl][el - 1];
        }
        if (ext_j) {
          nj = S.ring[c & 1][1][u][el];
          if (FWD) dnj = S.dring[c & 1][1][u][el];
        } else {
          nj = S.y[p][FWD ? jl - 1 : jl + 1][el];
          if (FWD) dnj = S.dv[p][jl - 1][el];
        }
        const double dphk = kdph[K];
        const double u2 = __dmul_rn(drh, dphk);
        const double v = __dmul_rn(sd, dphk);
        float y;
        if (FWD) {
          // y = r - [seam] - (a1/d) y(k-1) - (a2/d) y(j-1) - (a3/d) y(e-1)
          y = v_in;
          if (kk == npm2 - 1) {
            const float aik = __double2float_rn(-__dmul_rn(c17, kdpi[K]));
            y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, seam_d), seam_y));
          }
          if (kk > 0) {
            const float aik = __double2float_rn(-__dmul_rn(c17, kdpi[K - 1]));
            y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dprev), prev));
          }
          if (cpl_j) {
            const float aik = __double2float_rn(-__dmul_rn(__dmul_rn(u2, stj), dtij));
            y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dnj), nj));
          }
          if (cpl_e) {
            const float aik = __double2float_rn(-__dmul_rn(__dmul_rn(v, r2i), drii));
            y = __fsub_rn(y, __fmul_rn(__fdiv_rn(aik, dne), ne));
          }
          if (kk == 0) {
            seam_y = y;
            seam_d = d_own;
          }
          S.dv[t & 1][jl][el] = d_own;
        } else {
          // z = (y - a5 z(e+1) - a6 z(j+1) - a7 z(k+1) - [seam]) * dinv
          y = v_in;
          if (cpl_e) {
            const float aij = __double2float_rn(-__dmul_rn(__dmul_rn(v, r2i), drii));
            y = __fsub_rn(y, __fmul_rn(aij, ne));
          }
          if (cpl_j) {
            const float aij = __double2float_rn(-__dmul_rn(__dmul_rn(u2, stj), dtij));
            y = __fsub_rn(y, __fmul_rn(aij, nj));
          }
          if (kk < npm2 - 1) {
            const float aij = __double2float_rn(-__dmul_rn(c17, kdpi[K]));
            y = __fsub_rn(y, __fmul_rn(aij, prev));
          }
          if (kk == 0) {
            const float aij = __double2float_rn(-__dmul_rn(c17, kdpi[K - 1]));
            y = __fsub_rn(y, __fmul_rn(aij, seam_y));
          }
          y = __fmul_rn(y, d_own);
          if (kk == npm2 - 1) seam_y = y;
        }
        S.y[t & 1][jl][el] = y;
        pout[(long long)kk * plane] = y;
        if (pub_e) wave_publish(xe_out + (size_t)(t - (WE - 1)) * 16 + jl, epoch, y);
        if (pub_j) wave_publish(xj_out + (size_t)(t - (WJT - 1)) * 16 + el, epoch, y);
        prev = y;
        dprev = d_own;
      }
      __syncthreads();
    }
  }
  return true;
}

template <bool FWD>
__global__ void __launch_bounds__(WAVE_THREADS) k_dilu_wave(WaveArgs a) {
  extern __shared__ double wave_k[];  // dph(K), dp_i(K) for K = 0..np
  __shared__ WaveSmem S;
  const Geo &g = a.g;
  double *kdph = wave_k, *kdpi = wave_k + (g.np + 1);
  for (int K = threadIdx.x; K <= g.np; K += blockDim.x) {
    kdph[K] = K >= 1 ? a.m.dph[K] : 0.0;
    kdpi[K] = K >= 1 ? a.m.dp_i[K] : 0.0;
  }
  if (threadIdx.x == 0) S.abort = 0;
  __syncthreads();
  const unsigned epoch = *(volatile unsigned *)&a.ctl->epoch;
  const bool run = !(a.check && *(volatile int *)&a.st->status != ST_RUNNING);
  while (run) {
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(&a.ctl->ticket, 1u);
      S.tile = t < (unsigned)a.ntiles ? a.order[FWD ? t : a.ntiles - 1 - t] : make_int2(-1, -1);
    }
    __syncthreads();
    const int2 tile = S.tile;
    if (tile.x < 0) break;
    if (!wave_tile<FWD>(a, S, kdph, kdpi, epoch, tile.x, tile.y)) {
      if (threadIdx.x == 0) {
        atomicExch(&a.ctl->error, 1);
        if (a.st) atomicExch(&a.st->status, ST_TIMEOUT);
      }
      break;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.ctl->done, 1u) == gridDim.x - 1) {  // last block: reset for the next sweep
      atomicExch(&a.ctl->ticket, 0u);
      atomicExch(&a.ctl->done, 0u);
      __threadfence();
      atomicAdd(&a.ctl->epoch, 1u);
    }
  }
}

__global__ void k_narrow_rhs(long long n, const double *__restrict__ b, float *__restrict__ r32) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    r32[t] = (float)b[t];
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
  unsigned long long *xe = nullptr, *xj = nullptr;
  int2 *order = nullptr;
  WaveCtl *ctl = nullptr;
  int nte = 0, ntj = 0, ntiles = 0, ndiag = 0, wave_blocks = 0;
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
  D->nte = (g.nrm2 + WE - 1) / WE;
  D->ntj = (g.ntm2 + WJT - 1) / WJT;
  D->ntiles = D->nte * D->ntj;
  D->ndiag = g.npm2 + 16;
  const size_t nx = (size_t)D->ntiles * D->ndiag * 16;
  int st;
  if ((st = s->alloc((void **)&D->xe, 8 * nx)) || (st = s->alloc((void **)&D->xj, 8 * nx)) ||
      (st = s->alloc((void **)&D->order, sizeof(int2) * D->ntiles)) ||
      (st = s->alloc((void **)&D->ctl, sizeof(WaveCtl))))
    return st;
  // Tickets in order of the tile's first wavefront step WE te + WJT tj
  // (ties by te): a tile's producers (te-1, tj) and (te, tj-1) have smaller
  // keys; the backward sweep takes the tickets in reverse.
  std::vector<int2> ord;
  ord.reserve(D->ntiles);
  for (int tj = 0; tj < D->ntj; tj++)
    for (int te = 0; te < D->nte; te++) ord.push_back(make_int2(te, tj));
  std::stable_sort(ord.begin(), ord.end(), [](const int2 &x, const int2 &y) {
    const int kx = WE * x.x + WJT * x.y, ky = WE * y.x + WJT * y.y;
    return kx != ky ? kx < ky : x.x < y.x;
  });
  CK(cudaMemcpyAsync(D->order, ord.data(), sizeof(int2) * D->ntiles, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemsetAsync(D->xe, 0, 8 * nx, s->stream));
  CK(cudaMemsetAsync(D->xj, 0, 8 * nx, s->stream));
  const WaveCtl c0{0u, 0u, 1u, 0};  // tag 0 is the zeroed buffers': sweeps start at 1
  CK(cudaMemcpyAsync(D->ctl, &c0, sizeof(WaveCtl), cudaMemcpyHostToDevice, s->stream));
  D->wave_smem = sizeof(double) * 2 * (g.np + 1);
  const size_t smem_total = D->wave_smem + sizeof(WaveSmem);
  if (smem_total > 48 * 1024) {
    CK(cudaFuncSetAttribute(k_dilu_wave<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem));
    CK(cudaFuncSetAttribute(k_dilu_wave<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem));
  }
  int dev = 0, nsm = 0, occ_f = 0, occ_b = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_dilu_wave<true>, WAVE_THREADS, D->wave_smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_dilu_wave<false>, WAVE_THREADS, D->wave_smem));
  D->wave_blocks = std::max(1, std::min(std::max(1, std::min(occ_f, occ_b)) * nsm, D->ntiles));
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
  a.dfac = D->d;
  a.xe = D->xe;
  a.xj = D->xj;
  a.order = D->order;
  a.ctl = D->ctl;
  a.st = s->d_state;
  a.check = check ? 1 : 0;
  a.nte = D->nte;
  a.ntj = D->ntj;
  a.ntiles = D->ntiles;
  a.ndiag = D->ndiag;
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

// Average device time of the forward and of the backward sweep over `reps`
// applications to the FP32 right-hand side.
int dilu_time(Solver *s, int reps, double ms[2]) {
  DiluState *D = s->dilu;
  int st;
  if ((st = dilu_reset(s))) return st;
  k_narrow_rhs<<<grid1d(s->g.Np), NTHR, 0, s->stream>>>(s->g.Np, s->d_b, D->r32);
  cudaEvent_t e[3];
  for (auto &x : e) CK(cudaEventCreate(&x));
  ms[0] = ms[1] = 0.0;
  for (int it = 0; it < reps; it++) {
    CK(cudaEventRecord(e[0], s->stream));
    launch_wave(s, true, false);
    CK(cudaEventRecord(e[1], s->stream));
    launch_wave(s, false, false);
    CK(cudaEventRecord(e[2], s->stream));
    CK(cudaEventSynchronize(e[2]));
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, e[0], e[1]);
    cudaEventElapsedTime(&b, e[1], e[2]);
    ms[0] += a / reps;
    ms[1] += b / reps;
  }
  for (auto &x : e) cudaEventDestroy(x);
  return dilu_status(s);
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
