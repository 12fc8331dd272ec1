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
// The factorisation stores d and dinv; the FP32 couplings are the FP64
// coefficients of load_matrix_pot3d_solve formed in the reference's operand
// order and rounded to FP32 as diacsr rounds them.  The wavefront sweeps
// below read them (l = a/d forward, the upper a and dinv backward) from
// streams formed once after the factorisation, in their tile-skewed order.
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
#include <type_traits>
#include <vector>

#include "pot3d_internal.cuh"
#include "pot3d_solver.h"
#include "tma.cuh"

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
// (el-1, jl) and (el, jl-1) one step earlier: the 8 compute warps run in
// lockstep, one named barrier per step, and exchange them through shared
// memory.
//
// Streams.  A copy warp moves everything a tile reads with the bulk copy
// engine, a few steps ahead, into rings tracked by mbarriers, refilling a
// slot as soon as the compute warps report it free, so no copy is issued on
// their step-to-step dependent path: the
// sweep's private streams (coefficients and the intermediate y, stored
// tile-skewed as [tile][group of 4 steps][component][thread] float4 so a
// group of a block is one contiguous copy) and, forward, the r32 input as
// 16 x 16 x 4 boxes of phi planes (a 3-D TMA load, no multicast).  A thread
// then reads 4 steps of a coefficient with one 128-bit shared load.  The
// backward sweep's z32 output goes through a 40-plane ring in shared
// memory: each finished plane of the tile leaves as one 16 x 16 TMA store
// issued by the copy warp, which hands the slot back once the store has read
// it, so the compute warps issue no global stores for z32.
//
// Across tile faces values travel as 64-bit words holding the FP32 value
// and a sweep tag, indexed by the step at which the consumer needs them, so
// the words of one face for 8 consecutive steps are one contiguous block; a
// dedicated exchange warp polls them (bounded) into a ring ahead of the
// compute warps.  Tiles are taken in the order of the tickets of a global
// counter, sorted so that every tile's producers hold smaller tickets: a
// block only waits for a tile owned by a running block, and the kernel
// needs no co-residency.  The last block to finish resets the counter and
// advances the tag.
//
// The FP32 coefficients are formed once, after the factorisation, with the
// reference's operations (lusol's l = a/d of the lower entries and the FP32
// upper entries, src/pot3d.F90:5227-5302) and applied in lusol's order, so
// the sweeps are bit-identical to it.
// ============================================================================
constexpr int WE = 16, WJT = 16;        // lines per tile in e and j
constexpr int WAVE_THREADS = WE * WJT;  // one thread per line (compute warps)
constexpr int WCH = 8;                  // steps per exchange chunk
constexpr int WG = 4;                   // steps per stream group (one float4 per thread and component)
constexpr int WSL = 3;                  // stream group slots (groups g+1, g+2 in flight while g is read)
constexpr int WPD = 2;                  // r32 plane groups issued ahead
constexpr int WSK = (WE - 1) + (WJT - 1);
constexpr int WPG = 11;                 // r32 plane-group slots
constexpr int WROUT = 40;               // output plane ring (backward z32)
constexpr int WXR = 4;                  // exchange ring depth (chunks)
constexpr int WAVE_BLOCK = WAVE_THREADS + 64;  // + exchange warp + copy warp
constexpr unsigned WAVE_SPIN_LIMIT = 1u << 22;
constexpr uint32_t WAVE_MBAR_LIMIT = 1u << 26;
constexpr unsigned WAVE_POLL_NS = 32;        // exchange warp's sleep between polls of a face
static_assert(WCH % WG == 0, "a chunk is whole stream groups");
static_assert(WG * WPG > WSK + (WG - 1) + WG * WPD, "a plane group's slot is free when it is reissued");
static_assert(WROUT >= WSK + 2 * WG + 2, "the copy warp stores a finished plane before its slot is needed again");
static_assert(WPD == WSL - 1, "the r32 plane group of a step group travels with its coefficient group");

struct WaveCtl {
  unsigned ticket, done, epoch;
  int error;
};

struct WaveArgs {
  Geo g;
  float *z32;            // backward output (padded layout)
  float4 *ys;            // intermediate y, [tile][group][thread] (forward step groups)
  const float4 *lf;      // forward coefficients [tile][group][l_k, l_j, l_e][thread]
  const float4 *ub;      // backward coefficients [tile][group][u_e, u_j, u_k, dinv][thread]
  const float *seam_f;   // forward seam coefficient of the last plane, per line
  const float *seam_b;   // backward seam coupling of the first plane, per line
  unsigned long long *xe, *xj;  // e-face and j-face exchange words
  const int2 *order;     // ticket -> tile (te, tj) in forward order
  WaveCtl *ctl;
  SolveState *st;
  int check;             // skip when the solve state is no longer running
  unsigned spin_limit;   // polls of a bounded wait before it gives up (WAVE_SPIN_LIMIT)
  int stall_ticket;      // the block taking this ticket leaves its tile undone (-1: none); the
                         // failure-detection test uses it to make its consumers' waits run out
  int nte, ntj, ntiles, ndiag, nsteps;
  int pad;               // nsteps - (npm2 + WSK): idle steps, trailing forward, leading backward
  // Fused forms (the FP32-inner iteration of the refined mode):
  float4 *rs;            // forward: the FP32 recurrence residual in the stream layout, read and rewritten
  double *rz_part;       // backward: per-tile partial of rho = r.z
  unsigned *tile_done;   // batched backward: the case's finished tiles in this sweep
};

__device__ __forceinline__ void wave_publish(unsigned long long *p, unsigned epoch, float v) {
  const unsigned long long w = ((unsigned long long)epoch << 32) | __float_as_uint(v);
  // no memory clobber: the word carries its own tag, so nothing has to be
  // ordered around the store, and the compute warps' shared-memory traffic
  // is not serialised behind it
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w));
}
__device__ __forceinline__ unsigned long long wave_load(const unsigned long long *p) {
  unsigned long long w;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}
// Bulk copy global -> shared (16-byte aligned, size a multiple of 16),
// completing on the mbarrier.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

struct alignas(128) WaveSmemF {      // forward sweep
  float rin[WPG][WG][WJT][WE];       // r32 (fused: q32) plane groups (TMA boxes), slot = plane group % WPG
  float4 lf[WSL][4][WAVE_THREADS];   // coefficient groups (+ fused: the residual group)
  float y[2][WJT][WE + 1];           // step parity, line values
  float ring[WXR][2][WCH][16];       // chunk % WXR, face (0: e, 1: j), step in chunk, line
  uint64_t bar_s[WSL];                // one per stream slot, also counting the plane group of the step group
  int2 tile;
  int abort, ready, consumed, bcase, gdone, zflushed;  // zflushed unused forward
};
struct alignas(128) WaveSmemB {      // backward sweep
  float4 ub[WSL][4][WAVE_THREADS];   // coefficient groups
  float4 yin[WSL][WAVE_THREADS];     // y groups
  float zout[WROUT][WAVE_THREADS];   // z32 planes [jl][el], slot = plane % WROUT (TMA store source)
  float y[2][WJT][WE + 1];
  float ring[WXR][2][WCH][16];
  double red[WAVE_THREADS / 32];     // fused: the tile's rho partial, per compute warp
  uint64_t bar_s[WSL];
  int2 tile;
  // zflushed: z32 planes, from the top, whose TMA store has read its slot
  int abort, ready, consumed, bcase, gdone, zflushed;
};

template <bool FWD>
struct WaveSmemSel;
template <>
struct WaveSmemSel<true> {
  using type = WaveSmemF;
};
template <>
struct WaveSmemSel<false> {
  using type = WaveSmemB;
};

__device__ __forceinline__ void wave_bar_compute() { asm volatile("bar.sync 1, %0;" ::"n"(WAVE_THREADS) : "memory"); }
// Barrier of the compute warps that also returns whether any of them saw `flag`.
__device__ __forceinline__ bool wave_bar_compute_any(bool flag) {
  unsigned r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; bar.red.or.pred q, 1, %2, p; selp.u32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"((unsigned)flag), "n"(WAVE_THREADS)
      : "memory");
  return r != 0;
}

// Face geometry of one tile, shared by the compute warps and the exchange warp.
struct WaveFaces {
  int te, tj, ti;
  bool has_in[2];  // a producer tile exists across face 0 (e) / 1 (j)
  const unsigned long long *src[2];
};
template <bool FWD>
__device__ __forceinline__ WaveFaces wave_faces(const WaveArgs &a, int te, int tj) {
  WaveFaces f;
  f.te = te;
  f.tj = tj;
  f.ti = tj * a.nte + te;
  const int te_in = FWD ? te - 1 : te + 1, tj_in = FWD ? tj - 1 : tj + 1;
  f.has_in[0] = te_in >= 0 && te_in < a.nte;
  f.has_in[1] = tj_in >= 0 && tj_in < a.ntj;
  f.src[0] = a.xe + (size_t)(tj * a.nte + (f.has_in[0] ? te_in : te)) * a.ndiag * 16;
  f.src[1] = a.xj + (size_t)((f.has_in[1] ? tj_in : tj) * a.nte + te) * a.ndiag * 16;
  return f;
}
// Whether the consumer line `line` of face `face` needs the word of step t.
template <bool FWD>
__device__ __forceinline__ bool wave_needed(const WaveArgs &a, const WaveFaces &f, int face, int line, int t) {
  if (!f.has_in[face]) return false;
  const int el_c = face == 0 ? (FWD ? 0 : WE - 1) : line, jl_c = face == 0 ? line : (FWD ? 0 : WJT - 1);
  if (f.te * WE + el_c >= a.g.nrm2 || f.tj * WJT + jl_c >= a.g.ntm2) return false;
  const int sk_c = FWD ? el_c + jl_c : (WE - 1 - el_c) + (WJT - 1 - jl_c);
  const int q = t - (FWD ? 0 : a.pad) - sk_c;
  return t < a.ndiag && q >= 0 && q < a.g.npm2;
}

// Exchange warp: fills the face ring WXR chunks ahead of the compute warps,
// handing each 4-step group of a chunk over as soon as its words are current.
// Lane L serves face L >> 4, line L & 15, all WCH steps of a chunk.
template <bool FWD>
__device__ __forceinline__ void wave_exchange(const WaveArgs &a, typename WaveSmemSel<FWD>::type &S,
                                              const WaveFaces &f, unsigned epoch, int nch) {
  const int lane = threadIdx.x & 31;
  const int face = lane >> 4, line = lane & 15;
  const unsigned long long *src = f.src[face] + line;
  for (int c = 0; c < nch; c++) {
    // wait for a free ring slot (the compute warps consumed chunk c - WXR)
    unsigned it = 0;
    while (c - *(volatile int *)&S.consumed >= WXR && !*(volatile int *)&S.abort) {
      if (++it > a.spin_limit) {
        S.abort = 1;
        break;
      }
      __nanosleep(128);  // the ring is WXR chunks ahead: no hurry, and no issue slots taken
    }
    if (__any_sync(0xffffffffu, *(volatile int *)&S.abort != 0)) return;  // uniform over the warp
    bool ok = true;
    unsigned long long w[WCH];
    // every needed word of the chunk is loaded in each poll round (the loads
    // overlap), and a round reloads only the words not yet current; each
    // step group of the chunk is handed to the compute warps (S.ready counts
    // groups) as soon as all its words are current
    const unsigned long long done_word = (unsigned long long)epoch << 32;
#pragma unroll
    for (int s = 0; s < WCH; s++)
      w[s] = wave_needed<FWD>(a, f, face, line, c * WCH + s) ? 0ull : done_word;
    constexpr int NGC = WCH / WG;  // step groups per chunk
    int pub = 0;                   // groups of this chunk handed over
    unsigned pit = 0;
    for (;;) {
#pragma unroll
      for (int s = 0; s < WCH; s++)
        if ((unsigned)(w[s] >> 32) != epoch) w[s] = wave_load(src + (size_t)(c * WCH + s) * 16);
      while (pub < NGC) {
        bool cur = true;
#pragma unroll
        for (int s = 0; s < WCH; s++)
          if (s / WG == pub) cur = cur && (unsigned)(w[s] >> 32) == epoch;
        if (!__all_sync(0xffffffffu, cur)) break;
#pragma unroll
        for (int s = 0; s < WCH; s++)
          if (s / WG == pub) S.ring[c % WXR][face][s][line] = __uint_as_float((unsigned)w[s]);
        __syncwarp();
        pub++;
        if (lane == 0) {
          __threadfence_block();
          *(volatile int *)&S.ready = c * NGC + pub;
        }
      }
      if (pub == NGC) break;
      if (++pit > a.spin_limit) {
        ok = false;
        break;
      }
      if (pit > 2) __nanosleep(WAVE_POLL_NS);
    }
    if (!ok) S.abort = 1;
    __syncwarp();
  }
}

// Bounded mbarrier wait of the compute warps that also gives up once the
// block is aborting (the copy it waits for may then never be issued).
__device__ __forceinline__ bool wave_mbar_wait(uint64_t *bar, uint32_t parity, const volatile int *abort) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < WAVE_MBAR_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63) == 63 && *abort) return false;
  }
  return false;
}

// Copy warp: lane 0 issues the tile's bulk copies -- stream group g (the
// coefficients, backward also the forward's y) and, forward, the r32 plane
// group g as a TMA box, both completing on the slot's mbarrier -- as soon as
// the compute warps report the slot free (S.gdone = groups they finished).
// No copy is issued on the compute warps' dependent path.  Before it
// returns after an abort, lane 0 waits (bounded) for what it issued.
template <bool FWD, bool FUSE = false>
__device__ __forceinline__ void wave_copy(const WaveArgs &a, const CUtensorMap *map,
                                          typename WaveSmemSel<FWD>::type &S, const WaveFaces &f, int gbase,
                                          int qbase, bool acquire_map) {
  if ((threadIdx.x & 31) != 0) return;
  const int G = a.nsteps / WG, NQ = (a.g.npm2 + WG - 1) / WG;
  const int npm2 = a.g.npm2;
  const int shift = FWD ? 0 : a.pad;
  const int ti = f.ti;
  const volatile int *abort = &S.abort;
  if (acquire_map) tma_acquire_desc(map);
  int ns = 0;
  int zd = 0;  // backward: z32 planes stored, from the top (npm2-1, npm2-2, ...)
  unsigned it = 0;
  while ((ns < G || (!FWD && zd < npm2)) && !*abort) {
    const int gd = *(volatile int *)&S.gdone;
    __threadfence_block();
    bool worked = false;
    if (ns < G && ns < gd + WSL) {
      // the compute warps' reads of the slots being refilled (ordered before
      // gdone by their barrier and the fences) precede these async writes
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      do {
        const int slot = (gbase + ns) % WSL;
        uint64_t *bar = &S.bar_s[slot];
        if constexpr (FWD) {
          const bool plane = ns < NQ;
          mbar_expect_tx(bar, (FUSE ? 4 : 3) * WAVE_THREADS * 16 + (plane ? WG * WJT * WE * 4 : 0));
          bulk_load(&S.lf[slot][0][0], a.lf + ((size_t)ti * G + ns) * 3 * WAVE_THREADS, 3 * WAVE_THREADS * 16,
                    bar);
          if (FUSE)  // the group's residual r32 (stream layout)
            bulk_load(&S.lf[slot][3][0], a.rs + ((size_t)ti * G + ns) * WAVE_THREADS, WAVE_THREADS * 16, bar);
          if (plane)
            tma_load_3d(&S.rin[(qbase + ns) % WPG][0][0][0], map, f.te * WE, f.tj * WJT, ns * WG, bar);
        } else {
          mbar_expect_tx(bar, 5 * WAVE_THREADS * 16);
          bulk_load(&S.ub[slot][0][0], a.ub + ((size_t)ti * G + ns) * 4 * WAVE_THREADS, 4 * WAVE_THREADS * 16,
                    bar);
          bulk_load(&S.yin[slot][0], a.ys + ((size_t)ti * G + (G - 1 - ns)) * WAVE_THREADS, WAVE_THREADS * 16,
                    bar);
        }
        ns++;
      } while (ns < G && ns < gd + WSL);
      worked = true;
    }
    if constexpr (!FWD) {
      // Plane kd is finished once step npm2 + WSK + shift - kd - 1 is over:
      // with gd groups done, the top 4 gd - WSK - shift planes are.  Each is
      // stored from its ring slot as one 16 x 16 box (clipped at the
      // interior's edges); the slot is handed back (zflushed) once the store
      // has read it.
      const int nc = min(npm2, max(0, WG * gd - WSK - shift));
      if (zd < nc) {
        do {
          const int kd = npm2 - 1 - zd;
          tma_store_3d(map, f.te * WE, f.tj * WJT, kd, &S.zout[kd % WROUT][0]);
          zd++;
        } while (zd < nc);
        bulk_commit();
        bulk_wait_read_all();
        __threadfence_block();
        *(volatile int *)&S.zflushed = zd;
        worked = true;
      }
    }
    if (worked) {
      it = 0;
    } else {
      if (++it > a.spin_limit) {
        *(volatile int *)&S.abort = 1;
        break;
      }
      // the slots it refills are needed two groups (8 steps) later: a long
      // sleep costs nothing there and leaves the issue slots to the compute warps
      __nanosleep(128);
    }
  }
  if (*abort) {  // copies the compute warps may not wait for land before the block moves on
    for (int g = max(0, ns - WSL); g < ns; g++) {
      const int gg = gbase + g;
      mbar_wait(&S.bar_s[gg % WSL], (uint32_t)(gg / WSL) & 1u, WAVE_MBAR_LIMIT);
    }
  }
  if constexpr (!FWD) bulk_wait_all();  // the tile's z32 planes are in global memory
}

template <bool FWD, bool FUSE = false>
__device__ __forceinline__ bool wave_tile(const WaveArgs &a,
                                          typename WaveSmemSel<FWD>::type &S, const WaveFaces &f, unsigned epoch,
                                          int gbase, int qbase) {
  const Geo &g = a.g;
  const int T = threadIdx.x;
  const int te = f.te, tj = f.tj, ti = f.ti;
  const int el = T & (WE - 1), jl = T / WE;
  const int e = te * WE + el, jj = tj * WJT + jl;
  const bool valid = e < g.nrm2 && jj < g.ntm2;
  const int sk = FWD ? el + jl : (WE - 1 - el) + (WJT - 1 - jl);
  const int npm2 = g.npm2;
  const long long row = (long long)(valid ? jj : 0) * g.NRP + (valid ? e : 0);
  const int nsteps = a.nsteps;          // a multiple of WCH
  const int shift = FWD ? 0 : a.pad;    // backward: leading idle steps, so its y groups align
  const int G = nsteps / WG;            // stream groups
  const int te_out = FWD ? te + 1 : te - 1, tj_out = FWD ? tj + 1 : tj - 1;
  const bool pub_e = valid && (FWD ? el == WE - 1 : el == 0) && te_out >= 0 && te_out < a.nte;
  const bool pub_j = valid && (FWD ? jl == WJT - 1 : jl == 0) && tj_out >= 0 && tj_out < a.ntj;
  const bool ext_e = FWD ? el == 0 : el == WE - 1;    // e-neighbour across the face
  const bool ext_j = FWD ? jl == 0 : jl == WJT - 1;   // j-neighbour across the face
  const bool cpl_e = valid && (FWD ? e > 0 : e < g.nrm2 - 1);
  const bool cpl_j = valid && (FWD ? jj > 0 : jj < g.ntm2 - 1);
  unsigned long long *xe_out = a.xe + (size_t)ti * a.ndiag * 16 + jl - (size_t)(WE - 1) * 16;
  unsigned long long *xj_out = a.xj + (size_t)ti * a.ndiag * 16 + el - (size_t)(WJT - 1) * 16;
  const float seam_c = valid ? (FWD ? a.seam_f[row] : a.seam_b[row]) : 0.f;
  const int nch = nsteps / WCH;
  const int ring_e = (0 * WCH) * 16 + jl, ring_j = (1 * WCH) * 16 + el;
  const int y_e = ext_e ? 0 : jl * (WE + 1) + (FWD ? el - 1 : el + 1);
  const int y_j = ext_j ? 0 : (FWD ? jl - 1 : jl + 1) * (WE + 1) + el;

  // The copy warp issues the bulk copies; the mbarrier of a slot counts its
  // uses over the block's tiles (gbase) for the wait parity.
  const volatile int *abort = &S.abort;
  auto wait_s = [&](int gi) {
    const int gg = gbase + gi;
    return wave_mbar_wait(&S.bar_s[gg % WSL], (uint32_t)(gg / WSL) & 1u, abort);
  };

  float seam_y = 0.f;  // value at the line's first plane of the sweep
  float prev = 0.f;    // own value at the previous step
  // Fused forward: the box ring holds q32, and the residual half of the
  // inner update, r32 = r32 - alpha q rounded once, is formed from the
  // streamed r32 of the step (the operations of the unfused update, so the
  // values are the same) at the start of each step group, off the steps'
  // dependent chain, and written back to the stream.  Fused backward:
  // rho = r.z of the stored r32 and the z32 it computes, accumulated in FP64
  // (the r.z update's sum in another order); the thread reads its r32 from
  // the residual stream, which is in the forward's step order like the y
  // stream, one group ahead of use with a plain coalesced load (its latency
  // off the steps' chain, no shared memory).
  double alpha = 0.0;
  if constexpr (FUSE && FWD) alpha = *(const volatile double *)&a.st->alpha;
  double rz = 0.0;
  float4 r_cur = make_float4(0.f, 0.f, 0.f, 0.f), r_next = r_cur;
  if constexpr (FUSE && !FWD) r_next = a.rs[((size_t)ti * G + (G - 1)) * WAVE_THREADS + T];
  // forward: plane p = t - sk of this line sits in slot (qbase + p / WG) % WPG,
  // row p % WG (p < 0 at the first steps: the entry is never read); the slots
  // are consecutive in shared memory, so the plane's place is one index
  // p_lin = slot * WG + row into a ring of WPG * WG planes
  constexpr int NPL = WPG * WG;
  const float *rin_line = nullptr;  // + p_lin * WJT * WE
  int p_lin = 0;
  if constexpr (FWD) {
    rin_line = &S.rin[0][0][jl][el];
    const int p0 = -sk;  // plane at step 0
    const int pg = (p0 - (WG - 1)) / WG;  // floor(p0 / WG) for p0 <= 0
    p_lin = (((qbase + pg) % WPG + WPG) % WPG) * WG + (p0 - pg * WG);
  }
#pragma unroll 1
  for (int c = 0; c < nch; c++) {
    const float *ring = &S.ring[c % WXR][0][0][0];
#pragma unroll
    for (int h = 0; h < WCH / WG; h++) {
      const int gi = c * (WCH / WG) + h;
      {  // wait until the exchange warp has step group gi in the ring
        unsigned it = 0;
        while (*(volatile int *)&S.ready <= gi && !*(volatile int *)&S.abort) {
          if (++it > a.spin_limit) {
            S.abort = 1;
            break;
          }
          if (it > 4) __nanosleep(32);
        }
        __threadfence_block();
      }
      // the barrier that ended group gi-1 (which also decided, uniformly,
      // that no thread had aborted) released its slots: tell the copy warp,
      // which refills them
      if (T == 0) {
        __threadfence_block();
        *(volatile int *)&S.gdone = gi;
      }
      if (!wait_s(gi)) S.abort = 1;  // acted on at the next chunk
      if constexpr (!FWD) {
        // this group writes planes down to npm2 - WG (gi + 1) + shift; the
        // slot of each held the plane WROUT above it, which the copy warp
        // must have stored first
        const int need = WG * gi + WG - shift - WROUT;
        unsigned it = 0;
        while (*(volatile int *)&S.zflushed < need && !*(volatile int *)&S.abort) {
          if (++it > a.spin_limit) {
            S.abort = 1;
            break;
          }
          __nanosleep(20);
        }
      }
      const int sl = (gbase + gi) % WSL;
      float4 c0, c1, c2, c3 = make_float4(0.f, 0.f, 0.f, 0.f), yin4 = c3;
      if constexpr (FWD) {
        c0 = S.lf[sl][0][T];
        c1 = S.lf[sl][1][T];
        c2 = S.lf[sl][2][T];
        if constexpr (FUSE) c3 = S.lf[sl][3][T];  // the group's residual r32
      } else {
        c0 = S.ub[sl][0][T];
        c1 = S.ub[sl][1][T];
        c2 = S.ub[sl][2][T];
        c3 = S.ub[sl][3][T];
        yin4 = S.yin[sl][T];
      }
      if constexpr (FUSE && !FWD) {  // this group's residuals; the next group's load is issued
        r_cur = r_next;
        if (gi + 1 < G) r_next = a.rs[((size_t)ti * G + (G - 2 - gi)) * WAVE_THREADS + T];
      }
      float y4[WG], rn4[WG], vin4[WG];
      if constexpr (FWD && FUSE) {
        // every plane of the group's steps arrived with group gi's copies
#pragma unroll
        for (int u = 0; u < WG; u++) {
          const int pl = p_lin + u < NPL ? p_lin + u : p_lin + u - NPL;
          const float qv = rin_line[pl * (WJT * WE)];
          const float ro = u == 0 ? c3.x : u == 1 ? c3.y : u == 2 ? c3.z : c3.w;
          vin4[u] = (float)fma(-alpha, (double)qv, (double)ro);  // r32 - alpha q
        }
        p_lin = p_lin + WG < NPL ? p_lin + WG : p_lin + WG - NPL;
      }
      // The group's steps, in two compiled forms.  INNER: every thread's
      // plane is strictly inside its line at all four steps (neither the
      // first nor the last plane of the sweep, where the seam coupling and
      // the seam value live, and no idle step), so the seam term, its
      // coefficient select and the per-step activity test drop out; the
      // remaining terms keep lusol's order (the dropped term subtracted an
      // exact zero, so values are unchanged up to the sign of an exact-zero
      // result).  Most groups of a sweep are inner.
      auto steps = [&](auto inner_tag) -> bool {
        constexpr bool INNER = decltype(inner_tag)::value;
        bool aborted = false;
        // backward, inner: plane kk of step u sits in zout slot kk % WROUT, counted down from the group's first
        int zs0 = 0;
        if constexpr (!FWD && INNER) zs0 = (npm2 - 1 - (gi * WG - shift - sk)) % WROUT;
#pragma unroll
        for (int u = 0; u < WG; u++) {
          const int t = gi * WG + u;
          const int uc = h * WG + u;  // step within the chunk
          const float *yprev = &S.y[(t + 1) & 1][0][0];  // values of step t-1
          const float k0 = u == 0 ? c0.x : u == 1 ? c0.y : u == 2 ? c0.z : c0.w;
          const float k1 = u == 0 ? c1.x : u == 1 ? c1.y : u == 2 ? c1.z : c1.w;
          const float k2 = u == 0 ? c2.x : u == 1 ? c2.y : u == 2 ? c2.z : c2.w;
          const float k3 = u == 0 ? c3.x : u == 1 ? c3.y : u == 2 ? c3.z : c3.w;
          // backward y: forward step nsteps-1-t, component 3-u of the group
          float v_in = u == 0 ? yin4.w : u == 1 ? yin4.z : u == 2 ? yin4.y : yin4.x;
          if constexpr (FWD && FUSE) {
            v_in = vin4[u];
          } else if constexpr (FWD) {
            v_in = rin_line[p_lin * (WJT * WE)];
            p_lin = p_lin + 1 < NPL ? p_lin + 1 : 0;
          }
          // Branch-free step: a coupling the point does not have is applied as
          // the product of a zero coefficient (the streams hold zeros there) and
          // a finite operand (the neighbour value is zeroed by a select), which
          // subtracts an exact zero; the terms keep lusol's order, so the
          // values are lusol's (an exact-zero result may differ in its sign
          // only).  With no branches the scheduler overlaps the point's own
          // terms with the neighbour loads that follow the barrier.
          const int q = t - shift - sk;
          const bool act = INNER ? valid : valid && (unsigned)q < (unsigned)npm2;
          const int kk = FWD ? q : npm2 - 1 - q;
          const float *pe = ext_e ? ring + ring_e + uc * 16 : yprev + y_e;
          const float *pj = ext_j ? ring + ring_j + uc * 16 : yprev + y_j;
          const float ne = cpl_e ? *pe : 0.f;
          const float nj = cpl_j ? *pj : 0.f;
          float y;
          if constexpr (FWD) {
            // y = r - [seam] - l_k y(k-1) - l_j y(j-1) - l_e y(e-1); l_k = 0 on the first plane
            if constexpr (INNER) {
              y = __fsub_rn(v_in, __fmul_rn(k0, prev));
            } else {
              const float ks = kk == npm2 - 1 ? seam_c : 0.f;
              y = __fsub_rn(__fsub_rn(v_in, __fmul_rn(ks, seam_y)), __fmul_rn(k0, prev));
            }
            y = __fsub_rn(y, __fmul_rn(k1, nj));
            y = __fsub_rn(y, __fmul_rn(k2, ne));
            y = act ? y : 0.f;
            if constexpr (!INNER) seam_y = (act && kk == 0) ? y : seam_y;
            rn4[u] = act ? v_in : 0.f;
          } else {
            // z = (y - u_e z(e+1) - u_j z(j+1) - u_k z(k+1) - [seam]) * dinv; u_k = 0 on the last plane
            y = __fsub_rn(v_in, __fmul_rn(k0, ne));
            y = __fsub_rn(y, __fmul_rn(k1, nj));
            y = __fsub_rn(y, __fmul_rn(k2, prev));
            if constexpr (!INNER) {
              const float ks = kk == 0 ? seam_c : 0.f;
              y = __fsub_rn(y, __fmul_rn(ks, seam_y));
            }
            y = __fmul_rn(y, k3);
            y = act ? y : 0.f;
            if constexpr (!INNER) seam_y = (act && kk == npm2 - 1) ? y : seam_y;
            if constexpr (INNER) {
              const int zs = zs0 - u >= 0 ? zs0 - u : zs0 - u + WROUT;
              if (act) S.zout[zs][T] = y;
            } else {
              if (act) S.zout[kk % WROUT][T] = y;
            }
            if constexpr (FUSE) {
              // the point's r32 (forward step nsteps-1-t, component 3-u, as
              // for y); r and z are exact zeros where the thread has no point
              const float rr = u == 0 ? r_cur.w : u == 1 ? r_cur.z : u == 2 ? r_cur.y : r_cur.x;
              rz = fma((double)rr, (double)y, rz);
            }
          }
          S.y[t & 1][jl][el] = y;
          if (pub_e && act) wave_publish(xe_out + (size_t)t * 16, epoch, y);
          if (pub_j && act) wave_publish(xj_out + (size_t)t * 16, epoch, y);
          prev = INNER ? y : act ? y : prev;  // inner: y is already 0 where the thread has no point
          y4[u] = y;
          // backward: the group's z32 plane writes become visible to the copy
          // warp's TMA stores (async proxy) across the barrier and gdone
          if (!FWD && u == WG - 1) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          if (u == WG - 1) {
            // the group's last barrier also ORs the abort flag, so every compute
            // warp leaves at the same group when any wait gave up
            aborted = wave_bar_compute_any(*(volatile int *)&S.abort != 0);
          } else {
            wave_bar_compute();
          }
        }
        return aborted;
      };
      // inner: 1 <= q <= npm2 - 2 for every thread (0 <= sk <= WSK) at every step of the group
      const bool inner = WG * gi >= shift + WSK + 1 && WG * gi + (WG - 1) <= shift + npm2 - 2;
      if (inner ? steps(std::true_type{}) : steps(std::false_type{})) return false;
      if constexpr (FWD) a.ys[((size_t)ti * G + gi) * WAVE_THREADS + T] = make_float4(y4[0], y4[1], y4[2], y4[3]);
      if constexpr (FWD && FUSE)
        a.rs[((size_t)ti * G + gi) * WAVE_THREADS + T] = make_float4(rn4[0], rn4[1], rn4[2], rn4[3]);
    }
    if (T == 0) *(volatile int *)&S.consumed = c + 1;
  }
  if (T == 0) {  // every group is done: the copy warp stores the last planes
    __threadfence_block();
    *(volatile int *)&S.gdone = G;
  }
  if constexpr (FUSE && !FWD) {  // the tile's rho partial, in a fixed order
    const double w = warp_sum(rz);
    if ((T & 31) == 0) S.red[T >> 5] = w;
    wave_bar_compute();
    if (T == 0) {
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < WAVE_THREADS / 32; q++) t += S.red[q];
      a.rz_part[ti] = t;
    }
  }
  return true;
}

// map: forward, the r32 load map (FUSE: q32); backward, the z32 store map.
// FUSE: the forms of the FP32-inner iteration of the refined mode (see
// wave_tile); the backward's last block then ends the iteration as the r.z
// update would: the tiles' partials summed in tile order, rho, beta, ncg and
// ernorm (rz_epilogue).
template <bool FWD, bool FUSE = false>
__global__ void __launch_bounds__(WAVE_BLOCK, 2) k_dilu_wave(const __grid_constant__ CUtensorMap map,
                                                                    WaveArgs a) {
  using Sm = typename WaveSmemSel<FWD>::type;
  extern __shared__ unsigned char wave_dyn[];
  Sm &S = *reinterpret_cast<Sm *>(wave_dyn + ((128 - (smem_u32(wave_dyn) & 127)) & 127));
  const int role = threadIdx.x < WAVE_THREADS ? 0 : (threadIdx.x < WAVE_THREADS + 32 ? 1 : 2);  // compute, exchange, copy
  if (threadIdx.x == 0) {
    for (int q = 0; q < WSL; q++) mbar_init(&S.bar_s[q], 1);
    mbar_init_fence();
    tma_prefetch_desc(&map);
  }
  __syncthreads();
  const unsigned epoch = *(volatile unsigned *)&a.ctl->epoch;
  const bool run = !(a.check && *(volatile int *)&a.st->status != ST_RUNNING);
  const int G = a.nsteps / WG, NQ = (a.g.npm2 + WG - 1) / WG;
  int gbase = 0, qbase = 0;  // bulk-copy groups of earlier tiles of this block
  while (run) {
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(&a.ctl->ticket, 1u);
      S.tile = (t < (unsigned)a.ntiles && (int)t != a.stall_ticket) ? a.order[FWD ? t : a.ntiles - 1 - t]
                                                                    : make_int2(-1, -1);
      S.abort = 0;
      S.ready = 0;
      S.consumed = 0;
      S.gdone = 0;
      S.zflushed = 0;
    }
    __syncthreads();
    const int2 tile = S.tile;
    if (tile.x < 0) break;
    const WaveFaces f = wave_faces<FWD>(a, tile.x, tile.y);
    bool ok = true;
    if (role == 1)
      wave_exchange<FWD>(a, S, f, epoch, a.nsteps / WCH);
    else if (role == 2)
      wave_copy<FWD, FUSE>(a, &map, S, f, gbase, qbase, false);
    else
      ok = wave_tile<FWD, FUSE>(a, S, f, epoch, gbase, qbase);
    if (!ok) S.abort = 1;
    __syncthreads();
    if (S.abort) {
      if (threadIdx.x == 0) {
        atomicExch(&a.ctl->error, 1);
        if (a.st) atomicExch(&a.st->status, ST_TIMEOUT);
      }
      break;
    }
    gbase += G;
    qbase += FWD ? NQ : 0;
  }
  __syncthreads();
  __shared__ int last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&a.ctl->done, 1u) == gridDim.x - 1;
    if (last) {  // last block: reset for the next sweep
      atomicExch(&a.ctl->ticket, 0u);
      atomicExch(&a.ctl->done, 0u);
      __threadfence();
      atomicAdd(&a.ctl->epoch, 1u);
    }
  }
  if constexpr (FUSE && !FWD) {
    __syncthreads();
    // every tile's partial is written (each block fenced before its count);
    // in a solve (check) that is still running, end the iteration
    if (last && run && a.check && threadIdx.x < 32) {
      __threadfence();
      double t = 0.0;
      for (int q = threadIdx.x; q < a.ntiles; q += 32) t += __ldcg(a.rz_part + q);
      t = warp_sum(t);
      if (threadIdx.x == 0 && *(volatile int *)&a.st->status == ST_RUNNING) rz_epilogue<UPD_ZDOT>(a.st, t);
    }
  }
}

// Batched sweeps: the tiles of many independent cases in one persistent
// kernel.  The ticket order interleaves the cases' tiles by wavefront key
// (each case keeps its own topological order), so every case's wavefront
// advances at once and the GPU is filled even where one case's wavefront is
// narrow.  A case is read from a table (its arguments and r32 tensor map,
// the map acquired for the tensormap proxy since it reached global memory by
// a host copy); tiles of a case that is no longer running are skipped.
struct alignas(64) WaveCase {
  CUtensorMap rmap;  // forward: r32 loads
  CUtensorMap zmap;  // backward: z32 stores
  CUtensorMap qmap;  // fused forward: q32 loads
  WaveArgs a;
};

// FUSE: the fused forms of the refined mode's inner iteration (wave_tile);
// a case's backward tile that finds all the case's other tiles finished
// ends the case's iteration as k_dilu_wave's last block does.
template <bool FWD, bool FUSE = false>
__global__ void __launch_bounds__(WAVE_BLOCK, 2)
    k_dilu_wave_batch(const WaveCase *__restrict__ cases, const int4 *__restrict__ order, int total, WaveCtl *ctl) {
  using Sm = typename WaveSmemSel<FWD>::type;
  extern __shared__ unsigned char wave_dyn[];
  Sm &S = *reinterpret_cast<Sm *>(wave_dyn + ((128 - (smem_u32(wave_dyn) & 127)) & 127));
  const int role = threadIdx.x < WAVE_THREADS ? 0 : (threadIdx.x < WAVE_THREADS + 32 ? 1 : 2);  // compute, exchange, copy
  if (threadIdx.x == 0) {
    for (int q = 0; q < WSL; q++) mbar_init(&S.bar_s[q], 1);
    mbar_init_fence();
  }
  __syncthreads();
  const unsigned epoch = *(volatile unsigned *)&ctl->epoch;
  int gbase = 0, qbase = 0;  // bulk-copy groups of earlier tiles of this block
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned t = atomicAdd(&ctl->ticket, 1u);
      int c = -1;
      int2 tl = make_int2(-1, -1);
      if (t < (unsigned)total) {
        const int4 o = order[FWD ? t : total - 1 - t];
        const WaveArgs &ca = cases[o.x].a;
        c = (ca.check && *(volatile int *)&ca.st->status != ST_RUNNING) ? -2 : o.x;  // -2: skip
        tl = make_int2(o.y, o.z);
      }
      S.bcase = c;
      S.tile = tl;
      S.abort = 0;
      S.ready = 0;
      S.consumed = 0;
      S.gdone = 0;
      S.zflushed = 0;
    }
    __syncthreads();
    const int c = S.bcase;
    const int2 tile = S.tile;
    if (tile.x < 0) break;
    if (c < 0) {  // case finished: its tiles are skipped
      __syncthreads();  // every thread has read S.bcase before thread 0 takes the next ticket
      continue;
    }
    const WaveCase &C = cases[c];
    const WaveArgs &a = C.a;
    const WaveFaces f = wave_faces<FWD>(a, tile.x, tile.y);
    bool ok = true;
    if (role == 1)
      wave_exchange<FWD>(a, S, f, epoch, a.nsteps / WCH);
    else if (role == 2)
      wave_copy<FWD, FUSE>(a, FWD ? (FUSE ? &C.qmap : &C.rmap) : &C.zmap, S, f, gbase, qbase, true);
    else
      ok = wave_tile<FWD, FUSE>(a, S, f, epoch, gbase, qbase);
    if (!ok) S.abort = 1;
    __syncthreads();
    if (S.abort) {
      if (threadIdx.x == 0) {
        atomicExch(&ctl->error, 1);
        atomicExch(&a.st->status, ST_TIMEOUT);
      }
      break;
    }
    if constexpr (FUSE && !FWD) {
      // the tile's partial is written (thread 0); the case's last tile ends
      // the case's iteration
      __shared__ int case_last;
      if (threadIdx.x == 0) {
        __threadfence();
        case_last = atomicAdd(a.tile_done, 1u) == (unsigned)a.ntiles - 1;
      }
      __syncthreads();
      if (case_last && threadIdx.x < 32) {
        __threadfence();
        double t = 0.0;
        for (int q = threadIdx.x; q < a.ntiles; q += 32) t += __ldcg(a.rz_part + q);
        t = warp_sum(t);
        if (threadIdx.x == 0) {
          if (*(volatile int *)&a.st->status == ST_RUNNING) rz_epilogue<UPD_ZDOT>(a.st, t);
          *a.tile_done = 0u;
        }
      }
    }
    gbase += a.nsteps / WG;
    qbase += FWD ? (a.g.npm2 + WG - 1) / WG : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->done, 1u) == gridDim.x - 1) {  // last block: reset for the next sweep
      atomicExch(&ctl->ticket, 0u);
      atomicExch(&ctl->done, 0u);
      __threadfence();
      atomicAdd(&ctl->epoch, 1u);
    }
  }
}

// Coefficient streams of the sweeps in the tile-skewed group layout, formed
// once from the factor with the reference's operations (Row7 operand order,
// FP32 division by the pivot); zero where a thread has no point at a step.
__global__ void k_wave_streams(Geo g, DevMesh m, const float *__restrict__ d, const float *__restrict__ dinv,
                               int nte, int ntiles, int nsteps, int pad, float4 *__restrict__ lf,
                               float4 *__restrict__ ub) {
  const int G = nsteps / WG;
  const long long total = (long long)ntiles * G * WAVE_THREADS;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int T = (int)(q % WAVE_THREADS);
    const long long rr = q / WAVE_THREADS;
    const int gi = (int)(rr % G);
    const int ti = (int)(rr / G);
    const int te = ti % nte, tj = ti / nte;
    const int el = T & (WE - 1), jl = T / WE;
    const int e = te * WE + el, jj = tj * WJT + jl;
    const bool valid = e < g.nrm2 && jj < g.ntm2;
    float l[3][WG] = {}, u[4][WG] = {};
    for (int s = 0; s < WG; s++) {
      const int t = gi * WG + s;
      const int kf = t - (el + jl);
      if (valid && kf >= 0 && kf < g.npm2) {  // forward point (e, jj, kf)
        const Row7 c = row7(m, e + 2, jj + 2, kf + 2);
        if (kf > 0) l[0][s] = __fdiv_rn((float)c.a1, d[g.idx(e, jj, kf - 1)]);
        if (jj > 0) l[1][s] = __fdiv_rn((float)c.a2, d[g.idx(e, jj - 1, kf)]);
        if (e > 0) l[2][s] = __fdiv_rn((float)c.a3, d[g.idx(e - 1, jj, kf)]);
      }
      const int qb = t - pad - ((WE - 1 - el) + (WJT - 1 - jl));
      if (valid && qb >= 0 && qb < g.npm2) {  // backward point (e, jj, npm2-1-qb)
        const int kb = g.npm2 - 1 - qb;
        const Row7 c = row7(m, e + 2, jj + 2, kb + 2);
        u[0][s] = e < g.nrm2 - 1 ? (float)c.a5 : 0.f;
        u[1][s] = jj < g.ntm2 - 1 ? (float)c.a6 : 0.f;
        u[2][s] = kb < g.npm2 - 1 ? (float)c.a7 : 0.f;
        u[3][s] = dinv[g.idx(e, jj, kb)];
      }
    }
    const size_t base = (size_t)ti * G + gi;
    for (int c = 0; c < 3; c++) lf[(base * 3 + c) * WAVE_THREADS + T] = make_float4(l[c][0], l[c][1], l[c][2], l[c][3]);
    for (int c = 0; c < 4; c++) ub[(base * 4 + c) * WAVE_THREADS + T] = make_float4(u[c][0], u[c][1], u[c][2], u[c][3]);
  }
}

// The same streams from a factored 1-based CSR with POT3D's 7-point pattern
// (the route of load_external_lu_solver for such a matrix): each row's L
// entries as ilu0 left them (a_ik / d_k) and its upper entries, found by
// their column offsets, and dinv; zero where a thread has no point at a step
// or the row has no such coupling.  The values are the ones k_wave_streams
// forms from the mesh, since the CSR holds the same FP32 coefficients.
__global__ void k_wave_streams_csr(Geo g, const int *__restrict__ ia, const int *__restrict__ ja,
                                   const int *__restrict__ dptr, const float *__restrict__ a,
                                   const float *__restrict__ dinv, int nte, int ntiles, int nsteps, int pad,
                                   float4 *__restrict__ lf, float4 *__restrict__ ub) {
  const int G = nsteps / WG;
  const long long P = (long long)g.nrm2 * g.ntm2;
  const long long total = (long long)ntiles * G * WAVE_THREADS;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int T = (int)(q % WAVE_THREADS);
    const long long rr = q / WAVE_THREADS;
    const int gi = (int)(rr % G);
    const int ti = (int)(rr / G);
    const int te = ti % nte, tj = ti / nte;
    const int el = T & (WE - 1), jl = T / WE;
    const int e = te * WE + el, jj = tj * WJT + jl;
    const bool valid = e < g.nrm2 && jj < g.ntm2;
    float l[3][WG] = {}, u[4][WG] = {};
    for (int s = 0; s < WG; s++) {
      const int t = gi * WG + s;
      const int kf = t - (el + jl);
      if (valid && kf >= 0 && kf < g.npm2) {  // forward row (e, jj, kf)
        const long long i = ((long long)kf * g.ntm2 + jj) * g.nrm2 + e;
        for (int k = ia[i] - 1; k < dptr[i]; k++) {
          const long long c = ja[k] - 1;
          if (c == i - P) l[0][s] = a[k];
          else if (c == i - g.nrm2) l[1][s] = a[k];
          else if (c == i - 1) l[2][s] = a[k];
        }
      }
      const int qb = t - pad - ((WE - 1 - el) + (WJT - 1 - jl));
      if (valid && qb >= 0 && qb < g.npm2) {  // backward row (e, jj, npm2-1-qb)
        const int kb = g.npm2 - 1 - qb;
        const long long i = ((long long)kb * g.ntm2 + jj) * g.nrm2 + e;
        for (int k = dptr[i] + 1; k < ia[i + 1] - 1; k++) {
          const long long c = ja[k] - 1;
          if (c == i + 1) u[0][s] = a[k];
          else if (c == i + g.nrm2) u[1][s] = a[k];
          else if (c == i + P) u[2][s] = a[k];
        }
        u[3][s] = dinv[i];
      }
    }
    const size_t base = (size_t)ti * G + gi;
    for (int c = 0; c < 3; c++) lf[(base * 3 + c) * WAVE_THREADS + T] = make_float4(l[c][0], l[c][1], l[c][2], l[c][3]);
    for (int c = 0; c < 4; c++) ub[(base * 4 + c) * WAVE_THREADS + T] = make_float4(u[c][0], u[c][1], u[c][2], u[c][3]);
  }
}

// Seam couplings from the CSR: the last plane's L entry to the first plane
// (its smallest column) and the first plane's U entry to the last (largest).
__global__ void k_wave_seam_csr(Geo g, const int *__restrict__ ia, const int *__restrict__ ja,
                                const int *__restrict__ dptr, const float *__restrict__ a, float *__restrict__ seam_f,
                                float *__restrict__ seam_b) {
  const long long n = (long long)g.ntm2 * g.nrm2, P = n, W = (long long)(g.npm2 - 1) * P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q % g.nrm2), jj = (int)(q / g.nrm2);
    const long long row = (long long)jj * g.NRP + e;
    const long long il = W + q, i0 = q;  // the line's last and first plane rows
    float sf = 0.f, sb = 0.f;
    for (int k = ia[il] - 1; k < dptr[il]; k++)
      if (ja[k] - 1 == il - W) sf = a[k];
    for (int k = dptr[i0] + 1; k < ia[i0 + 1] - 1; k++)
      if (ja[k] - 1 == i0 + W) sb = a[k];
    seam_f[row] = sf;
    seam_b[row] = sb;
  }
}

// Per-line seam coefficients: forward a7/d(e, j, 0) of the last plane,
// backward a1 of the first plane.
__global__ void k_wave_seam(Geo g, DevMesh m, const float *__restrict__ d, float *__restrict__ seam_f,
                            float *__restrict__ seam_b) {
  const long long n = (long long)g.ntm2 * g.nrm2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q % g.nrm2), jj = (int)(q / g.nrm2);
    const long long row = (long long)jj * g.NRP + e;
    const Row7 cl = row7(m, e + 2, jj + 2, g.npm2 - 1 + 2);
    seam_f[row] = __fdiv_rn((float)cl.a7, d[g.idx(e, jj, 0)]);
    const Row7 cf = row7(m, e + 2, jj + 2, 2);
    seam_b[row] = (float)cf.a1;
  }
}

// r32 (padded layout) into the fused forward's residual stream, in the
// tile-skewed group layout of the coefficient streams; zero where a thread
// has no point at a step.
__global__ void k_wave_r_stream(Geo g, const float *__restrict__ r32, int nte, int ntiles, int nsteps,
                                float4 *__restrict__ rs) {
  const int G = nsteps / WG;
  const long long total = (long long)ntiles * G * WAVE_THREADS;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int T = (int)(q % WAVE_THREADS);
    const long long rr = q / WAVE_THREADS;
    const int gi = (int)(rr % G);
    const int ti = (int)(rr / G);
    const int te = ti % nte, tj = ti / nte;
    const int el = T & (WE - 1), jl = T / WE;
    const int e = te * WE + el, jj = tj * WJT + jl;
    const bool valid = e < g.nrm2 && jj < g.ntm2;
    float v[WG];
#pragma unroll
    for (int s = 0; s < WG; s++) {
      const int kf = gi * WG + s - (el + jl);
      v[s] = (valid && kf >= 0 && kf < g.npm2) ? r32[g.idx(e, jj, kf)] : 0.f;
    }
    rs[q] = make_float4(v[0], v[1], v[2], v[3]);
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
  float4 *lf = nullptr, *ub = nullptr, *ys = nullptr;  // tile-skewed group streams
  float4 *rs = nullptr;      // refined mode: the inner iterations' r32 in the stream layout
  double *rz_part = nullptr; // refined mode: per-tile rho partials of the fused backward
  float *qmap_ptr = nullptr; // the q32 vector qmap describes
  CUtensorMap qmap;          // q32 in 16 x 16 x 4 boxes (fused forward loads)
  float *seam_f = nullptr, *seam_b = nullptr;
  int2 *order = nullptr;
  WaveCtl *ctl = nullptr;
  CUtensorMap rmap;  // r32 in 16 x 16 x 4 boxes (forward loads)
  CUtensorMap zmap;  // z32 interior in 16 x 16 x 1 boxes (backward stores)
  int nte = 0, ntj = 0, ntiles = 0, ndiag = 0, nsteps = 0, wave_blocks = 0;
  size_t wave_smem_f = 0, wave_smem_b = 0;
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

// Exchange buffers, streams, tile order and launch shape of the sweeps.
static int wave_setup(Solver *s) {
  DiluState *D = s->dilu;
  const Geo &g = s->g;
  D->nte = (g.nrm2 + WE - 1) / WE;
  D->ntj = (g.ntm2 + WJT - 1) / WJT;
  D->ntiles = D->nte * D->ntj;
  D->nsteps = (g.npm2 + WSK + WCH - 1) / WCH * WCH;  // whole chunks (and stream groups)
  D->ndiag = D->nsteps - (WSK / 2 - 1);               // consumer steps that receive face words
  const size_t nx = (size_t)D->ntiles * D->ndiag * 16;
  const size_t ng = (size_t)D->ntiles * (D->nsteps / WG) * WAVE_THREADS;  // float4 per stream component
  int st;
  if ((st = s->alloc((void **)&D->xe, 8 * nx)) || (st = s->alloc((void **)&D->xj, 8 * nx)) ||
      (st = s->alloc((void **)&D->order, sizeof(int2) * D->ntiles)) ||
      (st = s->alloc((void **)&D->lf, sizeof(float4) * 3 * ng)) || (st = s->alloc((void **)&D->ys, sizeof(float4) * ng)) ||
      (st = s->alloc((void **)&D->ub, sizeof(float4) * 4 * ng)) ||
      (st = s->alloc((void **)&D->seam_f, sizeof(float) * (size_t)g.ntm2 * g.NRP)) ||
      (st = s->alloc((void **)&D->seam_b, sizeof(float) * (size_t)g.ntm2 * g.NRP)) ||
      (st = s->alloc((void **)&D->ctl, sizeof(WaveCtl))))
    return st;
  if (s->precision == POT3D_FP32_REFINED &&
      ((st = s->alloc((void **)&D->rs, sizeof(float4) * ng)) ||
       (st = s->alloc((void **)&D->rz_part, sizeof(double) * D->ntiles))))
    return st;
  if ((st = encode_padded_map(g, D->r32, false, WE, WJT, WG, &D->rmap))) return st;
  if ((st = encode_padded_map(g, D->z32, false, WE, WJT, 1, &D->zmap, true))) return st;
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
  CK(cudaMemsetAsync(D->seam_f, 0, sizeof(float) * (size_t)g.ntm2 * g.NRP, s->stream));
  CK(cudaMemsetAsync(D->seam_b, 0, sizeof(float) * (size_t)g.ntm2 * g.NRP, s->stream));
  const WaveCtl c0{0u, 0u, 1u, 0};  // tag 0 is the zeroed buffers': sweeps start at 1
  CK(cudaMemcpyAsync(D->ctl, &c0, sizeof(WaveCtl), cudaMemcpyHostToDevice, s->stream));
  D->wave_smem_f = sizeof(WaveSmemF) + 128;  // + alignment slack of the dynamic base
  D->wave_smem_b = sizeof(WaveSmemB) + 128;
  CK(cudaFuncSetAttribute(k_dilu_wave<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem_f));
  CK(cudaFuncSetAttribute(k_dilu_wave<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D->wave_smem_b));
  CK(cudaFuncSetAttribute(k_dilu_wave<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)D->wave_smem_f));
  CK(cudaFuncSetAttribute(k_dilu_wave<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)D->wave_smem_b));
  int dev = 0, nsm = 0, occ_f = 0, occ_b = 0, occ_ff = 0, occ_fb = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_dilu_wave<true>, WAVE_BLOCK, D->wave_smem_f));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_dilu_wave<false>, WAVE_BLOCK, D->wave_smem_b));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ff, k_dilu_wave<true, true>, WAVE_BLOCK, D->wave_smem_f));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_fb, k_dilu_wave<false, true>, WAVE_BLOCK, D->wave_smem_b));
  const int occ = std::min(std::min(occ_f, occ_b), std::min(occ_ff, occ_fb));
  D->wave_blocks = std::max(1, std::min(std::max(1, occ) * nsm, D->ntiles));
  return POT3D_OK;
}

static WaveArgs wave_args(Solver *s, bool check) {
  DiluState *D = s->dilu;
  WaveArgs a{};
  a.g = s->g;
  a.z32 = D->z32;
  a.ys = D->ys;
  a.lf = D->lf;
  a.ub = D->ub;
  a.seam_f = D->seam_f;
  a.seam_b = D->seam_b;
  a.xe = D->xe;
  a.xj = D->xj;
  a.order = D->order;
  a.ctl = D->ctl;
  a.st = s->d_state;
  a.check = check ? 1 : 0;
  a.spin_limit = WAVE_SPIN_LIMIT;
  a.stall_ticket = -1;
  a.nte = D->nte;
  a.ntj = D->ntj;
  a.ntiles = D->ntiles;
  a.ndiag = D->ndiag;
  a.nsteps = D->nsteps;
  a.pad = D->nsteps - (s->g.npm2 + WSK);
  return a;
}

static void launch_wave(Solver *s, bool fwd, bool check) {
  DiluState *D = s->dilu;
  const WaveArgs a = wave_args(s, check);
  if (fwd)
    k_dilu_wave<true><<<D->wave_blocks, WAVE_BLOCK, D->wave_smem_f, s->stream>>>(D->rmap, a);
  else
    k_dilu_wave<false><<<D->wave_blocks, WAVE_BLOCK, D->wave_smem_b, s->stream>>>(D->zmap, a);
}

// ---- batched sweeps over many cases -------------------------------------
struct DiluBatch {
  WaveCase *d_cases = nullptr;
  int4 *d_order = nullptr;
  WaveCtl *ctl = nullptr;
  unsigned *tile_done = nullptr;  // fused: per case, its backward tiles finished in this sweep
  int n = 0, total = 0, blocks = 0;
  bool fused = false;             // every case in the refined mode: the fused sweeps
  size_t smem_f = 0, smem_b = 0;
};

void dilu_batch_destroy(DiluBatch *B) {
  if (!B) return;
  if (B->d_cases) cudaFree(B->d_cases);
  if (B->d_order) cudaFree(B->d_order);
  if (B->ctl) cudaFree(B->ctl);
  if (B->tile_done) cudaFree(B->tile_done);
  delete B;
}

static int fused_args(Solver *s, bool check, const float *q32, WaveArgs *out);

int dilu_batch_setup(Solver *const *cases, int n, cudaStream_t stream, DiluBatch **out) {
  *out = nullptr;
  DiluBatch *B = new DiluBatch();
  std::vector<WaveCase> h(n);
  std::vector<int4> ord;
  B->n = n;
  B->fused = true;
  for (int q = 0; q < n; q++) B->fused = B->fused && cases[q]->dilu && cases[q]->dilu->rs;
  if (B->fused &&
      pot3d_cuda_status(cudaMalloc(&B->tile_done, sizeof(unsigned) * n), "cudaMalloc(batch tile counters)")) {
    dilu_batch_destroy(B);
    return POT3D_ERR_CUDA;
  }
  for (int q = 0; q < n; q++) {
    DiluState *D = cases[q]->dilu;
    if (!D) {
      dilu_batch_destroy(B);
      pot3d_set_error("batched ILU(0) sweeps: a case has no ILU(0) factor");
      return POT3D_ERR_ARG;
    }
    h[q].rmap = D->rmap;
    h[q].zmap = D->zmap;
    if (B->fused) {
      int st;
      if ((st = fused_args(cases[q], true, cases[q]->m_q32, &h[q].a))) {
        dilu_batch_destroy(B);
        return st;
      }
      h[q].qmap = D->qmap;
      h[q].a.tile_done = B->tile_done + q;
    } else {
      h[q].a = wave_args(cases[q], true);
    }
    for (int tj = 0; tj < D->ntj; tj++)
      for (int te = 0; te < D->nte; te++) ord.push_back(make_int4(q, te, tj, 0));
  }
  // Every case keeps its producers-first order; the cases' wavefronts interleave.
  std::stable_sort(ord.begin(), ord.end(), [](const int4 &x, const int4 &y) {
    const int kx = WE * x.y + WJT * x.z, ky = WE * y.y + WJT * y.z;
    if (kx != ky) return kx < ky;
    return x.x != y.x ? x.x < y.x : x.y < y.y;
  });
  B->total = (int)ord.size();
  int st;
  auto fail = [&](int code) {
    dilu_batch_destroy(B);
    return code;
  };
  if ((st = pot3d_cuda_status(cudaMalloc(&B->d_cases, sizeof(WaveCase) * n), "cudaMalloc(batch sweep cases)")) ||
      (st = pot3d_cuda_status(cudaMalloc(&B->d_order, sizeof(int4) * ord.size()), "cudaMalloc(batch sweep order)")) ||
      (st = pot3d_cuda_status(cudaMalloc(&B->ctl, sizeof(WaveCtl)), "cudaMalloc(batch sweep control)")))
    return fail(st);
  // Sweep tags of the batch live above 2^31, the cases' own sweeps below it,
  // so the shared exchange buffers never hold a word a later sweep accepts.
  const WaveCtl c0{0u, 0u, 0x80000001u, 0};
  if (B->fused &&
      (st = pot3d_cuda_status(cudaMemsetAsync(B->tile_done, 0, sizeof(unsigned) * n, stream), "batch tile counters")))
    return fail(st);
  if ((st = pot3d_cuda_status(
           cudaMemcpyAsync(B->d_cases, h.data(), sizeof(WaveCase) * n, cudaMemcpyHostToDevice, stream),
           "cudaMemcpy(batch sweep cases)")) ||
      (st = pot3d_cuda_status(
           cudaMemcpyAsync(B->d_order, ord.data(), sizeof(int4) * ord.size(), cudaMemcpyHostToDevice, stream),
           "cudaMemcpy(batch sweep order)")) ||
      (st = pot3d_cuda_status(cudaMemcpyAsync(B->ctl, &c0, sizeof(WaveCtl), cudaMemcpyHostToDevice, stream),
                              "cudaMemcpy(batch sweep control)")) ||
      (st = pot3d_cuda_status(cudaStreamSynchronize(stream), "batch sweep set-up")))
    return fail(st);
  B->smem_f = sizeof(WaveSmemF) + 128;
  B->smem_b = sizeof(WaveSmemB) + 128;
  int dev = 0, nsm = 0, occ_f = 0, occ_b = 0;
  if ((st = pot3d_cuda_status(cudaFuncSetAttribute(k_dilu_wave_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)B->smem_f),
                              "cudaFuncSetAttribute")) ||
      (st = pot3d_cuda_status(cudaFuncSetAttribute(k_dilu_wave_batch<false>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_b),
                              "cudaFuncSetAttribute")) ||
      (st = pot3d_cuda_status(cudaFuncSetAttribute(k_dilu_wave_batch<true, true>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_f),
                              "cudaFuncSetAttribute")) ||
      (st = pot3d_cuda_status(cudaFuncSetAttribute(k_dilu_wave_batch<false, true>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->smem_b),
                              "cudaFuncSetAttribute")) ||
      (st = pot3d_cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) ||
      (st = pot3d_cuda_status(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count")) ||
      (st = pot3d_cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_dilu_wave_batch<true>,
                                                                            WAVE_BLOCK, B->smem_f),
                              "occupancy")) ||
      (st = pot3d_cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_dilu_wave_batch<false>,
                                                                            WAVE_BLOCK, B->smem_b),
                              "occupancy")))
    return fail(st);
  B->blocks = std::max(1, std::min(std::max(1, std::min(occ_f, occ_b)) * nsm, B->total));
  *out = B;
  return POT3D_OK;
}

// The two sweeps of every running case of the batch (z32 = (LU)^-1 r32).
int dilu_batch_sweeps(DiluBatch *B, cudaStream_t stream) {
  k_dilu_wave_batch<true><<<B->blocks, WAVE_BLOCK, B->smem_f, stream>>>(B->d_cases, B->d_order, B->total,
                                                                              B->ctl);
  k_dilu_wave_batch<false><<<B->blocks, WAVE_BLOCK, B->smem_b, stream>>>(B->d_cases, B->d_order, B->total,
                                                                               B->ctl);
  return pot3d_cuda_status(cudaGetLastError(), "batched ILU(0) sweeps");
}

// The fused sweeps of the refined mode's inner iteration for every running
// case (dilu_sweeps_fused per case, with the cases' q32 in their tables).
int dilu_batch_sweeps_fused(DiluBatch *B, cudaStream_t stream) {
  if (!B->fused) {
    pot3d_set_error("fused batched ILU(0) sweeps need every case in the refined mode");
    return POT3D_ERR_ARG;
  }
  k_dilu_wave_batch<true, true><<<B->blocks, WAVE_BLOCK, B->smem_f, stream>>>(B->d_cases, B->d_order, B->total,
                                                                                    B->ctl);
  k_dilu_wave_batch<false, true><<<B->blocks, WAVE_BLOCK, B->smem_b, stream>>>(B->d_cases, B->d_order,
                                                                                     B->total, B->ctl);
  return pot3d_cuda_status(cudaGetLastError(), "fused batched ILU(0) sweeps");
}
bool dilu_batch_fused(const DiluBatch *B) { return B && B->fused; }

// Clear the batch sweeps' ticket counter (and the fused backward's per-case
// tile counters, which a sweep that gave up can leave behind) and advance
// their tag.
int dilu_batch_reset(DiluBatch *B, cudaStream_t stream) {
  k_wave_reset<<<1, 1, 0, stream>>>(B->ctl);
  if (B->fused) CK(cudaMemsetAsync(B->tile_done, 0, sizeof(unsigned) * B->n, stream));
  return pot3d_cuda_status(cudaGetLastError(), "k_wave_reset(batch)");
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
  k_wave_streams<<<148 * 8, NTHR, 0, s->stream>>>(g, s->m, D->d, D->dinv, D->nte, D->ntiles, D->nsteps,
                                                   D->nsteps - (g.npm2 + WSK), D->lf, D->ub);
  k_wave_seam<<<grid1d((long long)g.ntm2 * g.nrm2), NTHR, 0, s->stream>>>(g, s->m, D->d, D->seam_f, D->seam_b);
  return pot3d_cuda_status(cudaGetLastError(), "sweep coefficient streams");
}

// Wavefront sweeps for a caller's factored CSR with the 7-point pattern of a
// nrm2 x ntm2 x npm2 interior (load_external_lu_solver's route): s carries
// only the grid and a stream; the streams come from the CSR (device arrays).
int dilu_setup_csr(Solver *s, const int *ia, const int *ja, const int *dptr, const float *a, const float *dinv) {
  const Geo &g = s->g;
  s->dilu = new DiluState();
  DiluState *D = s->dilu;
  int st;
  const size_t fb = sizeof(float) * (size_t)g.Np;
  if ((st = s->alloc((void **)&D->r32, fb)) || (st = s->alloc((void **)&D->z32, fb))) return st;
  if ((st = wave_setup(s))) return st;
  k_wave_streams_csr<<<148 * 8, NTHR, 0, s->stream>>>(g, ia, ja, dptr, a, dinv, D->nte, D->ntiles, D->nsteps,
                                                      D->nsteps - (g.npm2 + WSK), D->lf, D->ub);
  k_wave_seam_csr<<<grid1d((long long)g.ntm2 * g.nrm2), NTHR, 0, s->stream>>>(g, ia, ja, dptr, a, D->seam_f,
                                                                             D->seam_b);
  return pot3d_cuda_status(cudaGetLastError(), "sweep streams from the CSR");
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

// The residual stream of the fused sweeps from the padded r32 (after the
// refined solve has formed r32 from an FP64 residual).
int dilu_r_stream(Solver *s) {
  DiluState *D = s->dilu;
  if (!D->rs) {
    pot3d_set_error("fused ILU(0) sweeps need a solver in the refined mode");
    return POT3D_ERR_ARG;
  }
  k_wave_r_stream<<<grid1d((long long)D->ntiles * (D->nsteps / WG) * WAVE_THREADS), NTHR, 0, s->stream>>>(
      s->g, D->r32, D->nte, D->ntiles, D->nsteps, D->rs);
  return pot3d_cuda_status(cudaGetLastError(), "k_wave_r_stream");
}

// Arguments of the fused sweeps (and the q32 box map, encoded on the host
// only, so also valid while a stream is being captured).
static int fused_args(Solver *s, bool check, const float *q32, WaveArgs *out) {
  DiluState *D = s->dilu;
  if (!D->rs) {
    pot3d_set_error("fused ILU(0) sweeps need a solver in the refined mode");
    return POT3D_ERR_ARG;
  }
  if (D->qmap_ptr != q32) {
    int st;
    if ((st = encode_padded_map(s->g, q32, false, WE, WJT, WG, &D->qmap))) return st;
    D->qmap_ptr = const_cast<float *>(q32);
  }
  WaveArgs a = wave_args(s, check);
  a.rs = D->rs;
  a.rz_part = D->rz_part;
  *out = a;
  return POT3D_OK;
}
static void launch_wave_fused(Solver *s, bool fwd, const WaveArgs &a) {
  DiluState *D = s->dilu;
  if (fwd)
    k_dilu_wave<true, true><<<D->wave_blocks, WAVE_BLOCK, D->wave_smem_f, s->stream>>>(D->qmap, a);
  else
    k_dilu_wave<false, true><<<D->wave_blocks, WAVE_BLOCK, D->wave_smem_b, s->stream>>>(D->zmap, a);
}

// The sweeps of one FP32-inner iteration of the refined mode: the forward
// applies the inner update's residual half (r32 -= alpha q32, on the
// residual stream) before its recurrence; the backward computes rho = r.z
// (r32 from the residual stream), and its last block ends the iteration
// (rho, beta, ncg, ernorm).
int dilu_sweeps_fused(Solver *s, const float *q32) {
  WaveArgs a;
  int st;
  if ((st = fused_args(s, true, q32, &a))) return st;
  launch_wave_fused(s, true, a);
  launch_wave_fused(s, false, a);
  return pot3d_cuda_status(cudaGetLastError(), "fused ILU(0) sweeps");
}

// Average device time of the forward and of the backward sweep over `reps`
// applications, in the forms the solver iterates with: the plain sweeps on
// the FP32 right-hand side, or, for a solver in the refined mode, the fused
// sweeps (its residual stream from the right-hand side, q32 zero, the
// solve state left alone).
int dilu_time(Solver *s, int reps, double ms[2]) {
  DiluState *D = s->dilu;
  int st;
  if ((st = dilu_reset(s))) return st;
  k_narrow_rhs<<<grid1d(s->g.Np), NTHR, 0, s->stream>>>(s->g.Np, s->d_b, D->r32);
  const bool fused = D->rs != nullptr;
  WaveArgs fa{};
  if (fused) {
    if ((st = dilu_r_stream(s)) || (st = fused_args(s, false, s->m_q32, &fa))) return st;
    CK(cudaMemsetAsync(s->m_q32, 0, sizeof(float) * s->g.Np, s->stream));
  }
  cudaEvent_t e[3];
  for (auto &x : e) CK(cudaEventCreate(&x));
  ms[0] = ms[1] = 0.0;
  for (int it = 0; it < reps; it++) {
    CK(cudaEventRecord(e[0], s->stream));
    if (fused) {
      launch_wave_fused(s, true, fa);
      CK(cudaEventRecord(e[1], s->stream));
      launch_wave_fused(s, false, fa);
    } else {
      launch_wave(s, true, false);
      CK(cudaEventRecord(e[1], s->stream));
      launch_wave(s, false, false);
    }
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

// Failure-detection check: the forward sweep with the block that takes the
// first ticket leaving its tile undone, so no face word of that tile is ever
// published and every wait for one runs out after spin_limit polls.  Returns
// the sweep's status (POT3D_ERR_TIMEOUT when the waits gave up as they must)
// and leaves the sweeps reset for the next solve.
int dilu_test_stall(Solver *s, unsigned spin_limit) {
  DiluState *D = s->dilu;
  int st;
  if ((st = dilu_reset(s))) return st;
  k_narrow_rhs<<<grid1d(s->g.Np), NTHR, 0, s->stream>>>(s->g.Np, s->d_b, D->r32);
  WaveArgs a = wave_args(s, false);
  a.spin_limit = spin_limit;
  a.stall_ticket = 0;
  k_dilu_wave<true><<<D->wave_blocks, WAVE_BLOCK, D->wave_smem_f, s->stream>>>(D->rmap, a);
  if ((st = pot3d_cuda_status(cudaGetLastError(), "stalled sweep"))) return st;
  const int sweep_status = dilu_status(s);
  if ((st = dilu_reset(s))) return st;
  CK(cudaStreamSynchronize(s->stream));
  return sweep_status;
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
