// BF16 GEMM on the fifth-generation tensor cores (tcgen05) of sm_100a, used
// by the learned warm start (the Fourier-style neural operator):
//
//   D[b][m][n] = sum_k A[b][m][k] * B[b][n][k]  (+ bias[n])
//
// A and B are BF16 with K contiguous; accumulation is FP32 in tensor memory
// (TMEM); D is written as FP32 or BF16.  One CTA of 128 threads owns a
// 128 x BN tile: thread 0 streams 128x64 (A) and BNx64 (B) tiles through a
// four-stage shared-memory ring with 3-D TMA loads (128-byte swizzle, no
// multicast) and issues tcgen05.mma (M=128, N=BN, K=16 per instruction)
// whose completion is signalled to mbarriers by tcgen05.commit; all four
// warps then read their 32 TMEM lanes with tcgen05.ld for the epilogue.
// Every wait is bounded; a timeout sets *err and the kernel still drains and
// frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "pot3d_internal.cuh"
#include "tma.cuh"

namespace {

using pot3d::mbar_expect_tx;
using pot3d::mbar_init;
using pot3d::mbar_init_fence;
using pot3d::mbar_wait;
using pot3d::smem_u32;
using pot3d::tma_load_3d;

constexpr int GM = 128;       // rows per CTA tile (UMMA M)
constexpr int GK = 64;        // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int GSTAGES = 4;
constexpr uint32_t GWAIT = 1u << 26;

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// UMMA shared-memory descriptor of a K-major tile written by TMA with the
// 128-byte swizzle: rows of 128 bytes, 8-row atoms 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);  // start address
  d |= (uint64_t)(16 >> 4) << 16;          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset: next 8-row atom
  d |= (uint64_t)1 << 46;                  // descriptor version for sm_100
  d |= (uint64_t)2 << 61;                  // layout: 128-byte swizzle
  return d;
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4)                 // D format F32
         | (1u << 7)               // A format BF16
         | (1u << 10)              // B format BF16
         | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; q++) v[q] = __uint_as_float(r[q]);
}

template <int BN>
struct GemmSmem {
  static constexpr int a_bytes = GM * GK * 2;   // 16 KB
  static constexpr int b_bytes = BN * GK * 2;
  static constexpr int stage = a_bytes + b_bytes;  // multiple of 1024
  static constexpr int total = GSTAGES * stage + 1024;
};

template <int BN, bool OUT_BF16>
__global__ void __launch_bounds__(128, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, void *D,
              const float *__restrict__ bias, int M, int N, int K, long long ldd, long long bstride_d, int accumulate,
              int *err) {
  using S = GemmSmem<BN>;
  extern __shared__ __align__(1024) unsigned char gsm[];
  __shared__ __align__(8) uint64_t full[GSTAGES], empty[GSTAGES], done;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(gsm) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * GM, n0 = blockIdx.y * BN, bz = blockIdx.z;
  const int nk = K / GK;
  constexpr uint32_t ncols = BN < 32 ? 32 : BN;

  if (warp == 0) tmem_alloc(&tmem_base, ncols);
  if (tid == 0) {
    failed = 0;
    for (int s = 0; s < GSTAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    mbar_init_fence();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base;

  if (tid == 0) {
    auto load = [&](int kb) {
      const int s = kb % GSTAGES;
      unsigned char *sa = base + s * S::stage;
      mbar_expect_tx(&full[s], S::stage);
      tma_load_3d(sa, &ta, kb * GK, m0, bz, &full[s]);
      tma_load_3d(sa + S::a_bytes, &tb, kb * GK, n0, bz, &full[s]);
    };
    int issued = 0;
    for (; issued < GSTAGES && issued < nk; issued++) load(issued);
    constexpr uint32_t idesc = idesc_bf16(GM, BN);
    bool ok = true;
    for (int kb = 0; kb < nk && ok; kb++) {
      const int s = kb % GSTAGES;
      if (!mbar_wait(&full[s], (kb / GSTAGES) & 1, GWAIT)) {
        ok = false;
        break;
      }
      fence_after();
      const uint32_t sa = smem_u32(base + s * S::stage);
      const uint64_t da = smem_desc_sw128(sa), db = smem_desc_sw128(sa + S::a_bytes);
#pragma unroll
      for (int kk = 0; kk < GK / 16; kk++)  // 16 BF16 = 32 bytes per instruction
        umma_bf16(tmem, da + 2 * kk, db + 2 * kk, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
      // Refill the stage used one step earlier once its MMAs have read it.
      if (kb >= 1 && issued < nk) {
        const int sp = (kb - 1) % GSTAGES;
        if (!mbar_wait(&empty[sp], ((kb - 1) / GSTAGES) & 1, GWAIT)) {
          ok = false;
          break;
        }
        load(issued);
        issued++;
      }
    }
    if (!ok) {
      failed = 1;
      atomicExch(err, 1);
    }
    umma_commit(&done);  // arrives once every issued MMA has completed
  }
  const bool got = mbar_wait(&done, 0, GWAIT);
  fence_after();
  if (!got && lane == 0) atomicExch(err, 1);
  __syncthreads();
  if (got && !failed) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < M) {
        const long long off = (long long)bz * bstride_d + (long long)row * ldd;
#pragma unroll
        for (int q = 0; q < 32; q++) {
          const int col = n0 + c0 + q;
          if (col < N) {
            float o = v[q] + (bias ? bias[col] : 0.0f);
            if (OUT_BF16) {
              __nv_bfloat16 *d = reinterpret_cast<__nv_bfloat16 *>(D) + off + col;
              if (accumulate) o += __bfloat162float(*d);
              *d = __float2bfloat16_rn(o);
            } else {
              float *d = reinterpret_cast<float *>(D) + off + col;
              if (accumulate) o += *d;
              *d = o;
            }
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  }
  return fn;
}

// 3-D map of a BF16 [batch][rows][K] array, box 64 x box_rows x 1, 128B swizzle.
int map_bf16(CUtensorMap *m, const void *ptr, int batch, int rows, int K, int box_rows) {
  EncodeFn fn = encode();
  if (!fn) {
    pot3d_set_error("cuTensorMapEncodeTiled is not available");
    return POT3D_ERR_CUDA;
  }
  cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)K * 2, (cuuint64_t)K * 2 * rows};
  cuuint32_t box[3] = {(cuuint32_t)GK, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    pot3d_set_error("cuTensorMapEncodeTiled(bf16) failed: " + std::to_string((int)r));
    return POT3D_ERR_CUDA;
  }
  return POT3D_OK;
}

template <int BN, bool OB>
int launch(const CUtensorMap &ta, const CUtensorMap &tb, void *D, const float *bias, int batch, int M, int N, int K,
           long long ldd, long long bsd, int acc, int *err, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<BN, OB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         GemmSmem<BN>::total);
    if (e != cudaSuccess) return pot3d_cuda_status(e, "cudaFuncSetAttribute(k_gemm_tc)");
    attr = true;
  }
  dim3 grid((M + GM - 1) / GM, (N + BN - 1) / BN, batch);
  k_gemm_tc<BN, OB><<<grid, 128, GemmSmem<BN>::total, st>>>(ta, tb, D, bias, M, N, K, ldd, bsd, acc, err);
  return pot3d_cuda_status(cudaGetLastError(), "k_gemm_tc");
}

}  // namespace

// D[b][m][n] (+)= sum_k A[b][m][k] B[b][n][k] (+ bias[n]): BF16 inputs, FP32
// accumulation, FP32 (out_bf16 = 0) or BF16 output.  D rows are ldd
// elements apart (ldd >= N) and batches bstride_d apart; with accumulate the
// product is added to D.  K must be a multiple of 64 and N of 16; err
// (device int) is set if a bounded wait ran out.
extern "C" int pot3d_tc_gemm(const void *A, const void *B, void *D, const float *bias, int batch, int M, int N,
                             int K, long long ldd, long long bstride_d, int accumulate, int out_bf16, int *err,
                             void *stream) {
  if (!A || !B || !D || !err || batch < 1 || M < 1 || N < 16 || K < 64 || K % 64 || N % 16 || ldd < N) {
    pot3d_set_error("pot3d_tc_gemm: K must be a positive multiple of 64, N a multiple of 16, ldd >= N");
    return POT3D_ERR_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) {
    pot3d_set_error("pot3d_tc_gemm: A and B must be 16-byte aligned");
    return POT3D_ERR_ARG;
  }
  const int BN = N <= 32 ? 32 : (N <= 64 ? 64 : 128);
  CUtensorMap ta, tb;
  int st;
  if ((st = map_bf16(&ta, A, batch, M, K, GM))) return st;
  if ((st = map_bf16(&tb, B, batch, N, K, BN))) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define POT3D_GEMM_CASE(bn)                                                                                   \
  if (BN == bn)                                                                                               \
    return out_bf16 ? launch<bn, true>(ta, tb, D, bias, batch, M, N, K, ldd, bstride_d, accumulate, err, s)   \
                    : launch<bn, false>(ta, tb, D, bias, batch, M, N, K, ldd, bstride_d, accumulate, err, s);
  POT3D_GEMM_CASE(32)
  POT3D_GEMM_CASE(64)
  POT3D_GEMM_CASE(128)
#undef POT3D_GEMM_CASE
  return POT3D_ERR_ARG;
}
