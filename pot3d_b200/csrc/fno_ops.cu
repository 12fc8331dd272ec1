// Elementwise, layout and optimiser kernels of the learned warm start (the
// Fourier-style neural operator); its contractions run on pot3d_tc_gemm.
//
//   pot3d_fno_permute  4-D permutation with zero padding / cropping and an
//                      optional add into an FP32 output
//   pot3d_fno_gelu     GELU (tanh form) forward, or its derivative applied to
//                      an incoming gradient
//   pot3d_fno_colsum   deterministic column sums (bias gradients)
//   pot3d_fno_relmse   per-sample relative squared error and its gradient
//   pot3d_fno_adam     Adam step on FP32 master weights with a BF16 copy
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "pot3d_internal.cuh"

namespace {

enum { DT_F32 = 0, DT_BF16 = 1 };

__device__ __forceinline__ float ld(const void *p, long long i, int dt) {
  return dt == DT_F32 ? reinterpret_cast<const float *>(p)[i]
                      : __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(p)[i]);
}
__device__ __forceinline__ void st(void *p, long long i, int dt, float v) {
  if (dt == DT_F32)
    reinterpret_cast<float *>(p)[i] = v;
  else
    reinterpret_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn(v);
}

struct Dims4 {
  long long d[4];
};

// out[o0][o1][o2][o3] = in[i] with i[perm[a]] = o[a]; zero where i is
// outside in's extent.  With add, out (FP32) += value.
__global__ void k_permute(const void *__restrict__ in, int in_dt, Dims4 id, void *__restrict__ out, int out_dt, Dims4 od,
                          int p0, int p1, int p2, int p3, int add) {
  const long long n = od.d[0] * od.d[1] * od.d[2] * od.d[3];
  const int perm[4] = {p0, p1, p2, p3};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long o[4];
    long long r = t;
    o[3] = r % od.d[3];
    r /= od.d[3];
    o[2] = r % od.d[2];
    r /= od.d[2];
    o[1] = r % od.d[1];
    o[0] = r / od.d[1];
    long long i[4];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      i[perm[a]] = o[a];
    }
#pragma unroll
    for (int a = 0; a < 4; a++) inside = inside && i[a] < id.d[a];
    float v = 0.0f;
    if (inside) v = ld(in, ((i[0] * id.d[1] + i[1]) * id.d[2] + i[2]) * id.d[3] + i[3], in_dt);
    if (add)
      reinterpret_cast<float *>(out)[t] += v;
    else
      st(out, t, out_dt, v);
  }
}

__device__ __forceinline__ float gelu_f(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}
__device__ __forceinline__ float gelu_d(float x) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float u = k0 * (x + k1 * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k0 * (1.0f + 3.0f * k1 * x * x);
}

// forward: out[m][c] = gelu(pre[m][c]) for c < C, 0 for C <= c < ldo.
// backward: out[m][c] = grad[m][c] * gelu'(pre[m][c]) (c < C), 0 beyond.
__global__ void k_gelu(const float *__restrict__ pre, long long M, int C, int ldp, const void *__restrict__ grad,
                       int g_dt, int ldg, void *__restrict__ out, int out_dt, int ldo, int backward) {
  const long long n = M * ldo;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long m = t / ldo;
    const int c = (int)(t % ldo);
    float v = 0.0f;
    if (c < C) {
      const float x = pre[m * ldp + c];
      v = backward ? ld(grad, m * ldg + c, g_dt) * gelu_d(x) : gelu_f(x);
    }
    st(out, t, out_dt, v);
  }
}

// out[c] = sum_m in[m][c], c < C: per-block partial sums in a fixed order.
__global__ void k_colsum(const float *__restrict__ in, long long M, int C, int ld, float *__restrict__ part) {
  const int c = blockIdx.y;
  float s = 0.0f;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < M; m += (long long)gridDim.x * blockDim.x)
    s += in[m * ld + c];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(long long)c * gridDim.x + blockIdx.x] = red[0];
}
__global__ void k_colsum_final(const float *__restrict__ part, int nb, int C, float *__restrict__ out, int add) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.0f;
  for (int b = 0; b < nb; b++) s += part[(long long)c * nb + b];
  out[c] = add ? out[c] + s : s;
}

// Per sample b: loss_b = sum (pred - tgt)^2 / sum tgt^2 over npos x R values;
// grad = 2 (pred - tgt) / sum tgt^2 * scale.  pred rows have ldp >= R.
__global__ void k_relmse(const float *__restrict__ pred, int ldp, const void *__restrict__ tgt, int t_dt,
                         long long npos, int R, float scale, float *__restrict__ grad, float *__restrict__ loss) {
  const int b = blockIdx.x;
  const float *pb = pred + (long long)b * npos * ldp;
  float *gb = grad + (long long)b * npos * ldp;
  const long long tb = (long long)b * npos * R;
  __shared__ float r1[256], r2[256];
  float se = 0.0f, st2 = 0.0f;
  for (long long t = threadIdx.x; t < npos * R; t += blockDim.x) {
    const long long p = t / R;
    const int c = (int)(t % R);
    const float tv = ld(tgt, tb + t, t_dt);
    const float d = pb[p * ldp + c] - tv;
    se += d * d;
    st2 += tv * tv;
  }
  r1[threadIdx.x] = se;
  r2[threadIdx.x] = st2;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      r1[threadIdx.x] += r1[threadIdx.x + o];
      r2[threadIdx.x] += r2[threadIdx.x + o];
    }
    __syncthreads();
  }
  const float den = fmaxf(r2[0], 1e-30f);
  if (threadIdx.x == 0) loss[b] = r1[0] / den;
  const float f = 2.0f * scale / den;
  for (long long t = threadIdx.x; t < npos * ldp; t += blockDim.x) {
    const long long p = t / ldp;
    const int c = (int)(t % ldp);
    gb[t] = c < R ? f * (pb[t] - ld(tgt, tb + p * R + c, t_dt)) : 0.0f;
  }
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1, float *__restrict__ m2,
                       __nv_bfloat16 *__restrict__ wb, long long n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const float gt = g[t];
    const float a = b1 * m1[t] + (1.0f - b1) * gt;
    const float v = b2 * m2[t] + (1.0f - b2) * gt * gt;
    m1[t] = a;
    m2[t] = v;
    const float upd = lr * (a / c1) / (sqrtf(v / c2) + eps);
    const float nw = w[t] - upd;
    w[t] = nw;
    if (wb) wb[t] = __float2bfloat16_rn(nw);
  }
}

// x[b][p][0] = br0n[b][p]; x[b][p][1..3] = consts[p][0..2]; other channels 0.
__global__ void k_inputs(const float *__restrict__ br0n, const float *__restrict__ consts, long long B, long long npos,
                         __nv_bfloat16 *__restrict__ x) {
  const long long n = B * npos * 64;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t & 63);
    const long long bp = t >> 6;
    const long long p = bp % npos;
    float v = 0.0f;
    if (c == 0)
      v = br0n[bp];
    else if (c < 4)
      v = consts[p * 3 + (c - 1)];
    x[t] = __float2bfloat16_rn(v);
  }
}

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" int pot3d_fno_permute(const void *in, int in_dt, const long long *in_dims, void *out, int out_dt,
                                 const long long *out_dims, const int *perm, int add, void *stream) {
  Dims4 id, od;
  for (int a = 0; a < 4; a++) {
    id.d[a] = in_dims[a];
    od.d[a] = out_dims[a];
    if (id.d[a] < 1 || od.d[a] < 1 || perm[a] < 0 || perm[a] > 3) {
      pot3d_set_error("pot3d_fno_permute: bad dims or permutation");
      return POT3D_ERR_ARG;
    }
  }
  if (add && out_dt != DT_F32) {
    pot3d_set_error("pot3d_fno_permute: add needs an FP32 output");
    return POT3D_ERR_ARG;
  }
  const long long n = od.d[0] * od.d[1] * od.d[2] * od.d[3];
  k_permute<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(in, in_dt, id, out, out_dt, od, perm[0], perm[1], perm[2],
                                                            perm[3], add);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_permute");
}

extern "C" int pot3d_fno_gelu(const float *pre, long long M, int C, int ldp, const void *grad, int g_dt, int ldg,
                              void *out, int out_dt, int ldo, int backward, void *stream) {
  if (M < 1 || C < 1 || ldp < C || ldo < C || (backward && (!grad || ldg < C))) {
    pot3d_set_error("pot3d_fno_gelu: bad sizes");
    return POT3D_ERR_ARG;
  }
  k_gelu<<<grid_for(M * ldo), 256, 0, (cudaStream_t)stream>>>(pre, M, C, ldp, grad, g_dt, ldg, out, out_dt, ldo,
                                                               backward);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_gelu");
}

extern "C" int pot3d_fno_colsum(const float *in, long long M, int C, int ld, float *out, int add, float *scratch,
                                int scratch_len, void *stream) {
  const int nb = 64;
  if (M < 1 || C < 1 || ld < C || scratch_len < nb * C) {
    pot3d_set_error("pot3d_fno_colsum: bad sizes or scratch too small");
    return POT3D_ERR_ARG;
  }
  k_colsum<<<dim3(nb, C), 256, 0, (cudaStream_t)stream>>>(in, M, C, ld, scratch);
  k_colsum_final<<<(C + 127) / 128, 128, 0, (cudaStream_t)stream>>>(scratch, nb, C, out, add);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_colsum");
}

extern "C" int pot3d_fno_relmse(const float *pred, int ldp, const void *tgt, int t_dt, int nbatch, long long npos,
                                int R, float scale, float *grad, float *loss, void *stream) {
  if (nbatch < 1 || npos < 1 || R < 1 || ldp < R) {
    pot3d_set_error("pot3d_fno_relmse: bad sizes");
    return POT3D_ERR_ARG;
  }
  k_relmse<<<nbatch, 256, 0, (cudaStream_t)stream>>>(pred, ldp, tgt, t_dt, npos, R, scale, grad, loss);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_relmse");
}

extern "C" int pot3d_fno_adam(float *w, const float *g, float *m1, float *m2, void *wb, long long n, float lr, float b1,
                              float b2, float eps, int step, void *stream) {
  if (n < 1 || step < 1) {
    pot3d_set_error("pot3d_fno_adam: bad sizes");
    return POT3D_ERR_ARG;
  }
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, reinterpret_cast<__nv_bfloat16 *>(wb), n, lr, b1,
                                                         b2, eps, c1, c2);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_adam");
}

extern "C" int pot3d_fno_inputs(const float *br0n, const float *consts, long long B, long long npos, void *x,
                                void *stream) {
  if (B < 1 || npos < 1) {
    pot3d_set_error("pot3d_fno_inputs: bad sizes");
    return POT3D_ERR_ARG;
  }
  k_inputs<<<grid_for(B * npos * 64), 256, 0, (cudaStream_t)stream>>>(br0n, consts, B, npos,
                                                                     reinterpret_cast<__nv_bfloat16 *>(x));
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_inputs");
}

namespace {
// x[b][pos * R + i] = sigma[b] * out[b][pos][i], i < R: the network output
// (FP32, Rp channels per position) cropped to the radial levels and scaled
// back to the solver's packed FP64 layout (positions (phi, theta), r fastest).
__global__ void k_guess(const float *__restrict__ out, long long B, long long npos, int Rp, int R,
                        const double *__restrict__ sigma, double *__restrict__ x) {
  const long long n = B * npos * R;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % R);
    const long long bp = t / R;  // b * npos + pos
    const long long b = bp / npos;
    x[t] = (double)out[bp * Rp + i] * sigma[b];
  }
}
// The same with the radial levels resampled: the network's Rs levels (those
// of the mesh it was trained on) interpolated linearly onto the solver's R
// levels, level i from source levels idx[i] and idx[i]+1 with weight w[i]
// (outside [0, 1] at the ends: linear extrapolation).
__global__ void k_guess_resampled(const float *__restrict__ out, long long B, long long npos, int Rp,
                                  const int *__restrict__ idx, const double *__restrict__ w, int R,
                                  const double *__restrict__ sigma, double *__restrict__ x) {
  const long long n = B * npos * R;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % R);
    const long long bp = t / R;  // b * npos + pos
    const long long b = bp / npos;
    const float *o = out + bp * Rp + idx[i];
    const double lo = (double)o[0], hi = (double)o[1];
    x[t] = fma(w[i], hi - lo, lo) * sigma[b];
  }
}
}  // namespace

extern "C" int pot3d_fno_guess_resampled(const float *out, long long B, long long npos, int Rp, int Rs,
                                         const int *idx, const double *w, int R, const double *sigma, double *x,
                                         void *stream) {
  if (B < 1 || npos < 1 || R < 1 || Rs < 2 || Rp < Rs) {
    pot3d_set_error("pot3d_fno_guess_resampled: bad sizes");
    return POT3D_ERR_ARG;
  }
  k_guess_resampled<<<grid_for(B * npos * R), 256, 0, (cudaStream_t)stream>>>(out, B, npos, Rp, idx, w, R, sigma,
                                                                              x);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_guess_resampled");
}

extern "C" int pot3d_fno_guess(const float *out, long long B, long long npos, int Rp, int R, const double *sigma,
                               double *x, void *stream) {
  if (B < 1 || npos < 1 || R < 1 || Rp < R) {
    pot3d_set_error("pot3d_fno_guess: bad sizes");
    return POT3D_ERR_ARG;
  }
  k_guess<<<grid_for(B * npos * R), 256, 0, (cudaStream_t)stream>>>(out, B, npos, Rp, R, sigma, x);
  return pot3d_cuda_status(cudaGetLastError(), "pot3d_fno_guess");
}
