/*
 * pot3d_learned.h -- kernels of the learned warm start (a Fourier-style
 * neural operator that predicts the PCG initial guess from Br).  No
 * counterpart in the reference: POT3D always starts from x = 0
 * (src/pot3d.F90:3924); these entry points produce the guess passed to
 * pot3d_gpu_cgsolve_dev instead.  All pointers are DEVICE pointers; stream is
 * a cudaStream_t (NULL = default).  Return 0 or a POT3D_ERR_* code.
 */
#ifndef POT3D_LEARNED_H
#define POT3D_LEARNED_H

#ifdef __cplusplus
extern "C" {
#endif

/* D[b][m][n] (+)= sum_k A[b][m][k] B[b][n][k] (+ bias[n]) on the tcgen05
 * tensor cores: A, B BF16 with K contiguous, FP32 accumulation, FP32 or BF16
 * D with row stride ldd and batch stride bstride_d.  K % 64 == 0, N % 16 ==
 * 0; *err (device int) is set if a bounded wait ran out. */
int pot3d_tc_gemm(const void *A, const void *B, void *D, const float *bias, int batch, int M, int N, int K,
                  long long ldd, long long bstride_d, int accumulate, int out_bf16, int *err, void *stream);

/* 4-D permutation out[o] = in[i], i[perm[a]] = o[a], zero outside in
 * (padding/cropping); dtypes 0 = FP32, 1 = BF16; add: FP32 out += value. */
int pot3d_fno_permute(const void *in, int in_dt, const long long *in_dims, void *out, int out_dt,
                      const long long *out_dims, const int *perm, int add, void *stream);

/* GELU (tanh form) of pre[M][C] into out (zero-padded to ldo columns), or
 * with backward != 0 the incoming gradient times GELU'(pre). */
int pot3d_fno_gelu(const float *pre, long long M, int C, int ldp, const void *grad, int g_dt, int ldg, void *out,
                   int out_dt, int ldo, int backward, void *stream);

/* out[c] (+)= sum_m in[m][c] for c < C (deterministic; scratch >= 64*C). */
int pot3d_fno_colsum(const float *in, long long M, int C, int ld, float *out, int add, float *scratch,
                     int scratch_len, void *stream);

/* Per-sample relative squared error of pred[b][p][0..R) against tgt and its
 * gradient scaled by `scale`. */
int pot3d_fno_relmse(const float *pred, int ldp, const void *tgt, int t_dt, int nbatch, long long npos, int R,
                     float scale, float *grad, float *loss, void *stream);

/* One Adam step on FP32 weights w with gradient g (moments m1, m2); writes
 * a BF16 copy into wb when wb is not NULL. */
int pot3d_fno_adam(float *w, const float *g, float *m1, float *m2, void *wb, long long n, float lr, float b1,
                   float b2, float eps, int step, void *stream);

/* Network inputs x[b][p][64] (BF16): channel 0 = br0n[b][p], channels 1..3 =
 * consts[p][0..2], the rest 0. */
int pot3d_fno_inputs(const float *br0n, const float *consts, long long B, long long npos, void *x, void *stream);
/* Initial guesses from the network output: x[b][pos*R + i] = sigma[b] *
 * out[b][pos][i] for i < R (out FP32 with Rp >= R channels per position,
 * sigma FP64 on the device, x FP64 in the solver's packed layout). */
int pot3d_fno_guess(const float *out, long long B, long long npos, int Rp, int R, const double *sigma, double *x,
                    void *stream);
/* The same for a network trained on another radial mesh: its Rs output
 * levels (Rs <= Rp) are interpolated linearly onto the solver's R levels,
 * x[b][pos*R + i] = sigma[b] * (o[idx[i]] + w[i] * (o[idx[i]+1] - o[idx[i]]))
 * with o = out[b][pos] and 0 <= idx[i] <= Rs-2 (idx, w: device arrays of R;
 * w outside [0, 1] extrapolates at the ends).  No counterpart in the
 * reference, whose initial guess is zero (src/pot3d.F90:3924). */
int pot3d_fno_guess_resampled(const float *out, long long B, long long npos, int Rp, int Rs, const int *idx,
                              const double *w, int R, const double *sigma, double *x, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* POT3D_LEARNED_H */
