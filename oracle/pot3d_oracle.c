/*
 * pot3d_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement of POT3D's PCG hot path, used by the test suite, the
 * smoke check and the CPU-baseline leg of bench.py as the checker.  Nothing
 * in the product library links to or calls this file.
 *
 * Every routine follows the reference Fortran (src/pot3d.F90 of POT3D
 * v4.7.0) line by line: same loop orders, same operand orders, FP32 where
 * the reference uses r_typ_pc=REAL32 (src/pot3d.F90:94).  It is compiled
 * with -ffp-contract=off so each multiply and add rounds separately.
 * Parity is pinned by the reference's own test-suite outputs (energies and
 * convergence histories in testsuite/<case>/reference/pot3d.out) and by the
 * mesh tables those outputs print.
 *
 * Array conventions: 1-D mesh arrays are passed 0-based (Fortran element
 * k is C element k-1).  3-D fields are Fortran column-major (nr,nt,np).
 * The CG vectors are the reference's packed interior vectors,
 * idx = (k-2)*ntm2*nrm2 + (j-2)*nrm2 + (i-2)  (src/pot3d.F90:4930).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.1415926535897932 /* constants module, src/pot3d.F90:106 */

/* ------------------------------------------------------------------ */
/* Mesh generation: genmesh and helpers (src/pot3d.F90:2864-3752).      */
/* ------------------------------------------------------------------ */

/* fold, src/pot3d.F90:3707-3752 */
static double orc_fold(double x0, double x1, double x) {
  if (x0 == x1) return x;
  double xl = x1 - x0;
  double f = fmod(x - x0, xl) + x0;
  if (f < x0) f = f + xl;
  if (f >= x1) f = f - xl;
  return f;
}

/* map_xi_to_c, src/pot3d.F90:3374-3492.  Arrays are 1-based views. */
static int orc_map_xi_to_c(int periodic, int ns, const double *xi, const double *cs,
                           const double *a, const double *r, double cshft,
                           double xi_shift, double xiv, double *cv) {
  const double eps = 1.e-5;
  double xiv_p;
  if (periodic) {
    xiv_p = xiv + xi_shift;
    xiv_p = orc_fold(0.0, 1.0, xiv_p);
  } else {
    xiv_p = xiv;
  }
  int i;
  for (i = 1; i <= ns; i++)
    if (xiv_p >= xi[i] && xiv_p <= xi[i + 1]) break;
  if (i > ns) return -1;
  double d = xiv_p - xi[i];
  double d1 = xi[i + 1] - xi[i];
  double da = a[i] * d;
  double da1 = a[i] * d1;
  double fac;
  if (fabs(da1) < eps)
    fac = (d * (1.0 + 0.5 * da)) / (d1 * (1.0 + 0.5 * da1));
  else
    fac = (exp(da) - 1.0) / (r[i] - 1.0);
  double c = cs[i] + (cs[i + 1] - cs[i]) * fac;
  if (periodic) {
    c = c - cshft;
    c = orc_fold(cs[1], cs[ns + 1], c);
  }
  *cv = c;
  return 0;
}

/* map_c_to_xi, src/pot3d.F90:3494-3586 */
static int orc_map_c_to_xi(int periodic, int ns, const double *xi, const double *cs,
                           const double *a, const double *r, double cv, double *xiv) {
  const double eps = 1.e-5;
  double cv_p = periodic ? orc_fold(cs[1], cs[ns + 1], cv) : cv;
  int i;
  for (i = 1; i <= ns; i++)
    if (cv_p >= cs[i] && cv_p <= cs[i + 1]) break;
  if (i > ns) return -1;
  double d = (cv_p - cs[i]) / (cs[i + 1] - cs[i]);
  double da = (r[i] - 1.0) * d;
  double fac;
  if (fabs(da) < eps)
    fac = d * (xi[i + 1] - xi[i]);
  else
    fac = log(da + 1.0) / a[i];
  *xiv = xi[i] + fac;
  return 0;
}

/* filter_coord, src/pot3d.F90:3588-3640 (f is 1-based view) */
static void orc_filter_coord(int n, double *f) {
  double *ff = (double *)malloc(sizeof(double) * (n + 1));
  for (int i = 1; i <= n; i++) ff[i] = f[i];
  for (int i = 2; i <= n - 1; i++) f[i] = 0.25 * (ff[i - 1] + 2.0 * ff[i] + ff[i + 1]);
  free(ff);
}

/* filter_coord_periodic, src/pot3d.F90:3642-3705 */
static void orc_filter_coord_periodic(double xl, int n, double *f) {
  double *ff = (double *)malloc(sizeof(double) * (n + 2));
  double f1old = f[1];
  for (int i = 1; i <= n; i++) ff[i] = f[i];
  ff[0] = f[n - 1] - xl;
  ff[n + 1] = f[2] + xl;
  for (int i = 1; i <= n; i++) f[i] = 0.25 * (ff[i - 1] + 2.0 * ff[i] + ff[i + 1]);
  double f1new = f[1];
  for (int i = 1; i <= n; i++) f[i] = f[i] - f1new + f1old;
  free(ff);
}

/*
 * genmesh, src/pot3d.F90:2864-3372.  frac/dratio have nseg entries
 * (0-based), c receives nc points (0-based).  Returns 0 on success and a
 * nonzero code where the reference calls endrun.
 */
int orc_genmesh(int nc, double c0, double c1, int nseg, const double *frac0,
                const double *dratio0, int nfilt, int periodic, double c_shift,
                double *c0based) {
  const double eps = 1.e-5;
  const double *frac = frac0 - 1;     /* 1-based */
  const double *dratio = dratio0 - 1; /* 1-based */
  double *c = c0based - 1;
  if (nc < 2) return 1;
  if (c0 >= c1) return 2;
  int nf;
  for (nf = 1; nf <= nseg - 1; nf++)
    if (frac[nf + 1] == 0.0) break;
  int ns;
  double *cs, *r;
  if (nf == 1 && frac[1] == 0.0) {
    ns = 1;
    cs = (double *)calloc(ns + 2, sizeof(double));
    r = (double *)calloc(ns + 1, sizeof(double));
    cs[1] = c0;
    cs[2] = c1;
    r[1] = 1.0;
  } else {
    for (int i = 2; i <= nf; i++)
      if (frac[i] < frac[i - 1]) return 3;
    if (periodic) {
      if (frac[1] < 0.0 || frac[nf] > 1.0) return 4;
      if (frac[1] == 0.0 && frac[nf] == 1.0) return 5;
    } else {
      if (frac[1] != 0.0) return 6;
      if (frac[nf] != 1.0) return 7;
    }
    int nr = periodic ? nf : nf - 1;
    for (int i = 1; i <= nr; i++)
      if (dratio[i] <= 0.0) return 8;
    ns = nf - 1;
    if (periodic) {
      if (frac[1] != 0.0) ns = ns + 1;
      if (frac[nf] != 1.0) ns = ns + 1;
    }
    cs = (double *)calloc(ns + 2, sizeof(double));
    r = (double *)calloc(ns + 1, sizeof(double));
    if (periodic) {
      if (frac[1] != 0.0) {
        cs[1] = c0;
        for (int i = 1; i <= nf; i++) cs[i + 1] = c0 + (c1 - c0) * frac[i];
        if (frac[nf] != 1.0) {
          double alpha = (1.0 - frac[nf]) / (frac[1] + 1.0 - frac[nf]);
          r[1] = dratio[nr] / (1.0 + alpha * (dratio[nr] - 1.0));
          for (int i = 1; i <= nr; i++) r[i + 1] = dratio[i];
          cs[ns + 1] = c1;
          r[ns] = 1.0 + alpha * (dratio[nr] - 1.0);
        } else {
          r[1] = dratio[nr];
          for (int i = 2; i <= nr; i++) r[i] = dratio[i - 1];
        }
      } else {
        for (int i = 1; i <= nf; i++) cs[i] = c0 + (c1 - c0) * frac[i];
        for (int i = 1; i <= nr; i++) r[i] = dratio[i];
        cs[ns + 1] = c1;
      }
    } else {
      for (int i = 1; i <= nf; i++) cs[i] = c0 + (c1 - c0) * frac[i];
      for (int i = 1; i <= nr; i++) r[i] = dratio[i];
    }
  }
  /* label 100 */
  double *xi = (double *)calloc(ns + 2, sizeof(double));
  double *a = (double *)calloc(ns + 1, sizeof(double));
  double *f = (double *)calloc(ns + 1, sizeof(double));
  for (int i = 1; i <= ns; i++) {
    double dr = r[i] - 1.0;
    if (fabs(dr) < eps)
      f[i] = (cs[i + 1] - cs[i]) * (1.0 + 0.5 * dr);
    else
      f[i] = (cs[i + 1] - cs[i]) * log(r[i]) / dr;
  }
  double fac = 0.0;
  for (int i = ns; i >= 1; i--) fac = fac / r[i] + f[i];
  double d = f[1] / fac;
  xi[1] = 0.0;
  for (int i = 2; i <= ns; i++) {
    xi[i] = xi[i - 1] + d;
    if (i < ns) d = d * f[i] / (f[i - 1] * r[i - 1]);
  }
  xi[ns + 1] = 1.0;
  for (int i = 1; i <= ns; i++) a[i] = log(r[i]) / (xi[i + 1] - xi[i]);
  double cshft = 0.0, xi_shift = 0.0;
  int rc = 0;
  if (periodic) {
    cshft = -c_shift;
    rc = orc_map_c_to_xi(periodic, ns, xi, cs, a, r, cshft, &xi_shift);
  }
  if (rc == 0) {
    double dxi = 1.0 / (nc - 1.0);
    c[1] = c0;
    for (int j = 2; j <= nc - 1 && rc == 0; j++) {
      double xiv = (j - 1) * dxi;
      rc = orc_map_xi_to_c(periodic, ns, xi, cs, a, r, cshft, xi_shift, xiv, &c[j]);
    }
    c[nc] = c1;
    for (int i = 1; i <= nfilt; i++) {
      if (periodic)
        orc_filter_coord_periodic(c1 - c0, nc, c);
      else
        orc_filter_coord(nc, c);
    }
  }
  free(cs);
  free(r);
  free(xi);
  free(a);
  free(f);
  return rc ? 9 : 0;
}

/*
 * Mesh arrays at one rank (local == global, nrm=nrm1, ntm=ntm1, npm=np;
 * src/pot3d.F90:1801,1967,1975).  Lengths: r,dr: nr-1; rh,drh: nr;
 * t,dt,st: nt-1; th,dth,sth: nt; p,dp,ph,dph: np.
 */
typedef struct {
  int nr, nt, np;
  double *r, *dr, *rh, *drh;
  double *t, *dt, *th, *dth, *st, *sth;
  double *p, *dp, *ph, *dph;
} orc_mesh;

/* set_global_mesh, src/pot3d.F90:2583-2708 (arrays allocated by caller). */
int orc_set_mesh(orc_mesh *m, double r0, double r1, int nseg, const double *rfrac,
                 const double *drratio, int nfrmesh, const double *tfrac,
                 const double *dtratio, int nftmesh, const double *pfrac,
                 const double *dpratio, int nfpmesh, double phishift) {
  const int nr = m->nr, nt = m->nt, np = m->np;
  const int nrm1 = nr - 1, ntm1 = nt - 1, npm1 = np - 1;
  const double pl = 2.0 * ORC_PI - 0.0;
  int rc;
  /* 1-based views */
  double *r = m->r - 1, *dr = m->dr - 1, *rh = m->rh - 1, *drh = m->drh - 1;
  double *t = m->t - 1, *dt = m->dt - 1, *th = m->th - 1, *dth = m->dth - 1;
  double *p = m->p - 1, *dp = m->dp - 1, *ph = m->ph - 1, *dph = m->dph - 1;

  rc = orc_genmesh(nrm1, r0, r1, nseg, rfrac, drratio, nfrmesh, 0, 0.0, m->r);
  if (rc) return 10 + rc;
  for (int i = 2; i <= nrm1; i++) {
    rh[i] = .5 * (r[i] + r[i - 1]);
    drh[i] = r[i] - r[i - 1];
  }
  rh[1] = rh[2] - drh[2];
  rh[nr] = rh[nrm1] + drh[nrm1];
  drh[1] = drh[2];
  drh[nr] = drh[nrm1];
  for (int i = 1; i <= nrm1; i++) dr[i] = rh[i + 1] - rh[i];

  rc = orc_genmesh(ntm1, 0.0, ORC_PI, nseg, tfrac, dtratio, nftmesh, 0, 0.0, m->t);
  if (rc) return 20 + rc;
  for (int j = 2; j <= ntm1; j++) {
    th[j] = .5 * (t[j] + t[j - 1]);
    dth[j] = t[j] - t[j - 1];
  }
  th[1] = th[2] - dth[2];
  th[nt] = th[ntm1] + dth[ntm1];
  dth[1] = dth[2];
  dth[nt] = dth[ntm1];
  for (int j = 1; j <= ntm1; j++) dt[j] = th[j + 1] - th[j];

  rc = orc_genmesh(npm1, 0.0, 2.0 * ORC_PI, nseg, pfrac, dpratio, nfpmesh, 1, phishift,
                   m->p);
  if (rc) return 30 + rc;
  p[np] = p[2] + pl;
  for (int k = 2; k <= np; k++) {
    ph[k] = 0.5 * (p[k] + p[k - 1]);
    dph[k] = p[k] - p[k - 1];
  }
  ph[1] = ph[npm1] - pl;
  dph[1] = dph[npm1];
  for (int k = 1; k <= npm1; k++) dp[k] = ph[k + 1] - ph[k];
  dp[np] = dp[2];
  dph[np] = dph[2];
  dp[1] = dp[npm1];

  for (int j = 0; j < ntm1; j++) m->st[j] = sin(m->t[j]);
  for (int j = 0; j < nt; j++) m->sth[j] = sin(m->th[j]);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Br boundary map: intrp2d / interp / readbr (src/pot3d.F90:6672-7072) */
/* ------------------------------------------------------------------ */

/* interp, src/pot3d.F90:7028-7072 (x 0-based, returns 1-based index) */
static int orc_interp(const double *x, int n, double xv, int *i1, double *alpha) {
  for (int i = 1; i <= n - 1; i++) {
    if (xv >= x[i - 1] && xv <= x[i]) {
      *alpha = (xv - x[i - 1]) / (x[i] - x[i - 1]);
      *i1 = i;
      return 0;
    }
  }
  return -1;
}

/*
 * readbr after the file read (src/pot3d.F90:6751-6829) plus the |Br| flip of
 * set_flux for option 'open' (src/pot3d.F90:3832).  fi is the map in
 * Fortran order fi(ntn,npn) with scales tn, pn.  br0 is (nt,np)
 * column-major.  option: 0='potential', 1='open', 2='ss'.
 */
int orc_readbr(const orc_mesh *m, int ntn, int npn, const double *tn, const double *pn,
               const double *fi, int option, int do_not_balance_flux, double *br0) {
  const int nt = m->nt, np = m->np, ntm1 = nt - 1, npm1 = np - 1;
  const double pl_i = 1.0 / (2.0 * ORC_PI);
#define BR0(j, k) br0[((j)-1) + (size_t)nt * ((k)-1)]
#define FI(i, j) fi[((i)-1) + (size_t)ntn * ((j)-1)]
  /* flint monotonicity check of the scales (src/pot3d.F90:6934-7026) */
  for (int i = 1; i < ntn; i++)
    if (!(tn[i] > tn[i - 1])) return 1;
  for (int i = 1; i < npn; i++)
    if (!(pn[i] > pn[i - 1])) return 1;
  /* intrp2d into br0_g(2:ntm1,2:npm1) at th_g(2:ntm1), ph_g(2:npm1) */
  for (int k = 2; k <= npm1; k++) {
    double yv = m->ph[k - 1];
    if (yv < pn[0] || yv > pn[npn - 1]) return 2;
    int jj;
    double ay;
    if (orc_interp(pn, npn, yv, &jj, &ay)) return 2;
    for (int j = 2; j <= ntm1; j++) {
      double xv = m->th[j - 1];
      if (xv < tn[0] || xv > tn[ntn - 1]) return 2;
      int ii;
      double ax;
      if (orc_interp(tn, ntn, xv, &ii, &ax)) return 2;
      BR0(j, k) = (1. - ax) * ((1. - ay) * FI(ii, jj) + ay * FI(ii, jj + 1)) +
                  ax * ((1. - ay) * FI(ii + 1, jj) + ay * FI(ii + 1, jj + 1));
    }
  }
  /* periodic copy */
  for (int j = 1; j <= nt; j++) {
    BR0(j, 1) = BR0(j, npm1);
    BR0(j, np) = BR0(j, 2);
  }
  /* poles: m=0 only */
  double sum0 = 0.0, sum1 = 0.0;
  for (int k = 2; k <= npm1; k++) sum0 += BR0(2, k) * m->dph[k - 1];
  for (int k = 2; k <= npm1; k++) sum1 += BR0(ntm1, k) * m->dph[k - 1];
  sum0 = sum0 * pl_i;
  sum1 = sum1 * pl_i;
  for (int k = 1; k <= np; k++) {
    BR0(1, k) = 2.0 * sum0 - BR0(2, k);
    BR0(nt, k) = 2.0 * sum1 - BR0(ntm1, k);
  }
  /* flux balance */
  double area = 0.0, fluxp = 0.0, fluxm = 0.0;
  for (int j = 2; j <= ntm1; j++) {
    for (int k = 2; k <= npm1; k++) {
      double da = m->sth[j - 1] * m->dth[j - 1] * m->dph[k - 1];
      if (BR0(j, k) > 0.)
        fluxp = fluxp + BR0(j, k) * da;
      else
        fluxm = fluxm + BR0(j, k) * da;
      area = area + da;
    }
  }
  if (!((option == 2 || option == 1) && do_not_balance_flux)) {
    double br00err = (fluxp + fluxm) / area;
    for (int k = 1; k <= np; k++)
      for (int j = 1; j <= nt; j++) BR0(j, k) = BR0(j, k) - br00err;
  }
  /* set_flux: the monopole trick for 'open' (src/pot3d.F90:3816-3833) */
  if (option == 1) {
    for (size_t q = 0; q < (size_t)nt * np; q++) br0[q] = fabs(br0[q]);
  }
#undef BR0
#undef FI
  return 0;
}

/* ------------------------------------------------------------------ */
/* Seeded synthetic Br maps.  Not a reference routine: the reference    */
/* reads its Br maps from HDF5 files.  This restates the product's      */
/* generator (pot3d_host_synthetic_br, pot3d_b200/csrc/host_mesh.cpp)   */
/* operation for operation, so inputs can be built with the oracle      */
/* alone; tests/test_oracle.py checks the two bit for bit.              */
/* Spherical harmonics l = 1..lmax (orthonormal, N(0,1)/l^2, scaled to  */
/* 5 G RMS), nbip Gaussian bipoles (sigma 3 deg, +-50 G), area-weighted */
/* mean removed; seed -> splitmix64 -> Box-Muller.                      */
/* ------------------------------------------------------------------ */
static uint64_t orc_sm_next(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double orc_sm_uniform(uint64_t *s) { return (double)(orc_sm_next(s) >> 11) * (1.0 / 9007199254740992.0); }
static double orc_sm_normal(uint64_t *s) {
  const double u1 = 1.0 - orc_sm_uniform(s);
  const double u2 = orc_sm_uniform(s);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * ORC_PI * u2);
}

int orc_synthetic_br(unsigned long long seed, int lmax, int nbip, int ntn, int npn, double *tn, double *pn,
                     double *fi) {
  if (ntn < 3 || npn < 3 || lmax < 1) return 1;
  uint64_t rng = seed;
  const int L = lmax, W = lmax + 1;
  for (int j = 0; j < ntn; j++) tn[j] = ORC_PI * j / (ntn - 1);
  for (int k = 0; k < npn; k++) pn[k] = 2.0 * ORC_PI * k / (npn - 1);
  double *ac = calloc((size_t)W * W, sizeof(double)), *as = calloc((size_t)W * W, sizeof(double));
  double *Fc = malloc(sizeof(double) * (size_t)ntn * W), *Fs = malloc(sizeof(double) * (size_t)ntn * W);
  double *cm = malloc(sizeof(double) * W), *sm = malloc(sizeof(double) * W);
  if (!ac || !as || !Fc || !Fs || !cm || !sm) {
    free(ac); free(as); free(Fc); free(Fs); free(cm); free(sm);
    return 2;
  }
  for (int l = 1; l <= L; l++)
    for (int m = 0; m <= l; m++) {
      const double s = 1.0 / ((double)l * l);
      ac[l * W + m] = orc_sm_normal(&rng) * s;
      if (m > 0) as[l * W + m] = orc_sm_normal(&rng) * s;
    }
  for (int j = 0; j < ntn; j++) {
    const double x = cos(tn[j]), sx = sin(tn[j]);
    double p_mm = 1.0 / sqrt(4.0 * ORC_PI);
    for (int m = 0; m <= L; m++) {
      if (m > 0) p_mm *= sqrt((2.0 * m + 1.0) / (2.0 * m)) * sx;
      double pl2 = 0.0, pl1 = p_mm, fc = 0.0, fs = 0.0;
      const double norm = (m == 0) ? 1.0 : sqrt(2.0);
      for (int l = m; l <= L; l++) {
        double pl;
        if (l == m) {
          pl = p_mm;
        } else if (l == m + 1) {
          pl = sqrt(2.0 * m + 3.0) * x * p_mm;
        } else {
          const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
          const double b = sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
          pl = a * (x * pl1 - b * pl2);
        }
        if (l > m) {
          pl2 = pl1;
          pl1 = pl;
        }
        if (l >= 1) {
          fc += norm * ac[l * W + m] * pl;
          fs += norm * as[l * W + m] * pl;
        }
        if (l == m) {
          pl2 = 0.0;
          pl1 = pl;
        }
      }
      Fc[(size_t)j * W + m] = fc;
      Fs[(size_t)j * W + m] = fs;
    }
  }
  double wsum = 0.0, ssq = 0.0;
  for (int k = 0; k < npn; k++) {
    for (int m = 0; m <= L; m++) {
      cm[m] = cos(m * pn[k]);
      sm[m] = sin(m * pn[k]);
    }
    for (int j = 0; j < ntn; j++) {
      double v = 0.0;
      for (int m = 0; m <= L; m++) v += Fc[(size_t)j * W + m] * cm[m] + Fs[(size_t)j * W + m] * sm[m];
      fi[j + (size_t)ntn * k] = v;
      const double w = sin(tn[j]);
      wsum += w;
      ssq += w * v * v;
    }
  }
  const double rms = sqrt(ssq / wsum);
  const double scale = rms > 0 ? 5.0 / rms : 0.0;
  for (size_t q = 0; q < (size_t)ntn * npn; q++) fi[q] *= scale;
  const double deg = ORC_PI / 180.0, sig = 3.0 * deg, half_sep = 3.0 * deg;
  for (int b = 0; b < nbip; b++) {
    const double lat = (-35.0 + 70.0 * orc_sm_uniform(&rng)) * deg;
    const double lon = 360.0 * orc_sm_uniform(&rng) * deg;
    const double tilt = (-20.0 + 40.0 * orc_sm_uniform(&rng)) * deg;
    const double sgn = orc_sm_uniform(&rng) < 0.5 ? 1.0 : -1.0;
    for (int side = 0; side < 2; side++) {
      const double sd = side == 0 ? 1.0 : -1.0;
      const double slat = lat + sd * half_sep * sin(tilt);
      const double slon = lon + sd * half_sep * cos(tilt) / cos(lat);
      const double amp = 50.0 * sgn * sd;
      const double cl = cos(slat), sl = sin(slat);
      for (int k = 0; k < npn; k++)
        for (int j = 0; j < ntn; j++) {
          const double plat = 0.5 * ORC_PI - tn[j];
          double c = sl * sin(plat) + cl * cos(plat) * cos(pn[k] - slon);
          c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
          const double d = acos(c);
          fi[j + (size_t)ntn * k] += amp * exp(-0.5 * (d * d) / (sig * sig));
        }
    }
  }
  double num = 0.0;
  for (int k = 0; k < npn - 1; k++)
    for (int j = 0; j < ntn; j++) num += sin(tn[j]) * fi[j + (size_t)ntn * k];
  double den = 0.0;
  for (int k = 0; k < npn - 1; k++)
    for (int j = 0; j < ntn; j++) den += sin(tn[j]);
  const double mean = num / den;
  for (size_t q = 0; q < (size_t)ntn * npn; q++) fi[q] -= mean;
  free(ac); free(as); free(Fc); free(Fs); free(cm); free(sm);
  return 0;
}

/* ------------------------------------------------------------------ */
/* The solve context: coefficients, preconditioner, work arrays.        */
/* ------------------------------------------------------------------ */

typedef struct {
  int nr, nt, np, nrm1, ntm1, npm1, nrm2, ntm2, npm2;
  long N;
  int ifprec;
  double pm_r1, pl_i, dr1, drn;
  /* derived 1-D arrays, 1-based like the Fortran local_mesh module */
  double *drh, *dth, *sth_i, *dp_i, *dph, *st, *dt_i, *sth, *r2, *dr_i;
  double *dr, *rh, *dt, *dp;
  double *br0, *br1; /* (nt,np) column-major; br1 only for validation */
  double *a;         /* a(N,7): coefficient m of point idx at a[(m-1)*N+idx] */
  float *a_i;        /* diagonal preconditioner */
  /* ILU0 storage (1-based CSR like the reference) */
  long M;
  int *ia, *ja, *dptr, *n1, *n2, *luja;
  float *acsr, *lu, *lud_i;
  int ilu_icode;
  double *x_ax;   /* (nr,nt,np) scratch */
  double *sum0, *sum1;
} orc_ctx;

#define XA(x, i, j, k) (x)[((i)-1) + (size_t)c->nr * (((j)-1) + (size_t)c->nt * ((k)-1))]

/* Deterministic dot: fixed chunking independent of thread count. */
#define ORC_DOT_CHUNKS 256
static double orc_dot(const double *x, const double *y, long n) {
  double part[ORC_DOT_CHUNKS];
  long chunk = (n + ORC_DOT_CHUNKS - 1) / ORC_DOT_CHUNKS;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < ORC_DOT_CHUNKS; c++) {
    long lo = c * chunk, hi = lo + chunk < n ? lo + chunk : n;
    double s = 0.0;
    for (long i = lo; i < hi; i++) s = s + x[i] * y[i];
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < ORC_DOT_CHUNKS; c++) s += part[c];
  return s;
}

/* load_matrix_pot3d_solve, src/pot3d.F90:4565-4613 */
static void orc_load_matrix(orc_ctx *c) {
  const long N = c->N;
  double *drh = c->drh, *dth = c->dth, *sth_i = c->sth_i, *dp_i = c->dp_i, *dph = c->dph;
  double *st = c->st, *dt_i = c->dt_i, *sth = c->sth, *r2 = c->r2, *dr_i = c->dr_i;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= c->npm1; k++)
    for (int j = 2; j <= c->ntm1; j++)
      for (int i = 2; i <= c->nrm1; i++) {
        long ii = (long)(k - 2) * c->ntm2 * c->nrm2 + (long)(j - 2) * c->nrm2 + (i - 2);
        double a1 = -drh[i] * dth[j] * sth_i[j] * dp_i[k - 1];
        double a2 = -drh[i] * dph[k] * st[j - 1] * dt_i[j - 1];
        double a3 = -sth[j] * dth[j] * dph[k] * r2[i - 1] * dr_i[i - 1];
        double a5 = -sth[j] * dth[j] * dph[k] * r2[i] * dr_i[i];
        double a6 = -drh[i] * dph[k] * st[j] * dt_i[j];
        double a7 = -drh[i] * dth[j] * sth_i[j] * dp_i[k];
        double a4 = -(a1 + a2 + a3 + a5 + a6 + a7);
        c->a[0 * N + ii] = a1;
        c->a[1 * N + ii] = a2;
        c->a[2 * N + ii] = a3;
        c->a[3 * N + ii] = a4;
        c->a[4 * N + ii] = a5;
        c->a[5 * N + ii] = a6;
        c->a[6 * N + ii] = a7;
      }
}

/* set_boundary_points + sum_over_phi at one rank, src/pot3d.F90:5376-5487 */
static void orc_set_boundary_points(orc_ctx *c, double *x, double vmask) {
  const int nr = c->nr, nt = c->nt, nrm1 = c->nrm1, ntm1 = c->ntm1, npm1 = c->npm1;
#define BR0(j, k) c->br0[((j)-1) + (size_t)nt * ((k)-1)]
#define BR1(j, k) c->br1[((j)-1) + (size_t)nt * ((k)-1)]
  for (int k = 2; k <= npm1; k++)
    for (int j = 2; j <= ntm1; j++) XA(x, 1, j, k) = XA(x, 2, j, k) - vmask * BR0(j, k) * c->dr1;
  if (c->br1) {
    for (int k = 2; k <= npm1; k++)
      for (int j = 2; j <= ntm1; j++)
        XA(x, nr, j, k) = XA(x, nrm1, j, k) + vmask * BR1(j, k) * c->drn;
  } else {
    for (int k = 2; k <= npm1; k++)
      for (int j = 2; j <= ntm1; j++) XA(x, nr, j, k) = c->pm_r1 * XA(x, nrm1, j, k);
  }
  for (int i = 1; i <= nr; i++) {
    double s0 = 0., s1 = 0.;
    for (int k = 2; k <= npm1; k++) s0 = s0 + XA(x, i, 2, k) * c->dph[k] * c->pl_i;
    for (int k = 2; k <= npm1; k++) s1 = s1 + XA(x, i, ntm1, k) * c->dph[k] * c->pl_i;
    c->sum0[i] = s0;
    c->sum1[i] = s1;
  }
  for (int k = 2; k <= npm1; k++)
    for (int i = 1; i <= nr; i++) XA(x, i, 1, k) = 2.0 * c->sum0[i] - XA(x, i, 2, k);
  for (int k = 2; k <= npm1; k++)
    for (int i = 1; i <= nr; i++) XA(x, i, nt, k) = 2.0 * c->sum1[i] - XA(x, i, ntm1, k);
#undef BR0
#undef BR1
}

/* seam_hhh at one rank: periodic phi planes, src/pot3d.F90:5746-5758 */
static void orc_seam(orc_ctx *c, double *x) {
  size_t plane = (size_t)c->nr * c->nt;
  memcpy(x + 0 * plane, x + (size_t)(c->np - 2) * plane, plane * sizeof(double));
  memcpy(x + (size_t)(c->np - 1) * plane, x + 1 * plane, plane * sizeof(double));
}

/* unpack_scalar, src/pot3d.F90:5304-5335 */
static void orc_unpack(orc_ctx *c, double *s, const double *x) {
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= c->npm1; k++)
    for (int j = 2; j <= c->ntm1; j++)
      for (int i = 2; i <= c->nrm1; i++)
        XA(s, i, j, k) = x[(long)(k - 2) * c->ntm2 * c->nrm2 + (long)(j - 2) * c->nrm2 + (i - 2)];
}

/* delsq, src/pot3d.F90:5337-5374 */
static void orc_delsq(orc_ctx *c, const double *x, double *y) {
  const long N = c->N;
  const double *a = c->a;
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= c->npm1; k++)
    for (int j = 2; j <= c->ntm1; j++)
      for (int i = 2; i <= c->nrm1; i++) {
        long ii = (long)(k - 2) * c->ntm2 * c->nrm2 + (long)(j - 2) * c->nrm2 + (i - 2);
        y[ii] = a[0 * N + ii] * XA(x, i, j, k - 1) + a[1 * N + ii] * XA(x, i, j - 1, k) +
                a[2 * N + ii] * XA(x, i - 1, j, k) + a[3 * N + ii] * XA(x, i, j, k) +
                a[4 * N + ii] * XA(x, i + 1, j, k) + a[5 * N + ii] * XA(x, i, j + 1, k) +
                a[6 * N + ii] * XA(x, i, j, k + 1);
      }
}

/* ax, src/pot3d.F90:5102-5150 */
int orc_ax(orc_ctx *c, const double *x, double *y) {
  orc_unpack(c, c->x_ax, x);
  orc_set_boundary_points(c, c->x_ax, 0.0);
  orc_seam(c, c->x_ax);
  orc_delsq(c, c->x_ax, y);
  return 0;
}

/* ---------------- ILU0 path (src/pot3d.F90:4717-5100) --------------- */

/* getM, src/pot3d.F90:5020-5100 (IA 1-based, M = IA(N+1)) */
static void orc_getM(orc_ctx *c) {
  long i = 0;
  c->ia[1] = 1;
  for (int mk = 2; mk <= c->npm1; mk++)
    for (int mj = 2; mj <= c->ntm1; mj++)
      for (int mi = 2; mi <= c->nrm1; mi++) {
        i++;
        int ok[8] = {0, 1, 1, 1, 1, 1, 1, 1};
        if (mi == 2) ok[3] = 0;
        if (mi == c->nrm1) ok[5] = 0;
        if (mj == 2) ok[2] = 0;
        if (mj == c->ntm1) ok[6] = 0;
        int n = 0;
        for (int jj = 1; jj <= 7; jj++) n += ok[jj];
        c->ia[i + 1] = c->ia[i] + n;
      }
  c->M = c->ia[c->N + 1];
}

/* diacsr, src/pot3d.F90:4870-5018 (nproc_p=1: periodic entries kept) */
static void orc_diacsr(orc_ctx *c) {
  const long N = c->N;
  const long ioff[8] = {0, -(long)c->nrm2 * c->ntm2, -c->nrm2, -1, 0, 1, c->nrm2,
                        (long)c->nrm2 * c->ntm2};
  for (int mk = 2; mk <= c->npm1; mk++)
    for (int mj = 2; mj <= c->ntm1; mj++)
      for (int mi = 2; mi <= c->nrm1; mi++) {
        long i = (long)(mk - 2) * (c->ntm1 - 1) * (c->nrm1 - 1) + (long)(mj - 2) * (c->nrm1 - 1) +
                 (mi - 1);
        long ko = c->ia[i];
        int ok[8] = {0, 1, 1, 1, 1, 1, 1, 1};
        if (mi == 2) ok[3] = 0;
        if (mi == c->nrm1) ok[5] = 0;
        if (mj == 2) ok[2] = 0;
        if (mj == c->ntm1) ok[6] = 0;
        for (int jj = 1; jj <= 7; jj++)
          if (ok[jj]) {
            long j = i + ioff[jj];
            if (j > N) {
              j = j - N;
              c->acsr[ko] = (float)c->a[(jj - 1) * N + (i - 1)];
              c->ja[ko] = (int)j;
              ko++;
            }
          }
        for (int jj = 1; jj <= 7; jj++)
          if (ok[jj]) {
            long j = i + ioff[jj];
            if (j >= 1 && j <= N) {
              if (jj == 4) c->dptr[i] = (int)ko;
              c->acsr[ko] = (float)c->a[(jj - 1) * N + (i - 1)];
              c->ja[ko] = (int)j;
              ko++;
            }
          }
        for (int jj = 1; jj <= 7; jj++)
          if (ok[jj]) {
            long j = i + ioff[jj];
            if (j < 1) {
              j = N + j;
              c->acsr[ko] = (float)c->a[(jj - 1) * N + (i - 1)];
              c->ja[ko] = (int)j;
              ko++;
            }
          }
      }
}

/* ilu0, src/pot3d.F90:4717-4813 (FP32, Saad's row-wise ILU(0)) */
static int orc_ilu0(orc_ctx *c) {
  const long N = c->N;
  int *iw = (int *)calloc(N + 1, sizeof(int));
  float *A = c->acsr;
  int *JA = c->ja, *IA = c->ia, *A_da = c->dptr;
  int icode = 0;
  for (long i = 2; i <= N; i++) {
    int IA_i = IA[i], IA_ip1m1 = IA[i + 1] - 1;
    for (int ij = IA_i; ij <= IA_ip1m1; ij++) iw[JA[ij]] = ij;
    int ik;
    for (ik = IA_i; ik <= A_da[i] - 1; ik++) {
      int k = JA[ik];
      float Aik = A[ik] / A[A_da[k]];
      A[ik] = Aik;
      for (int kj = A_da[k] + 1; kj <= IA[k + 1] - 1; kj++) {
        int ij = iw[JA[kj]];
        if (ij != 0) A[ij] = A[ij] - Aik * A[kj];
      }
    }
    if (A[ik] == 0) {
      icode = (int)i;
      break;
    }
    for (int ij = IA_i; ij <= IA_ip1m1; ij++) iw[JA[ij]] = 0;
  }
  free(iw);
  return icode;
}

/* lu2luopt, src/pot3d.F90:4815-4868 */
static void orc_lu2luopt(orc_ctx *c) {
  long ii = 0;
  for (long i = 1; i <= c->N; i++) {
    for (int k = c->ia[i]; k <= c->dptr[i] - 1; k++) {
      ii++;
      c->lu[ii] = c->acsr[k];
      c->luja[ii] = c->ja[k];
    }
    c->n1[i] = c->dptr[i] - 1 - c->ia[i];
    c->n2[i] = c->ia[i + 1] - 2 - c->dptr[i];
  }
  for (long i = c->N; i >= 1; i--)
    for (int k = c->dptr[i] + 1; k <= c->ia[i + 1] - 1; k++) {
      ii++;
      c->lu[ii] = c->acsr[k];
      c->luja[ii] = c->ja[k];
    }
}

/* lusol, src/pot3d.F90:5227-5302 (x is the 0-based FP32 vector) */
void orc_lusol(orc_ctx *c, float *x0) {
  float *x = x0 - 1;
  long k2 = 0;
  for (long i = 1; i <= c->N; i++) {
    long k1 = k2 + 1;
    k2 = k1 + c->n1[i];
    for (long k = k1; k <= k2; k++) x[i] = x[i] - c->lu[k] * x[c->luja[k]];
  }
  for (long i = c->N; i >= 1; i--) {
    long k1 = k2 + 1;
    k2 = k1 + c->n2[i];
    for (long k = k1; k <= k2; k++) x[i] = x[i] - c->lu[k] * x[c->luja[k]];
    x[i] = x[i] * c->lud_i[i];
  }
}

/* load_preconditioner_pot3d_solve, src/pot3d.F90:4615-4715 */
static int orc_load_preconditioner(orc_ctx *c) {
  const long N = c->N;
  if (c->ifprec == 1) {
    for (long ii = 0; ii < N; ii++) c->a_i[ii] = (float)(1.0 / c->a[3 * N + ii]);
  } else if (c->ifprec == 2) {
    orc_diacsr(c);
    c->ilu_icode = orc_ilu0(c);
    orc_lu2luopt(c);
    for (long i = 1; i <= N; i++) c->lud_i[i] = (float)(1.0 / (double)c->acsr[c->dptr[i]]);
    if (c->ilu_icode) return 100;
  }
  return 0;
}

/* prec_inv, src/pot3d.F90:5152-5225 */
int orc_prec(orc_ctx *c, double *x) {
  const long N = c->N;
  if (c->ifprec == 1) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; i++) x[i] = c->a_i[i] * x[i];
  } else if (c->ifprec == 2) {
    float *x32 = (float *)malloc(sizeof(float) * N);
    for (long i = 0; i < N; i++) x32[i] = (float)x[i];
    orc_lusol(c, x32);
    for (long i = 0; i < N; i++) x[i] = (double)x32[i];
    free(x32);
  }
  return 0;
}

typedef struct {
  int nr, nt, np;
  const double *r, *dr, *rh, *drh;
  const double *t, *dt, *th, *dth, *st, *sth;
  const double *p, *dp, *ph, *dph;
} orc_mesh_in;

static double *dup1(const double *src, int n) {
  /* 1-based copy with one spare slot on each side */
  double *d = (double *)calloc(n + 2, sizeof(double));
  for (int i = 0; i < n; i++) d[i + 1] = src[i];
  return d;
}

/* Build the solve context: local mesh aux arrays (src/pot3d.F90:2710-2862),
 * coefficients and preconditioner.  br1 may be NULL (no validation BC). */
orc_ctx *orc_create(const orc_mesh_in *m, const double *br0, const double *br1, double pm_r1,
                    int ifprec, int *status) {
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->nr = m->nr;
  c->nt = m->nt;
  c->np = m->np;
  c->nrm1 = c->nr - 1;
  c->ntm1 = c->nt - 1;
  c->npm1 = c->np - 1;
  c->nrm2 = c->nr - 2;
  c->ntm2 = c->nt - 2;
  c->npm2 = c->np - 2;
  c->N = (long)c->nrm2 * c->ntm2 * c->npm2;
  c->ifprec = ifprec;
  c->pm_r1 = pm_r1;
  c->pl_i = 1.0 / (2.0 * ORC_PI - 0.0);
  c->drh = dup1(m->drh, c->nr);
  c->dth = dup1(m->dth, c->nt);
  c->dph = dup1(m->dph, c->np);
  c->st = dup1(m->st, c->ntm1);
  c->sth = dup1(m->sth, c->nt);
  c->dr = dup1(m->dr, c->nrm1);
  c->rh = dup1(m->rh, c->nr);
  c->dt = dup1(m->dt, c->ntm1);
  c->dp = dup1(m->dp, c->np);
  c->r2 = (double *)calloc(c->nrm1 + 2, sizeof(double));
  c->dr_i = (double *)calloc(c->nrm1 + 2, sizeof(double));
  for (int i = 1; i <= c->nrm1; i++) {
    c->r2[i] = m->r[i - 1] * m->r[i - 1];
    c->dr_i[i] = 1.0 / m->dr[i - 1];
  }
  c->dr1 = m->dr[0];
  c->drn = m->dr[c->nrm1 - 1];
  c->sth_i = (double *)calloc(c->nt + 2, sizeof(double));
  for (int j = 1; j <= c->nt; j++) c->sth_i[j] = 1.0 / m->sth[j - 1];
  c->dt_i = (double *)calloc(c->ntm1 + 2, sizeof(double));
  for (int j = 1; j <= c->ntm1; j++) c->dt_i[j] = 1.0 / m->dt[j - 1];
  c->dp_i = (double *)calloc(c->np + 2, sizeof(double));
  for (int k = 1; k <= c->np; k++) c->dp_i[k] = 1.0 / m->dp[k - 1];
  size_t nf = (size_t)c->nt * c->np;
  c->br0 = (double *)malloc(nf * sizeof(double));
  memcpy(c->br0, br0, nf * sizeof(double));
  if (br1) {
    c->br1 = (double *)malloc(nf * sizeof(double));
    memcpy(c->br1, br1, nf * sizeof(double));
  }
  c->a = (double *)malloc(sizeof(double) * 7 * (size_t)c->N);
  c->a_i = (float *)calloc(c->N, sizeof(float));
  c->x_ax = (double *)calloc((size_t)c->nr * c->nt * c->np, sizeof(double));
  c->sum0 = (double *)calloc(c->nr + 2, sizeof(double));
  c->sum1 = (double *)calloc(c->nr + 2, sizeof(double));
  orc_load_matrix(c);
  if (ifprec == 2) {
    c->ia = (int *)calloc(c->N + 2, sizeof(int));
    orc_getM(c);
    c->ja = (int *)calloc(c->M + 1, sizeof(int));
    c->luja = (int *)calloc(c->M + 1, sizeof(int));
    c->acsr = (float *)calloc(c->M + 1, sizeof(float));
    c->lu = (float *)calloc(c->M + 1, sizeof(float));
    c->dptr = (int *)calloc(c->N + 1, sizeof(int));
    c->n1 = (int *)calloc(c->N + 1, sizeof(int));
    c->n2 = (int *)calloc(c->N + 1, sizeof(int));
    c->lud_i = (float *)calloc(c->N + 1, sizeof(float));
  }
  *status = orc_load_preconditioner(c);
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  void *ptrs[] = {c->drh, c->dth, c->dph, c->st, c->sth, c->dr, c->rh, c->dt, c->dp, c->r2,
                  c->dr_i, c->sth_i, c->dt_i, c->dp_i, c->br0, c->br1, c->a, c->a_i, c->x_ax,
                  c->sum0, c->sum1, c->ia, c->ja, c->luja, c->acsr, c->lu, c->dptr, c->n1,
                  c->n2, c->lud_i};
  for (size_t q = 0; q < sizeof(ptrs) / sizeof(ptrs[0]); q++) free(ptrs[q]);
  free(c);
}

long orc_N(orc_ctx *c) { return c->N; }
long orc_M(orc_ctx *c) { return c->M; }
int orc_ilu_icode(orc_ctx *c) { return c->ilu_icode; }

/* Copies of the preconditioner data for kernel parity tests. */
void orc_get_ai(orc_ctx *c, float *out) { memcpy(out, c->a_i, sizeof(float) * c->N); }
void orc_get_coef(orc_ctx *c, double *out) { memcpy(out, c->a, sizeof(double) * 7 * c->N); }
/* The U diagonal after ILU0 and its FP32 inverse, 0-based. */
void orc_get_ilu_diag(orc_ctx *c, float *d, float *dinv) {
  for (long i = 1; i <= c->N; i++) {
    d[i - 1] = c->acsr[c->dptr[i]];
    dinv[i - 1] = c->lud_i[i];
  }
}
/* The 1-based CSR (before factorisation the caller builds its own copy). */
void orc_get_csr(orc_ctx *c, int *ia, int *ja, float *lu) {
  memcpy(ia, c->ia + 1, sizeof(int) * (c->N + 1));
  memcpy(ja, c->ja + 1, sizeof(int) * (c->M - 1));
  memcpy(lu, c->acsr + 1, sizeof(float) * (c->M - 1));
}
/* CSR of A with boundary couplings dropped, before factorisation. */
void orc_build_csr(orc_ctx *c, int *ia, int *ja, float *a) {
  int *sia = c->ia, *sja = c->ja;
  float *sa = c->acsr;
  int *sd = c->dptr;
  int *tia = (int *)calloc(c->N + 2, sizeof(int));
  c->ia = tia;
  orc_getM(c);
  c->ja = (int *)calloc(c->M + 1, sizeof(int));
  c->acsr = (float *)calloc(c->M + 1, sizeof(float));
  c->dptr = (int *)calloc(c->N + 1, sizeof(int));
  orc_diacsr(c);
  memcpy(ia, c->ia + 1, sizeof(int) * (c->N + 1));
  memcpy(ja, c->ja + 1, sizeof(int) * (c->M - 1));
  memcpy(a, c->acsr + 1, sizeof(float) * (c->M - 1));
  free(c->ia);
  free(c->ja);
  free(c->acsr);
  free(c->dptr);
  c->ia = sia;
  c->ja = sja;
  c->acsr = sa;
  c->dptr = sd;
}
/* Standalone ILU0 of a caller-supplied 1-based CSR (in place), for checking
 * the legacy load_external_lu_solver factorisation. */
int orc_ilu0_csr(long N, int *ia0, int *ja0, float *a0, int *dptr0) {
  orc_ctx tmp;
  memset(&tmp, 0, sizeof(tmp));
  tmp.N = N;
  tmp.ia = ia0 - 1;
  tmp.ja = ja0 - 1;
  tmp.acsr = a0 - 1;
  tmp.dptr = dptr0 - 1;
  return orc_ilu0(&tmp);
}

/* RHS by the boundary trick, src/pot3d.F90:3937-3950 */
int orc_rhs(orc_ctx *c, double *rhs) {
  memset(c->x_ax, 0, sizeof(double) * (size_t)c->nr * c->nt * c->np);
  orc_set_boundary_points(c, c->x_ax, 1.0);
  orc_seam(c, c->x_ax);
  orc_delsq(c, c->x_ax, rhs);
  for (long i = 0; i < c->N; i++) rhs[i] = -rhs[i];
  return 0;
}

/*
 * cgsolve + ernorm, src/pot3d.F90:4231-4485.  x: guess in / solution out;
 * r: RHS in / residual out.  Returns ierr (0 converged, 1 ncgmax exceeded).
 * The convergence history (every ncghist iterations, and the final one)
 * is written to hist_it/hist_eps when provided.
 */
int orc_cgsolve(orc_ctx *c, double *x, double *r, int ncgmax, double epscg, int ncghist,
                int *ncg_out, double *epsn_out, int *hist_n, int *hist_it, double *hist_eps,
                int hist_cap) {
  const long N = c->N;
  double *p = (double *)malloc(sizeof(double) * N);
  double *ap = (double *)malloc(sizeof(double) * N);
  int ncg = 0, ierr = -1, nh = 0;
  double epsn = 0.0;
#define ERNORM()                                                          \
  do {                                                                    \
    double epssq = rdotr / bdotb;                                         \
    epsn = (epssq >= 0 ? 1.0 : -1.0) * sqrt(fabs(epssq));                 \
    ierr = -1;                                                            \
    int logit = ncghist > 0 && (ncg % ncghist) == 0;                      \
    if (epsn < epscg) {                                                   \
      ierr = 0;                                                           \
      if (ncghist > 0) logit = 1;                                         \
    } else if (ncg >= ncgmax) {                                           \
      ierr = 1;                                                           \
    }                                                                     \
    if (logit && hist_it && nh < hist_cap) {                              \
      hist_it[nh] = ncg;                                                  \
      hist_eps[nh] = epsn;                                                \
      nh++;                                                               \
    }                                                                     \
  } while (0)
  for (long i = 0; i < N; i++) p[i] = r[i];
  orc_prec(c, p);
  double bdotb = orc_dot(r, p, N);
  double rdotr;
  if (bdotb == 0.) {
    for (long i = 0; i < N; i++) x[i] = 0.;
    epsn = 0.;
    ierr = 0;
    goto done;
  }
  orc_ax(c, x, ap);
  for (long i = 0; i < N; i++) {
    r[i] = r[i] - ap[i];
    p[i] = r[i];
  }
  orc_prec(c, p);
  rdotr = orc_dot(r, p, N);
  ERNORM();
  if (ierr >= 0) goto done;
  for (;;) {
    ncg = ncg + 1;
    orc_ax(c, p, ap);
    double pdotap = orc_dot(p, ap, N);
    double alphai = rdotr / pdotap;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; i++) {
      x[i] = x[i] + alphai * p[i];
      r[i] = r[i] - alphai * ap[i];
      ap[i] = r[i];
    }
    orc_prec(c, ap);
    double rdotr_old = rdotr;
    rdotr = orc_dot(r, ap, N);
    ERNORM();
    if (ierr >= 0) break;
    double betai = rdotr / rdotr_old;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; i++) p[i] = betai * p[i] + ap[i];
  }
#undef ERNORM
done:
  free(p);
  free(ap);
  *ncg_out = ncg;
  *epsn_out = epsn;
  if (hist_n) *hist_n = nh;
  return ierr;
}

/* Final phi with ghosts, src/pot3d.F90:3966-3969 */
int orc_finalize_phi(orc_ctx *c, const double *x, double *phi) {
  memset(phi, 0, sizeof(double) * (size_t)c->nr * c->nt * c->np);
  orc_unpack(c, phi, x);
  orc_set_boundary_points(c, phi, 1.0);
  orc_seam(c, phi);
  return 0;
}

/* getb + magnetic_energy, src/pot3d.F90:6187-6321 (B evaluated in place). */
int orc_energy(orc_ctx *c, const double *phi, double *w) {
  const int nrm1 = c->nrm1, ntm1 = c->ntm1, npm1 = c->npm1;
  const double *dr = c->dr, *rh = c->rh, *dt = c->dt, *sth = c->sth, *dp = c->dp;
  const double *drh = c->drh, *dth = c->dth, *dph = c->dph;
  const double half = .5;
  int nk = npm1 - 1;
  double *pw = (double *)calloc(3 * (size_t)(nk + 1), sizeof(double));
#define BR(i, j, k) ((XA(phi, (i) + 1, j, k) - XA(phi, i, j, k)) / dr[i])
#define BT(i, j, k) ((XA(phi, i, (j) + 1, k) - XA(phi, i, j, k)) / (rh[i] * dt[j]))
#define BP(i, j, k) ((XA(phi, i, j, (k) + 1) - XA(phi, i, j, k)) / (rh[i] * sth[j] * dp[k]))
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= npm1; k++) {
    double wr = 0., wt = 0., wp = 0.;
    for (int j = 2; j <= ntm1; j++)
      for (int i = 2; i <= nrm1; i++) {
        double dv = rh[i] * rh[i] * drh[i] * dth[j] * sth[j] * dph[k];
        double brav = half * (BR(i, j, k) + BR(i - 1, j, k));
        double btav = half * (BT(i, j, k) + BT(i, j - 1, k));
        double bpav = half * (BP(i, j, k) + BP(i, j, k - 1));
        wr = wr + half * (brav * brav) * dv;
        wt = wt + half * (btav * btav) * dv;
        wp = wp + half * (bpav * bpav) * dv;
      }
    pw[3 * (k - 2) + 0] = wr;
    pw[3 * (k - 2) + 1] = wt;
    pw[3 * (k - 2) + 2] = wp;
  }
#undef BR
#undef BT
#undef BP
  w[0] = w[1] = w[2] = 0.;
  for (int k = 0; k < nk; k++) {
    w[0] += pw[3 * k + 0];
    w[1] += pw[3 * k + 1];
    w[2] += pw[3 * k + 2];
  }
  free(pw);
  return 0;
}

/* getb, src/pot3d.F90:6187-6233: B on the staggered meshes, every point the
 * reference fills.  br is (nrm1,nt,np), bt (nr,ntm1,np), bp (nr,nt,npm1),
 * column-major; the products in the denominators round left to right. */
int orc_getb(orc_ctx *c, const double *phi, double *br, double *bt, double *bp) {
  const int nr = c->nr, nt = c->nt, np = c->np, nrm1 = c->nrm1, ntm1 = c->ntm1, npm1 = c->npm1;
  const double *dr = c->dr, *rh = c->rh, *dt = c->dt, *sth = c->sth, *dp = c->dp;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= np; k++)
    for (int j = 1; j <= nt; j++)
      for (int i = 1; i <= nrm1; i++)
        br[(i - 1) + (size_t)nrm1 * ((j - 1) + (size_t)nt * (k - 1))] =
            (XA(phi, i + 1, j, k) - XA(phi, i, j, k)) / dr[i];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= np; k++)
    for (int j = 1; j <= ntm1; j++)
      for (int i = 1; i <= nr; i++)
        bt[(i - 1) + (size_t)nr * ((j - 1) + (size_t)ntm1 * (k - 1))] =
            (XA(phi, i, j + 1, k) - XA(phi, i, j, k)) / (rh[i] * dt[j]);
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= npm1; k++)
    for (int j = 1; j <= nt; j++)
      for (int i = 1; i <= nr; i++)
        bp[(i - 1) + (size_t)nr * ((j - 1) + (size_t)nt * (k - 1))] =
            (XA(phi, i, j, k + 1) - XA(phi, i, j, k)) / (rh[i] * sth[j] * dp[k]);
  return 0;
}

int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
