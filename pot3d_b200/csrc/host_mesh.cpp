// Host-side input builders for the pot3d_gpu solve (see include/pot3d_host.h).
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/pot3d_host.h"

namespace {

constexpr double kPi = 3.1415926535897932;  // constants module, src/pot3d.F90:106

// fold, src/pot3d.F90:3707-3752: map x into [x0, x1).
double fold_into(double x0, double x1, double x) {
  if (x0 == x1) return x;
  const double len = x1 - x0;
  double f = std::fmod(x - x0, len) + x0;
  if (f < x0) f += len;
  if (f >= x1) f -= len;
  return f;
}

// Segment description of the piecewise-exponential mapping xi -> c.
struct Segments {
  std::vector<double> cs;     // segment limits in c (n+1)
  std::vector<double> ratio;  // spacing ratio end/start per segment (n)
  std::vector<double> xi;     // segment limits in xi (n+1)
  std::vector<double> amp;    // log(ratio)/dxi per segment (n)
  int n() const { return (int)ratio.size(); }
};

// Locate the segment of v in the limits lim (closed intervals, first hit).
int find_segment(const std::vector<double> &lim, double v) {
  for (size_t s = 0; s + 1 < lim.size(); s++)
    if (v >= lim[s] && v <= lim[s + 1]) return (int)s;
  return -1;
}

// map_xi_to_c, src/pot3d.F90:3374-3492.
int xi_to_c(const Segments &S, bool periodic, double cshift, double xishift, double xv, double *cv) {
  const double tiny = 1.e-5;
  const double xp = periodic ? fold_into(0.0, 1.0, xv + xishift) : xv;
  const int s = find_segment(S.xi, xp);
  if (s < 0) return -1;
  const double d = xp - S.xi[s], d1 = S.xi[s + 1] - S.xi[s];
  const double da = S.amp[s] * d, da1 = S.amp[s] * d1;
  double fac;
  if (std::fabs(da1) < tiny)
    fac = (d * (1.0 + 0.5 * da)) / (d1 * (1.0 + 0.5 * da1));
  else
    fac = (std::exp(da) - 1.0) / (S.ratio[s] - 1.0);
  double c = S.cs[s] + (S.cs[s + 1] - S.cs[s]) * fac;
  if (periodic) c = fold_into(S.cs.front(), S.cs.back(), c - cshift);
  *cv = c;
  return 0;
}

// map_c_to_xi, src/pot3d.F90:3494-3586.
int c_to_xi(const Segments &S, bool periodic, double cv, double *xv) {
  const double tiny = 1.e-5;
  const double cp = periodic ? fold_into(S.cs.front(), S.cs.back(), cv) : cv;
  const int s = find_segment(S.cs, cp);
  if (s < 0) return -1;
  const double d = (cp - S.cs[s]) / (S.cs[s + 1] - S.cs[s]);
  const double da = (S.ratio[s] - 1.0) * d;
  const double fac = (std::fabs(da) < tiny) ? d * (S.xi[s + 1] - S.xi[s]) : std::log(da + 1.0) / S.amp[s];
  *xv = S.xi[s] + fac;
  return 0;
}

}  // namespace

extern "C" int pot3d_host_genmesh(int nc, double c0, double c1, int nseg, const double *frac,
                                  const double *dratio, int nfilt, int periodic, double c_shift, double *c) {
  const double tiny = 1.e-5;
  if (nc < 2) return 1;
  if (c0 >= c1) return 2;
  // Number of FRAC values given: up to the first zero after the first entry.
  int nf = nseg;
  for (int q = 1; q < nseg; q++)
    if (frac[q] == 0.0) {
      nf = q;
      break;
    }
  Segments S;
  if (nf == 1 && frac[0] == 0.0) {  // uniform mesh
    S.cs = {c0, c1};
    S.ratio = {1.0};
  } else {
    for (int q = 1; q < nf; q++)
      if (frac[q] < frac[q - 1]) return 3;
    if (periodic) {
      if (frac[0] < 0.0 || frac[nf - 1] > 1.0) return 4;
      if (frac[0] == 0.0 && frac[nf - 1] == 1.0) return 5;
    } else {
      if (frac[0] != 0.0) return 6;
      if (frac[nf - 1] != 1.0) return 7;
    }
    const int nratio = periodic ? nf : nf - 1;
    for (int q = 0; q < nratio; q++)
      if (dratio[q] <= 0.0) return 8;
    const double span = c1 - c0;
    if (!periodic) {
      for (int q = 0; q < nf; q++) S.cs.push_back(c0 + span * frac[q]);
      S.ratio.assign(dratio, dratio + nratio);
    } else if (frac[0] == 0.0) {
      for (int q = 0; q < nf; q++) S.cs.push_back(c0 + span * frac[q]);
      S.cs.push_back(c1);
      S.ratio.assign(dratio, dratio + nratio);
    } else {
      // A leading segment from c0 to the first FRAC point; the wrap-around
      // segment (last ratio) is split between the two ends if 1 is absent.
      S.cs.push_back(c0);
      for (int q = 0; q < nf; q++) S.cs.push_back(c0 + span * frac[q]);
      const double last = dratio[nratio - 1];
      if (frac[nf - 1] != 1.0) {
        const double alpha = (1.0 - frac[nf - 1]) / (frac[0] + 1.0 - frac[nf - 1]);
        const double split = 1.0 + alpha * (last - 1.0);
        S.cs.push_back(c1);
        S.ratio.push_back(last / split);
        for (int q = 0; q < nratio; q++) S.ratio.push_back(dratio[q]);
        S.ratio.back() = split;
      } else {
        S.ratio.push_back(last);
        for (int q = 0; q + 1 < nratio; q++) S.ratio.push_back(dratio[q]);
      }
    }
  }
  const int ns = S.n();
  // Segment lengths in xi (f), total, xi limits and amplification factors.
  std::vector<double> f(ns);
  for (int s = 0; s < ns; s++) {
    const double dr = S.ratio[s] - 1.0;
    const double w = S.cs[s + 1] - S.cs[s];
    f[s] = (std::fabs(dr) < tiny) ? w * (1.0 + 0.5 * dr) : w * std::log(S.ratio[s]) / dr;
  }
  double total = 0.0;
  for (int s = ns - 1; s >= 0; s--) total = total / S.ratio[s] + f[s];
  S.xi.assign(ns + 1, 0.0);
  double step = f[0] / total;
  for (int s = 1; s < ns; s++) {
    S.xi[s] = S.xi[s - 1] + step;
    if (s < ns - 1) step = step * f[s] / (f[s - 1] * S.ratio[s - 1]);
  }
  S.xi[ns] = 1.0;
  S.amp.resize(ns);
  for (int s = 0; s < ns; s++) S.amp[s] = std::log(S.ratio[s]) / (S.xi[s + 1] - S.xi[s]);
  double cshift = 0.0, xishift = 0.0;
  if (periodic) {
    cshift = -c_shift;
    if (c_to_xi(S, true, cshift, &xishift)) return 9;
  }
  const double dxi = 1.0 / (nc - 1.0);
  c[0] = c0;
  for (int q = 1; q < nc - 1; q++)
    if (xi_to_c(S, periodic != 0, cshift, xishift, q * dxi, &c[q])) return 9;
  c[nc - 1] = c1;
  // (1,2,1)/4 filters, src/pot3d.F90:3588-3705.
  std::vector<double> tmp(nc + 2);
  for (int pass = 0; pass < nfilt; pass++) {
    if (periodic) {
      const double keep = c[0], len = c1 - c0;
      tmp[0] = c[nc - 2] - len;
      for (int q = 0; q < nc; q++) tmp[q + 1] = c[q];
      tmp[nc + 1] = c[1] + len;
      for (int q = 0; q < nc; q++) c[q] = 0.25 * (tmp[q] + 2.0 * tmp[q + 1] + tmp[q + 2]);
      const double moved = c[0];
      for (int q = 0; q < nc; q++) c[q] = c[q] - moved + keep;
    } else {
      for (int q = 0; q < nc; q++) tmp[q] = c[q];
      for (int q = 1; q < nc - 1; q++) c[q] = 0.25 * (tmp[q - 1] + 2.0 * tmp[q] + tmp[q + 1]);
    }
  }
  return 0;
}

// Half mesh and spacings of a non-periodic coordinate (src/pot3d.F90:2618-2629).
static void half_mesh(int n, const double *c, double *ch, double *dch, double *dc) {
  // c has n-1 points; ch, dch have n; dc has n-1.
  for (int q = 1; q < n - 1; q++) {
    ch[q] = .5 * (c[q] + c[q - 1]);
    dch[q] = c[q] - c[q - 1];
  }
  ch[0] = ch[1] - dch[1];
  ch[n - 1] = ch[n - 2] + dch[n - 2];
  dch[0] = dch[1];
  dch[n - 1] = dch[n - 2];
  for (int q = 0; q < n - 1; q++) dc[q] = ch[q + 1] - ch[q];
}

extern "C" int pot3d_host_mesh(pot3d_mesh_buf_t *m, double r0, double r1, int nseg, const double *rfrac,
                               const double *drratio, int nfrmesh, const double *tfrac, const double *dtratio,
                               int nftmesh, const double *pfrac, const double *dpratio, int nfpmesh,
                               double phishift) {
  const int nr = m->nr, nt = m->nt, np = m->np;
  int rc = pot3d_host_genmesh(nr - 1, r0, r1, nseg, rfrac, drratio, nfrmesh, 0, 0.0, m->r);
  if (rc) return 10 + rc;
  half_mesh(nr, m->r, m->rh, m->drh, m->dr);
  rc = pot3d_host_genmesh(nt - 1, 0.0, kPi, nseg, tfrac, dtratio, nftmesh, 0, 0.0, m->t);
  if (rc) return 20 + rc;
  half_mesh(nt, m->t, m->th, m->dth, m->dt);
  // Periodic phi (src/pot3d.F90:2651-2675).
  const double pl = 2.0 * kPi;
  rc = pot3d_host_genmesh(np - 1, 0.0, pl, nseg, pfrac, dpratio, nfpmesh, 1, phishift, m->p);
  if (rc) return 30 + rc;
  m->p[np - 1] = m->p[1] + pl;
  for (int k = 1; k < np; k++) {
    m->ph[k] = 0.5 * (m->p[k] + m->p[k - 1]);
    m->dph[k] = m->p[k] - m->p[k - 1];
  }
  m->ph[0] = m->ph[np - 2] - pl;
  m->dph[0] = m->dph[np - 2];
  for (int k = 0; k < np - 1; k++) m->dp[k] = m->ph[k + 1] - m->ph[k];
  m->dp[np - 1] = m->dp[1];
  m->dph[np - 1] = m->dph[1];
  m->dp[0] = m->dp[np - 2];
  for (int j = 0; j < nt - 1; j++) m->st[j] = std::sin(m->t[j]);
  for (int j = 0; j < nt; j++) m->sth[j] = std::sin(m->th[j]);
  return 0;
}

// Bracket v in the increasing table x (interp, src/pot3d.F90:7028-7072).
static int bracket(const double *x, int n, double v, int *i0, double *w) {
  for (int q = 0; q + 1 < n; q++)
    if (v >= x[q] && v <= x[q + 1]) {
      *i0 = q;
      *w = (v - x[q]) / (x[q + 1] - x[q]);
      return 0;
    }
  return -1;
}

extern "C" int pot3d_host_br0(const pot3d_mesh_buf_t *m, int ntn, int npn, const double *tn, const double *pn,
                              const double *fi, int option, int do_not_balance_flux, double *br0) {
  const int nt = m->nt, np = m->np;
  auto B = [&](int j, int k) -> double & { return br0[j + (size_t)nt * k]; };
  auto F = [&](int a, int b) { return fi[a + (size_t)ntn * b]; };
  for (int q = 1; q < ntn; q++)
    if (!(tn[q] > tn[q - 1])) return 1;
  for (int q = 1; q < npn; q++)
    if (!(pn[q] > pn[q - 1])) return 1;
  // intrp2d onto th(2:ntm1) x ph(2:npm1)  (src/pot3d.F90:6833-6932)
  for (int k = 1; k < np - 1; k++) {
    int kb;
    double ay;
    if (bracket(pn, npn, m->ph[k], &kb, &ay)) return 2;
    for (int j = 1; j < nt - 1; j++) {
      int jb;
      double ax;
      if (bracket(tn, ntn, m->th[j], &jb, &ax)) return 2;
      B(j, k) = (1. - ax) * ((1. - ay) * F(jb, kb) + ay * F(jb, kb + 1)) +
                ax * ((1. - ay) * F(jb + 1, kb) + ay * F(jb + 1, kb + 1));
    }
  }
  for (int j = 0; j < nt; j++) {  // periodic copy
    B(j, 0) = B(j, np - 2);
    B(j, np - 1) = B(j, 1);
  }
  const double pl_i = 1.0 / (2.0 * kPi);  // m=0 values at the poles
  double n0 = 0.0, n1 = 0.0;
  for (int k = 1; k < np - 1; k++) n0 += B(1, k) * m->dph[k];
  for (int k = 1; k < np - 1; k++) n1 += B(nt - 2, k) * m->dph[k];
  n0 *= pl_i;
  n1 *= pl_i;
  for (int k = 0; k < np; k++) {
    B(0, k) = 2.0 * n0 - B(1, k);
    B(nt - 1, k) = 2.0 * n1 - B(nt - 2, k);
  }
  double area = 0.0, fp = 0.0, fm = 0.0;  // flux balance (src/pot3d.F90:6800-6829)
  for (int j = 1; j < nt - 1; j++)
    for (int k = 1; k < np - 1; k++) {
      const double da = m->sth[j] * m->dth[j] * m->dph[k];
      if (B(j, k) > 0.)
        fp = fp + B(j, k) * da;
      else
        fm = fm + B(j, k) * da;
      area = area + da;
    }
  if (!((option == 1 || option == 2) && do_not_balance_flux)) {
    const double off = (fp + fm) / area;
    for (int k = 0; k < np; k++)
      for (int j = 0; j < nt; j++) B(j, k) = B(j, k) - off;
  }
  if (option == 1)  // 'open': monopole trick (src/pot3d.F90:3832)
    for (size_t q = 0; q < (size_t)nt * np; q++) br0[q] = std::fabs(br0[q]);
  return 0;
}

// ---- synthetic maps --------------------------------------------------------
namespace {
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double normal() {  // Box-Muller, one value per call
    const double u1 = 1.0 - uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
  }
};
}  // namespace

extern "C" int pot3d_host_synthetic_br(unsigned long long seed, int lmax, int nbip, int ntn, int npn, double *tn,
                                       double *pn, double *fi) {
  if (ntn < 3 || npn < 3 || lmax < 1) return 1;
  SplitMix64 rng{seed};
  for (int j = 0; j < ntn; j++) tn[j] = kPi * j / (ntn - 1);
  for (int k = 0; k < npn; k++) pn[k] = 2.0 * kPi * k / (npn - 1);
  // Coefficients: for l=1..lmax, m=0..l: a_l0; (a_lm, b_lm) for m>0.
  const int L = lmax;
  std::vector<double> ac((L + 1) * (L + 1), 0.0), as((L + 1) * (L + 1), 0.0);
  for (int l = 1; l <= L; l++)
    for (int m = 0; m <= l; m++) {
      const double s = 1.0 / ((double)l * l);
      ac[l * (L + 1) + m] = rng.normal() * s;
      if (m > 0) as[l * (L + 1) + m] = rng.normal() * s;
    }
  // Per theta row: F_m(theta) = sum_l a_lm Pbar_lm(cos theta), orthonormal
  // associated Legendre functions by the standard three-term recurrence.
  std::vector<double> Fc((size_t)ntn * (L + 1)), Fs((size_t)ntn * (L + 1));
  std::vector<double> pmm(L + 2);
  for (int j = 0; j < ntn; j++) {
    const double x = std::cos(tn[j]), sx = std::sin(tn[j]);
    double p_mm = 1.0 / std::sqrt(4.0 * kPi);
    for (int m = 0; m <= L; m++) {
      if (m > 0) p_mm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * sx;
      double pl2 = 0.0, pl1 = p_mm, fc = 0.0, fs = 0.0;
      const double norm = (m == 0) ? 1.0 : std::sqrt(2.0);
      for (int l = m; l <= L; l++) {
        double pl;
        if (l == m) {
          pl = p_mm;
        } else if (l == m + 1) {
          pl = std::sqrt(2.0 * m + 3.0) * x * p_mm;
        } else {
          const double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
          const double b = std::sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
          pl = a * (x * pl1 - b * pl2);
        }
        if (l > m) {
          pl2 = pl1;
          pl1 = pl;
        }
        if (l >= 1) {
          fc += norm * ac[l * (L + 1) + m] * pl;
          fs += norm * as[l * (L + 1) + m] * pl;
        }
        if (l == m) {
          pl2 = 0.0;
          pl1 = pl;
        }
      }
      Fc[(size_t)j * (L + 1) + m] = fc;
      Fs[(size_t)j * (L + 1) + m] = fs;
    }
  }
  double wsum = 0.0, ssq = 0.0;
  std::vector<double> cm(L + 1), sm(L + 1);
  for (int k = 0; k < npn; k++) {
    for (int m = 0; m <= L; m++) {
      cm[m] = std::cos(m * pn[k]);
      sm[m] = std::sin(m * pn[k]);
    }
    for (int j = 0; j < ntn; j++) {
      double v = 0.0;
      for (int m = 0; m <= L; m++) v += Fc[(size_t)j * (L + 1) + m] * cm[m] + Fs[(size_t)j * (L + 1) + m] * sm[m];
      fi[j + (size_t)ntn * k] = v;
      const double w = std::sin(tn[j]);
      wsum += w;
      ssq += w * v * v;
    }
  }
  const double rms = std::sqrt(ssq / wsum);
  const double scale = rms > 0 ? 5.0 / rms : 0.0;
  for (size_t q = 0; q < (size_t)ntn * npn; q++) fi[q] *= scale;
  // Bipoles: two Gaussian spots of opposite sign.
  const double deg = kPi / 180.0, sig = 3.0 * deg, half_sep = 3.0 * deg;
  for (int b = 0; b < nbip; b++) {
    const double lat = (-35.0 + 70.0 * rng.uniform()) * deg;
    const double lon = 360.0 * rng.uniform() * deg;
    const double tilt = (-20.0 + 40.0 * rng.uniform()) * deg;
    const double sgn = rng.uniform() < 0.5 ? 1.0 : -1.0;
    for (int side = 0; side < 2; side++) {
      const double sd = side == 0 ? 1.0 : -1.0;
      const double slat = lat + sd * half_sep * std::sin(tilt);
      const double slon = lon + sd * half_sep * std::cos(tilt) / std::cos(lat);
      const double amp = 50.0 * sgn * sd;
      const double cl = std::cos(slat), sl = std::sin(slat);
      for (int k = 0; k < npn; k++)
        for (int j = 0; j < ntn; j++) {
          const double plat = 0.5 * kPi - tn[j];
          double c = sl * std::sin(plat) + cl * std::cos(plat) * std::cos(pn[k] - slon);
          c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
          const double d = std::acos(c);
          fi[j + (size_t)ntn * k] += amp * std::exp(-0.5 * (d * d) / (sig * sig));
        }
    }
  }
  // Remove the area-weighted mean so the net flux vanishes.
  double num = 0.0;
  for (int k = 0; k < npn - 1; k++)
    for (int j = 0; j < ntn; j++) num += std::sin(tn[j]) * fi[j + (size_t)ntn * k];
  double den = 0.0;
  for (int k = 0; k < npn - 1; k++)
    for (int j = 0; j < ntn; j++) den += std::sin(tn[j]);
  const double mean = num / den;
  for (size_t q = 0; q < (size_t)ntn * npn; q++) fi[q] -= mean;
  return 0;
}
