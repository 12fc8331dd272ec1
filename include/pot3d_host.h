/*
 * pot3d_host.h -- host-side helpers of libpot3d_gpu.so (no GPU needed).
 *
 * In the drop-in configuration the Fortran host computes these itself; the
 * helpers let a C/C++/Python caller without the Fortran code build the same
 * inputs for the pot3d_gpu_* solve:
 *  - the 1-D meshes of set_global_mesh/genmesh (src/pot3d.F90:2583-2708,
 *    2864-3752) at one rank;
 *  - the boundary map br0 of readbr/set_flux (src/pot3d.F90:6672-6831,
 *    3754-3864): bilinear interpolation, periodic copy, pole m=0 values,
 *    flux balance and the |Br| of option 'open';
 *  - seeded synthetic Br maps (random real spherical harmonics plus
 *    Gaussian bipoles, zero net flux) for benchmarks and tests.
 * All functions return 0 on success, nonzero where the reference stops.
 */
#ifndef POT3D_HOST_H
#define POT3D_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

/* Output buffers for one rank's mesh, caller-allocated with the lengths of
 * pot3d_mesh_t (include/pot3d_gpu.h); same field order. */
typedef struct {
  int nr, nt, np;
  double *r, *dr;
  double *rh, *drh;
  double *t, *dt, *st;
  double *th, *dth, *sth;
  double *p, *dp;
  double *ph, *dph;
} pot3d_mesh_buf_t;

/* genmesh, src/pot3d.F90:2864-3372: nc points of a segmented exponential
 * mesh on [c0,c1]; frac/dratio hold nseg values (unused ones 0). */
int pot3d_host_genmesh(int nc, double c0, double c1, int nseg, const double *frac,
                       const double *dratio, int nfilt, int periodic, double c_shift,
                       double *c);

/* set_global_mesh, src/pot3d.F90:2583-2708 (theta on [0,pi], periodic phi on
 * [0,2pi]).  nseg values in each frac/ratio array. */
int pot3d_host_mesh(pot3d_mesh_buf_t *m, double r0, double r1, int nseg, const double *rfrac,
                    const double *drratio, int nfrmesh, const double *tfrac, const double *dtratio,
                    int nftmesh, const double *pfrac, const double *dpratio, int nfpmesh,
                    double phishift);

/* readbr + set_flux on a mesh: fi(ntn,npn) column-major with scales tn, pn
 * -> br0(nt,np) column-major.  option: 0 'potential', 1 'open', 2 'ss'. */
int pot3d_host_br0(const pot3d_mesh_buf_t *m, int ntn, int npn, const double *tn, const double *pn,
                   const double *fi, int option, int do_not_balance_flux, double *br0);

/* Seeded synthetic Br(theta,phi) on a uniform ntn x npn grid with theta in
 * [0,pi] and phi in [0,2pi]: orthonormal real spherical harmonics l=1..lmax
 * with N(0,1)/l^2 coefficients scaled to an area-weighted RMS of 5 G, plus
 * nbip Gaussian bipoles (sigma 3 deg, +-50 G, centre latitude in
 * [-35,35] deg, 6 deg separation, tilt in [-20,20] deg), then the
 * area-weighted mean removed.  Outputs tn(ntn), pn(npn), fi(ntn,npn). */
int pot3d_host_synthetic_br(unsigned long long seed, int lmax, int nbip, int ntn, int npn,
                            double *tn, double *pn, double *fi);

#ifdef __cplusplus
}
#endif

#endif /* POT3D_HOST_H */
