// ILU(0) preconditioner (placeholder until the wavefront sweeps land).
#include "pot3d_solver.h"
namespace pot3d {
int dilu_setup(Solver *) {
  pot3d_set_error("ifprec=2 is not available in this build");
  return POT3D_ERR_ARG;
}
void dilu_destroy(Solver *) {}
float *dilu_r32(Solver *) { return nullptr; }
float *dilu_z32(Solver *) { return nullptr; }
int dilu_sweeps(Solver *, bool) { return POT3D_ERR_ARG; }
int dilu_diag(Solver *, float *, float *) { return POT3D_ERR_ARG; }
int dilu_sweep_launches(Solver *) { return 0; }
}  // namespace pot3d
