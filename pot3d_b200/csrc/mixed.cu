// FP32-refined PCG (placeholder).
#include "pot3d_solver.h"
namespace pot3d {
int mixed_setup(Solver *) {
  pot3d_set_error("FP32-refined mode is not available in this build");
  return POT3D_ERR_ARG;
}
void mixed_destroy(Solver *) {}
int mixed_solve(Solver *, bool, int, double, int *, pot3d_solve_info_t *) { return POT3D_ERR_ARG; }
}  // namespace pot3d
