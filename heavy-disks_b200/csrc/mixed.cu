// Mixed-precision path: placeholder until the FP32-perturbation kernels land.
#include "engine.h"

struct MixedState {};

#define MX_UNSUPPORTED return fail(DG_ERR_UNSUPPORTED, "mixed precision", "not built yet")
int dg_handle::mixed_init() { MX_UNSUPPORTED; }
void dg_handle::mixed_release() {}
int dg_handle::mixed_enqueue_step() { MX_UNSUPPORTED; }
int dg_handle::mixed_enqueue_step_forces(const double *, const double *) { MX_UNSUPPORTED; }
int dg_handle::mixed_cfl_launch(int, int) { MX_UNSUPPORTED; }
int dg_handle::mixed_modes_launch(int, double *) { MX_UNSUPPORTED; }
int dg_handle::mixed_conserved_launch(double *) { MX_UNSUPPORTED; }
int dg_handle::mixed_upload_state(const double *, const double *, const double *) { MX_UNSUPPORTED; }
int dg_handle::mixed_download_state(double *, double *, double *) { MX_UNSUPPORTED; }
