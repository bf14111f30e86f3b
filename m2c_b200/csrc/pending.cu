// Entry points whose device implementation has not landed in this build:
// they report M2CG_ERR_UNSUPPORTED instead of computing anything.
#include "../../include/m2c_gpu.h"

extern "C" m2cg_status m2cg_batch_create(const m2cg_scheme*, int, const int*, const m2cg_material*, const double*,
                                         const double*, const m2cg_batch_tuning*, m2cg_batch** out) {
  if (out) *out = nullptr;
  return M2CG_ERR_UNSUPPORTED;
}
extern "C" m2cg_status m2cg_batch_run(m2cg_batch*, int) { return M2CG_ERR_UNSUPPORTED; }
extern "C" m2cg_status m2cg_batch_download(m2cg_batch*, double*, int*, double*) { return M2CG_ERR_UNSUPPORTED; }
extern "C" m2cg_status m2cg_batch_get_tuning(const m2cg_batch*, m2cg_batch_tuning*) { return M2CG_ERR_UNSUPPORTED; }
extern "C" m2cg_status m2cg_batch_destroy(m2cg_batch*) { return M2CG_OK; }
