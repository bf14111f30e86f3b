// Two-material machinery (placeholder until the level-set path lands).
#include "multiphase.h"

namespace m2c {
struct Multiphase {
  int dummy;
};
}  // namespace m2c

m2cg_status multiphase_create(cudaStream_t, const m2c::Grid3&, const m2c::SchemeK&, const m2cg_scheme&,
                              const m2cg_material*, int, const m2cg_levelset&, Multiphase** out) {
  *out = nullptr;
  return M2CG_ERR_UNSUPPORTED;
}
void multiphase_destroy(Multiphase* mp) { delete mp; }
m2cg_status multiphase_upload_phi(Multiphase*, cudaStream_t, const double*, double*, uint8_t*) { return M2CG_ERR_UNSUPPORTED; }
m2cg_status multiphase_download_phi(Multiphase*, cudaStream_t, double*) { return M2CG_ERR_UNSUPPORTED; }
void multiphase_set_step(Multiphase*, int) {}
m2cg_status multiphase_begin_step(Multiphase*, cudaStream_t, double* const*, const uint8_t*) { return M2CG_ERR_UNSUPPORTED; }
m2cg_status multiphase_stage(Multiphase*, cudaStream_t, m2c::StageArgs&) { return M2CG_ERR_UNSUPPORTED; }
m2cg_status multiphase_end_step(Multiphase*, cudaStream_t, double* const*, double* const*, uint8_t*, const double*,
                                m2c::DevError*, m2cg_counters*) {
  return M2CG_ERR_UNSUPPORTED;
}
void multiphase_counters(const Multiphase*, m2cg_counters*) {}
