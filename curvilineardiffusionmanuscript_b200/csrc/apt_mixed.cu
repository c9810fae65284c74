// apt_mixed.cu — FP32 correction sweeps with FP64 residual and defect-correction restarts.
#include "engine.h"

namespace cdm {

int Engine::mixed_alloc() {
  set_error("mixed precision is not available in this build");
  return CDM_BAD_INPUT;
}

int Engine::step_mixed(const cdm_step_opts*, double, double) {
  set_error("mixed precision is not available in this build");
  return CDM_BAD_INPUT;
}

}  // namespace cdm
