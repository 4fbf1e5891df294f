// tune.cu -- kernel-configuration registry behind the autotuner
// (massively_b200/tune.py): which tile shape each algorithm family uses on
// an executor.

#include "common.cuh"

namespace mb {
int radix_tune_count();
const char* radix_tune_text(int c);
}  // namespace mb

using namespace mb;

extern "C" {

int mb_tune_config_count(int family) {
  switch (family) {
    case MB_TUNE_RADIX: return radix_tune_count();
    case MB_TUNE_SCAN: return 3;
    case MB_TUNE_SEG: return 2;
    case MB_TUNE_SEARCH: return 2;
    case MB_TUNE_REDUCE: case MB_TUNE_SELECT: return 1;
    default: return 0;
  }
}

const char* mb_tune_describe(int family, int config) {
  if (family == MB_TUNE_RADIX) return radix_tune_text(config);
  if (family == MB_TUNE_SCAN && config == 1)
    return "scan one 32 KB tile per CTA, warp 0 runs the look-back after the tile scan";
  if (family == MB_TUNE_SCAN && config == 2)
    return "scan one 64 KB tile per CTA, a ninth warp runs the look-back";
  if (family == MB_TUNE_SEG && config == 0)
    return "segmented scan / reduce over offsets: tile-local work, then the carries of the "
           "segments crossing tiles";
  if (family == MB_TUNE_SEG && config == 1)
    return "segmented scan / reduce over offsets: a decoupled look-back carried across tiles";
  if (family == MB_TUNE_SEARCH && config == 0)
    return "bounds search by 128-byte lines: a sample level per 32 (u32) elements, the top "
           "level in shared memory";
  if (family == MB_TUNE_SEARCH && config == 1)
    return "bounds search: binary search over 16 KB of samples in shared memory, then over "
           "the source interval";
  if (config == 0) {
    switch (family) {
      case MB_TUNE_SCAN: return "scan one 32 KB tile per CTA, a ninth warp runs the look-back";
      case MB_TUNE_REDUCE: return "reduce 256 threads x 4 x 16-byte vectors, fixed grid";
      case MB_TUNE_SELECT: return "compaction 256 threads x 16 items";
      default: break;
    }
  }
  return nullptr;
}

int mb_tune_set(mb_executor* ex, int family, int config) {
  MB_TRY(check_exec(ex));
  if (family < 0 || family > 7) return set_error(MB_ERR_LAUNCH, "unknown tuning family");
  if (config != -1 && (config < 0 || config >= mb_tune_config_count(family)))
    return set_error(MB_ERR_LAUNCH, "tuning configuration out of range");
  ex->tune[family] = config;
  return MB_OK;
}

int mb_tune_get(mb_executor* ex, int family) {
  if (!ex || family < 0 || family > 7) return -1;
  return ex->tune[family];
}

}  // extern "C"
