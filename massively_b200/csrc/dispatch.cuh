// dispatch.cuh -- run-time element-type dispatch onto kernel templates.
#pragma once

#include "common.cuh"

// Calls FN<T>(args...) for the compute type id `ct` and returns its status.
#define MB_DISPATCH_CTYPE(ct, FN, ...)                 \
  switch (ct) {                                        \
    case MB_U32: return FN<uint32_t>(__VA_ARGS__);     \
    case MB_I32: return FN<int32_t>(__VA_ARGS__);      \
    case MB_U64: return FN<uint64_t>(__VA_ARGS__);     \
    case MB_I64: return FN<int64_t>(__VA_ARGS__);      \
    case MB_F32: return FN<float>(__VA_ARGS__);        \
    case MB_F64: return FN<double>(__VA_ARGS__);       \
    default: break;                                    \
  }
