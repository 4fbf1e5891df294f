// common.cuh -- shared device/host pieces of the massively_b200 library:
// element types, built-in operators, the lazy-view loader evaluated inside
// every consuming kernel, decoupled look-back status words with bounded
// waits, and the executor that owns a stream, a memory pool and the device
// status word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <type_traits>
#include <vector>

#include "../../include/massively_b200.h"

namespace mb {

// ------------------------------------------------------------ constants --

// A decoupled look-back that has not seen its predecessor after this long
// gives up, records MB_DEV_ERR_LOOKBACK in the status word and lets the
// launch finish; the host reports it as MB_ERR_LAUNCH.
constexpr uint64_t kSpinLimitNs = 2000000000ull;  // 2 s

enum DeviceError : uint32_t {
  MB_DEV_OK = 0,
  MB_DEV_ERR_LOOKBACK = 1,
  MB_DEV_ERR_BOUNDS = 2,
};

// ---------------------------------------------------------------- types --

inline size_t dtype_size(int dt) {
  switch (dt) {
    case MB_U8: case MB_I8: return 1;
    case MB_U16: case MB_I16: return 2;
    case MB_U32: case MB_I32: case MB_F32: return 4;
    case MB_U64: case MB_I64: case MB_F64: return 8;
    default: return 0;
  }
}
inline bool dtype_valid(int dt) { return dt >= MB_U8 && dt <= MB_F64; }
inline bool dtype_is_float(int dt) { return dt == MB_F32 || dt == MB_F64; }
inline bool dtype_is_signed(int dt) { return dt >= MB_I8 && dt <= MB_I64; }
__host__ __device__ __forceinline__ bool dtype_is_signed_dev(int dt) {
  return dt >= MB_I8 && dt <= MB_I64;
}

// Compute type of an element type: narrow integers are computed in the
// 32-bit type of the same signedness (wrapping add / mul / bit ops and
// min / max give the same low bits), then stored narrow.
inline int compute_type(int dt) {
  switch (dt) {
    case MB_U8: case MB_U16: case MB_U32: return MB_U32;
    case MB_I8: case MB_I16: case MB_I32: return MB_I32;
    default: return dt;
  }
}

template <class T> struct DTypeOf;
template <> struct DTypeOf<uint8_t> { static constexpr int value = MB_U8; };
template <> struct DTypeOf<uint16_t> { static constexpr int value = MB_U16; };
template <> struct DTypeOf<uint32_t> { static constexpr int value = MB_U32; };
template <> struct DTypeOf<uint64_t> { static constexpr int value = MB_U64; };
template <> struct DTypeOf<int8_t> { static constexpr int value = MB_I8; };
template <> struct DTypeOf<int16_t> { static constexpr int value = MB_I16; };
template <> struct DTypeOf<int32_t> { static constexpr int value = MB_I32; };
template <> struct DTypeOf<int64_t> { static constexpr int value = MB_I64; };
template <> struct DTypeOf<float> { static constexpr int value = MB_F32; };
template <> struct DTypeOf<double> { static constexpr int value = MB_F64; };

template <class T> struct UnsignedOf { using type = std::make_unsigned_t<T>; };
template <> struct UnsignedOf<float> { using type = uint32_t; };
template <> struct UnsignedOf<double> { using type = uint64_t; };

// -------------------------------------------------------------- operators --

// Operator ids usable as template arguments; kOpDyn reads the id at run time.
constexpr int kOpDyn = -1;

template <class T>
__device__ __forceinline__ T op_apply_rt(int op, T a, T b) {
  if constexpr (std::is_floating_point<T>::value) {
    switch (op) {
      case MB_OP_ADD: return a + b;
      case MB_OP_MUL: return a * b;
      case MB_OP_MIN: return b < a ? b : a;
      case MB_OP_MAX: return a < b ? b : a;
      case MB_OP_TAKE_RIGHT: return b;
      default: return a;  // MB_OP_TAKE_LEFT
    }
  } else {
    using U = typename UnsignedOf<T>::type;
    switch (op) {
      case MB_OP_ADD: return (T)(U)((U)a + (U)b);
      case MB_OP_MUL: return (T)(U)((U)a * (U)b);
      case MB_OP_MIN: return b < a ? b : a;
      case MB_OP_MAX: return a < b ? b : a;
      case MB_OP_BIT_AND: return (T)((U)a & (U)b);
      case MB_OP_BIT_OR: return (T)((U)a | (U)b);
      case MB_OP_BIT_XOR: return (T)((U)a ^ (U)b);
      case MB_OP_TAKE_RIGHT: return b;
      default: return a;  // MB_OP_TAKE_LEFT
    }
  }
}

// Binary operator with a compile-time id (OP >= 0) or a run-time one.
template <class T, int OP>
struct Op {
  int rt;
  __device__ __forceinline__ T operator()(T a, T b) const {
    if constexpr (OP == kOpDyn) {
      return op_apply_rt<T>(rt, a, b);
    } else {
      return op_apply_rt<T>(OP, a, b);
    }
  }
};

inline bool op_valid_for(int op, int ctype) {
  if (op < MB_OP_ADD || op > MB_OP_TAKE_RIGHT) return false;
  if (dtype_is_float(ctype) && op >= MB_OP_BIT_AND && op <= MB_OP_BIT_XOR) return false;
  return true;
}
inline bool op_commutative(int op) { return op != MB_OP_TAKE_LEFT && op != MB_OP_TAKE_RIGHT; }

// --------------------------------------------------------------- sources --

// Device copy of an mb_src (lazy view).  Kept by value in kernel params.
struct Src {
  int kind, dtype, map, vtype;
  const void* data;
  const uint32_t* index;
  uint64_t len, a, b;
  const uint32_t* len_dev;
};

inline Src to_src(const mb_src& s) {
  Src d;
  d.kind = s.kind; d.dtype = s.dtype; d.map = s.map; d.vtype = s.vtype;
  d.data = s.data; d.index = s.index; d.len = s.len; d.a = s.a; d.b = s.b;
  d.len_dev = s.len_dev;
  return d;
}

// True when the view is a plain device column whose element type equals T's,
// so kernels may use vectorised loads.
inline bool src_plain(const mb_src& s, int ctype) {
  return s.kind == MB_SRC_COLUMN && s.map == MB_UN_IDENTITY && s.dtype == ctype &&
         s.vtype == ctype;
}

__device__ __forceinline__ uint64_t ld_bits(int dtype, const void* p, uint64_t i) {
  switch (dtype) {
    case MB_U8: case MB_I8: return ((const uint8_t*)p)[i];
    case MB_U16: case MB_I16: return ((const uint16_t*)p)[i];
    case MB_U32: case MB_I32: case MB_F32: return ((const uint32_t*)p)[i];
    default: return ((const uint64_t*)p)[i];
  }
}

__device__ __forceinline__ int64_t sext_bits(int dtype, uint64_t bits) {
  switch (dtype) {
    case MB_I8: return (int64_t)(int8_t)bits;
    case MB_I16: return (int64_t)(int16_t)bits;
    case MB_I32: return (int64_t)(int32_t)bits;
    default: return (int64_t)bits;
  }
}

// Applies an mb_unary map to the raw bits of one element of type `dtype`
// and converts the result to T (the consumer's compute type).
template <class T>
__device__ __forceinline__ T map_to(int map, int dtype, uint64_t bits) {
  // Identity loads of the same floating type keep their exact bits (NaN
  // payloads included).
  if constexpr (std::is_same<T, float>::value) {
    if (map == MB_UN_IDENTITY && dtype == MB_F32) return __uint_as_float((uint32_t)bits);
  }
  if constexpr (std::is_same<T, double>::value) {
    if (map == MB_UN_IDENTITY && dtype == MB_F64) return __longlong_as_double((long long)bits);
  }
  if (dtype == MB_F32 || dtype == MB_F64) {
    double x = dtype == MB_F32 ? (double)__uint_as_float((uint32_t)bits)
                               : __longlong_as_double((long long)bits);
    switch (map) {
      case MB_UN_IS_TRUE: return (T)(x != 0.0);
      case MB_UN_IS_FALSE: return (T)(x == 0.0);
      case MB_UN_IS_NEGATIVE: return (T)(x < 0.0);
      case MB_UN_IS_POSITIVE: return (T)(x > 0.0);
      case MB_UN_NEGATE: x = -x; break;
      case MB_UN_ABS: x = fabs(x); break;
      default: break;
    }
    if constexpr (std::is_floating_point<T>::value) {
      return (T)x;
    } else {
      return (T)(int64_t)x;
    }
  } else if (dtype_is_signed_dev(dtype)) {
    int64_t x = sext_bits(dtype, bits);
    switch (map) {
      case MB_UN_IS_TRUE: return (T)(x != 0);
      case MB_UN_IS_FALSE: return (T)(x == 0);
      case MB_UN_IS_EVEN: return (T)((x & 1) == 0);
      case MB_UN_IS_ODD: return (T)((x & 1) != 0);
      case MB_UN_IS_NEGATIVE: return (T)(x < 0);
      case MB_UN_IS_POSITIVE: return (T)(x > 0);
      case MB_UN_NEGATE: x = (int64_t)(0ull - (uint64_t)x); break;
      case MB_UN_BIT_NOT: x = ~x; break;
      case MB_UN_ABS: x = x < 0 ? (int64_t)(0ull - (uint64_t)x) : x; break;
      default: break;
    }
    return (T)x;
  } else {
    uint64_t x = bits;
    switch (map) {
      case MB_UN_IS_TRUE: return (T)(x != 0);
      case MB_UN_IS_FALSE: return (T)(x == 0);
      case MB_UN_IS_EVEN: return (T)((x & 1) == 0);
      case MB_UN_IS_ODD: return (T)((x & 1) != 0);
      case MB_UN_IS_NEGATIVE: return (T)0;
      case MB_UN_IS_POSITIVE: return (T)(x != 0);
      case MB_UN_NEGATE: x = 0ull - x; break;
      case MB_UN_BIT_NOT: x = ~x; break;
      default: break;
    }
    return (T)x;
  }
}

// Element i of a lazy view, as T.
template <class T>
__device__ __forceinline__ T src_load(const Src& s, uint64_t i) {
  uint64_t bits;
  if (s.kind == MB_SRC_ADJACENT) {
    const T cur = map_to<T>(MB_UN_IDENTITY, s.dtype, ld_bits(s.dtype, s.data, i));
    if (i == 0) return cur;
    const T prev = map_to<T>(MB_UN_IDENTITY, s.dtype, ld_bits(s.dtype, s.data, i - 1));
    return op_apply_rt<T>((int)s.b, prev, cur);
  }
  switch (s.kind) {
    case MB_SRC_COLUMN: bits = ld_bits(s.dtype, s.data, i); break;
    case MB_SRC_CONSTANT: bits = s.a; break;
    case MB_SRC_COUNTING: bits = s.a + i; break;
    case MB_SRC_STRIDE: bits = s.a + i * s.b; break;
    case MB_SRC_PERMUTE: bits = ld_bits(s.dtype, s.data, s.index[i]); break;
    case MB_SRC_REVERSE: bits = ld_bits(s.dtype, s.data, s.len - 1 - i); break;
    case MB_SRC_REPEAT_EACH: bits = ld_bits(s.dtype, s.data, i / s.a); break;
    default: bits = ld_bits(s.dtype, s.data, i % s.a); break;  // MB_SRC_TILE
  }
  return map_to<T>(s.map, s.dtype, bits);
}

// Raw bits of element i of a view, in its produced type (vtype).
__device__ __forceinline__ uint64_t src_load_bits(const Src& s, uint64_t i) {
  if (s.kind == MB_SRC_COLUMN && s.map == MB_UN_IDENTITY && s.dtype == s.vtype)
    return ld_bits(s.dtype, s.data, i);
  switch (s.vtype) {
    case MB_F32: return __float_as_uint(src_load<float>(s, i));
    case MB_F64: return (uint64_t)__double_as_longlong(src_load<double>(s, i));
    case MB_U64: case MB_I64: return src_load<uint64_t>(s, i);
    default: return src_load<uint32_t>(s, i);
  }
}

// Logical length of a view: the device length when one is attached.
__device__ __forceinline__ uint64_t src_len(const Src& s) {
  if (s.len_dev) {
    uint64_t d = *s.len_dev;
    return d < s.len ? d : s.len;
  }
  return s.len;
}

// Stores T into an output column of element type `dtype` (narrowing casts).
template <class T>
__device__ __forceinline__ void st_cast(int dtype, void* p, uint64_t i, T v) {
  switch (dtype) {
    case MB_U8: ((uint8_t*)p)[i] = (uint8_t)v; break;
    case MB_I8: ((int8_t*)p)[i] = (int8_t)v; break;
    case MB_U16: ((uint16_t*)p)[i] = (uint16_t)v; break;
    case MB_I16: ((int16_t*)p)[i] = (int16_t)v; break;
    case MB_U32: ((uint32_t*)p)[i] = (uint32_t)v; break;
    case MB_I32: ((int32_t*)p)[i] = (int32_t)v; break;
    case MB_U64: ((uint64_t*)p)[i] = (uint64_t)v; break;
    case MB_I64: ((int64_t*)p)[i] = (int64_t)v; break;
    case MB_F32: ((float*)p)[i] = (float)v; break;
    default: ((double*)p)[i] = (double)v; break;
  }
}

// ---------------------------------------------------- look-back helpers --

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Records a device-side failure once (first writer wins).
__device__ __forceinline__ void raise_device_error(uint32_t* status, uint32_t code) {
  if (status) atomicCAS(status, 0u, code);
}

// Where a kernel reports a failure: the executor's status word (read by
// mb_sync) and a per-launch abort word (zeroed with the launch's scratch) that
// tells the other waiting blocks of the same launch to stop waiting.
struct DevErr {
  uint32_t* status;
  uint32_t* abort;
};

__device__ __forceinline__ void raise_device_error(DevErr e, uint32_t code) {
  if (e.status) atomicCAS(e.status, 0u, code);
  if (e.abort) atomicExch(e.abort, 1u);
}

// Bounded-wait bookkeeping for one spinning thread.  `expired()` is true
// once the wait passed kSpinLimitNs or another block of the same launch
// already gave up.
struct SpinGuard {
  uint64_t start;
  uint32_t iter;
  const uint32_t* status;
  __device__ __forceinline__ explicit SpinGuard(const uint32_t* abort_word)
      : start(0), iter(0), status(abort_word) {}
  __device__ __forceinline__ bool expired() {
    ++iter;
    if ((iter & 63u) != 0) return false;
    if (iter > 256) __nanosleep(64);
    uint64_t now = globaltimer_ns();
    if (start == 0) { start = now; return false; }
    if (status && ld_relaxed_u32(status) != 0) return true;
    return now - start > kSpinLimitNs;
  }
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

}  // namespace mb

// ------------------------------------------------------------- executor --

struct mb_executor {
  uint64_t id;
  int device;
  cudaStream_t own_stream;
  cudaStream_t stream;
  cudaMemPool_t pool;
  uint32_t* status_dev;    // device error word (MB_DEV_*)
  uint32_t* host_pinned;   // 64 bytes of pinned staging for small readbacks
  int tune[8];             // selected configuration per MB_TUNE_* family (-1 default)
  bool capturing;
  cudaGraph_t graph;
  // mb_kernel_timing: event pairs around the dominant kernels' launches.
  struct Span {
    int family;
    cudaEvent_t start, stop;
  };
  bool timing = false;
  std::vector<Span> spans;
};

namespace mb {

// Thread-local error state (mb_last_error_message / mb_last_error_detail).
int set_error(int code, const std::string& msg, uint64_t left = 0, uint64_t right = 0);
int check_cuda(cudaError_t e, const char* what);
#define MB_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::mb::check_cuda(e_, #call); \
  } while (0)
#define MB_TRY(call)                  \
  do {                                \
    int s_ = (call);                  \
    if (s_ != MB_OK) return s_;       \
  } while (0)

// Brackets the launches issued in its scope with CUDA events on the
// executor's stream while mb_kernel_timing is on (never inside a capture).
struct TimedLaunch {
  mb_executor* ex;
  int family;
  cudaEvent_t start = nullptr;
  TimedLaunch(mb_executor* e, int fam) : ex(e), family(fam) {
    if (!ex->timing || ex->capturing) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ex->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
      return;
    if (cudaEventCreate(&start) != cudaSuccess) { start = nullptr; return; }
    cudaEventRecord(start, ex->stream);
  }
  ~TimedLaunch() {
    if (!start) return;
    cudaEvent_t stop = nullptr;
    if (cudaEventCreate(&stop) != cudaSuccess) { cudaEventDestroy(start); return; }
    cudaEventRecord(stop, ex->stream);
    ex->spans.push_back({family, start, stop});
  }
};

// Stream-ordered scratch from the executor's pool, released at scope end
// (in stream order, so it stays valid for every kernel enqueued before).
struct Scratch {
  mb_executor* ex = nullptr;
  void* ptr = nullptr;
  Scratch() = default;
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  ~Scratch();
  int alloc(mb_executor* e, size_t bytes);
  template <class T> T* as() const { return (T*)ptr; }
};

// Common argument validation mirroring massively's checks.
int check_exec(mb_executor* ex);
int check_src(mb_executor* ex, const mb_src* s, const char* what);
int check_col(mb_executor* ex, const mb_col& c, const char* what);
int check_len_u32(uint64_t n);

// Launch-geometry helper: grid for `tiles` one-tile blocks.
inline unsigned grid_for(uint64_t tiles) { return (unsigned)(tiles == 0 ? 1 : tiles); }

// Reads a u32 device value into the host (synchronises the stream).
int read_u32(mb_executor* ex, const uint32_t* dev, uint32_t* host);

}  // namespace mb

namespace mb {

// The same encodings on raw unsigned bits (U = uint32_t / uint64_t), so keys
// never pass through floating-point registers.
enum KeyEnc : int { kEncUnsigned = 0, kEncSigned = 1, kEncFloat = 2 };

template <class U, int ENC>
__device__ __forceinline__ U enc_bits(U raw) {
  constexpr U sign = (U)1 << (sizeof(U) * 8 - 1);
  if constexpr (ENC == kEncFloat) {
    return (raw & sign) ? (U)~raw : (U)(raw ^ sign);
  } else if constexpr (ENC == kEncSigned) {
    return (U)(raw ^ sign);
  } else {
    return raw;
  }
}

// Order-preserving radix encoding of massively/src/core/radix.rs:46-89:
// unsigned as is, signed with the sign bit flipped, floats in total order
// (negative: every bit inverted; otherwise the sign bit set).
template <class K>
__device__ __forceinline__ typename UnsignedOf<K>::type radix_enc(K k) {
  using U = typename UnsignedOf<K>::type;
  U raw;
  if constexpr (std::is_same<K, double>::value) {
    raw = (U)__double_as_longlong(k);  // the bit pattern, NaN payloads included
  } else if constexpr (std::is_same<K, float>::value) {
    raw = (U)__float_as_uint(k);
  } else {
    memcpy(&raw, &k, sizeof(U));
  }
  constexpr U sign = (U)1 << (sizeof(U) * 8 - 1);
  if constexpr (std::is_floating_point<K>::value) {
    return (raw & sign) ? (U)~raw : (U)(raw ^ sign);
  } else if constexpr (std::is_signed<K>::value) {
    return (U)(raw ^ sign);
  } else {
    return raw;
  }
}

}  // namespace mb
