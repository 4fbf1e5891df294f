// reduce.cu -- vector::reduce: init op fold(x) in one launch.
//
// Replaces massively's multi-pass tile reduction (massively/src/core/
// reduce.rs:806-1012: 65,536-item tiles, repeated partial passes, a final
// [init, partial] pass, host-created scratch per call).  Here a fixed grid
// (a function of n only) streams the input with 128-bit loads; each block
// reduces one contiguous chunk, warps reduce with `redux.sync` (32-bit
// integer add / min / max) or a shuffle tree, and the last block to finish
// (atomic ticket) folds the block partials in a fixed order and applies
// `init`.  The association depends on n alone, so floating-point results are
// identical from run to run.  Operators that are not commutative
// (TAKE_LEFT / TAKE_RIGHT) fold to init / the last element.

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBlocks = 1184;  // 8 per SM of a 148-SM B200; constant, for determinism

template <class T>
struct RedCfg {
  static constexpr int VEC = 16 / sizeof(T);
  static constexpr int LOADS = 4;
  static constexpr int TILE = kThreads * VEC * LOADS;
};

// Ordered fold over the lanes that hold a value (lane order = operand order).
template <class T, class OpT>
__device__ __forceinline__ bool warp_fold(T& v, bool h, const OpT& op) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    T o = shfl_down(v, off);
    bool oh = __shfl_down_sync(kFull, h, off);
    if (lane + off < 32 && oh) {
      v = h ? op(v, o) : o;
      h = true;
    }
  }
  v = shfl_idx(v, 0);
  return __shfl_sync(kFull, h, 0);
}

template <class T, int OP>
__device__ __forceinline__ T warp_reduce_full(T v, const Op<T, OP>& op) {
  if constexpr (OP != kOpDyn && sizeof(T) == 4 && !std::is_floating_point<T>::value) {
    if constexpr (OP == MB_OP_ADD) return (T)__reduce_add_sync(kFull, (uint32_t)v);
    if constexpr (OP == MB_OP_MIN) {
      if constexpr (std::is_signed<T>::value) return (T)__reduce_min_sync(kFull, (int)v);
      else return (T)__reduce_min_sync(kFull, (unsigned)v);
    }
    if constexpr (OP == MB_OP_MAX) {
      if constexpr (std::is_signed<T>::value) return (T)__reduce_max_sync(kFull, (int)v);
      else return (T)__reduce_max_sync(kFull, (unsigned)v);
    }
  }
  warp_fold(v, true, op);
  return v;
}

template <class T>
struct RedParams {
  int op;
  T init;
  uint64_t chunk;  // items per block (multiple of the tile)
  T* partials;
  uint32_t* ticket;
  T* result;
};

// Block-wide ordered fold of (v, h) per thread; result valid in thread 0.
template <class T, class OpT>
__device__ __forceinline__ bool block_fold(T& v, bool h, const OpT& op, T* s_v, bool* s_h) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bool wh = warp_fold(v, h, op);
  if (lane == 0) { s_v[warp] = v; s_h[warp] = wh; }
  __syncthreads();
  bool bh = false;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kWarps; ++i)
      if (s_h[i]) { v = bh ? op(v, s_v[i]) : s_v[i]; bh = true; }
  }
  __syncthreads();
  return bh;
}

template <class T, int OP, bool PLAIN>
__global__ void __launch_bounds__(kThreads) reduce_kernel(Src in, uint64_t cap, RedParams<T> p) {
  using C = RedCfg<T>;
  constexpr int VEC = C::VEC;
  __shared__ T s_v[kWarps];
  __shared__ bool s_h[kWarps];
  __shared__ bool s_last;
  const Op<T, OP> op{p.op};
  const uint64_t n = in.len_dev ? min((uint64_t)*in.len_dev, cap) : cap;
  const uint64_t begin = blockIdx.x * p.chunk;
  const uint64_t end = min(begin + p.chunk, n);
  bool has = false;
  T acc = T(0);
  for (uint64_t base = begin; base < end; base += C::TILE) {
    if (PLAIN && base + C::TILE <= end) {
      T x[C::LOADS][VEC];
#pragma unroll
      for (int j = 0; j < C::LOADS; ++j) {
        uint4 u = __ldcs(reinterpret_cast<const uint4*>((const T*)in.data + base) +
                         j * kThreads + threadIdx.x);
        memcpy(x[j], &u, 16);
      }
#pragma unroll
      for (int j = 0; j < C::LOADS; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          acc = has ? op(acc, x[j][k]) : x[j][k];
          has = true;
        }
    } else {
      for (int j = 0; j < C::LOADS * VEC; ++j) {
        const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
        if (i < end) {
          T v;
          if constexpr (PLAIN) v = ((const T*)in.data)[i];
          else v = src_load<T>(in, i);
          acc = has ? op(acc, v) : v;
          has = true;
        }
      }
    }
  }
  bool bh;
  if (__syncthreads_and(has)) {
    // Every thread holds a value: redux / shuffle tree per warp.
    T w = warp_reduce_full<T, OP>(acc, op);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_v[warp] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      acc = s_v[0];
      for (int i = 1; i < kWarps; ++i) acc = op(acc, s_v[i]);
    }
    bh = true;
  } else {
    bh = block_fold(acc, has, op, s_v, s_h);
  }
  if (threadIdx.x == 0) {
    p.partials[blockIdx.x] = bh ? acc : p.init;
    __threadfence();
    const uint32_t t = atomicAdd(p.ticket, 1u);
    s_last = t == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // Last block: ordered fold of the partials of the non-empty blocks.
  const uint64_t used = min((uint64_t)gridDim.x, (n + p.chunk - 1) / p.chunk);
  bool h = false;
  T v = T(0);
  for (uint64_t b = threadIdx.x; b < used; b += kThreads) {
    T x = *((volatile T*)&p.partials[b]);
    v = h ? op(v, x) : x;
    h = true;
  }
  bh = block_fold(v, h, op, s_v, s_h);
  if (threadIdx.x == 0) *p.result = bh ? op(p.init, v) : p.init;
}

template <class T>
int reduce_run(mb_executor* ex, const mb_src& in, int op, const void* init, void* result_dev,
               void* result_host) {
  using C = RedCfg<T>;
  const uint64_t cap = in.len;
  T initv;
  memcpy(&initv, init, sizeof(T));
  Scratch scratch;
  const uint64_t tiles = std::max<uint64_t>(1, (cap + C::TILE - 1) / C::TILE);
  const unsigned blocks = (unsigned)std::min<uint64_t>(tiles, kMaxBlocks);
  const uint64_t tiles_per_block = (tiles + blocks - 1) / blocks;
  MB_TRY(scratch.alloc(ex, 256 + (size_t)blocks * sizeof(T) + 64));
  char* base = scratch.as<char>();
  MB_CUDA(cudaMemsetAsync(base, 0, 256, ex->stream));
  RedParams<T> p{};
  p.op = op;
  p.init = initv;
  p.chunk = tiles_per_block * C::TILE;
  p.ticket = (uint32_t*)base;
  p.result = result_dev ? (T*)result_dev : (T*)(base + 64);
  p.partials = (T*)(base + 256);
  const bool plain = src_plain(in, DTypeOf<T>::value) && (uintptr_t)in.data % 16 == 0;
  const Src s = to_src(in);
#define MB_RED_LAUNCH(OPID)                                                                  \
  do {                                                                                       \
    if (plain) reduce_kernel<T, OPID, true><<<blocks, kThreads, 0, ex->stream>>>(s, cap, p); \
    else reduce_kernel<T, OPID, false><<<blocks, kThreads, 0, ex->stream>>>(s, cap, p);      \
  } while (0)
  switch (op) {
    case MB_OP_ADD: MB_RED_LAUNCH(MB_OP_ADD); break;
    case MB_OP_MIN: MB_RED_LAUNCH(MB_OP_MIN); break;
    case MB_OP_MAX: MB_RED_LAUNCH(MB_OP_MAX); break;
    default: MB_RED_LAUNCH(kOpDyn); break;
  }
#undef MB_RED_LAUNCH
  MB_CUDA(cudaGetLastError());
  if (result_host) {
    if (ex->capturing)
      return set_error(MB_ERR_LAUNCH, "a host-valued result cannot be read inside graph capture");
    MB_CUDA(cudaMemcpyAsync(ex->host_pinned, p.result, sizeof(T), cudaMemcpyDeviceToHost,
                            ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
    memcpy(result_host, ex->host_pinned, sizeof(T));
  }
  return MB_OK;
}

int write_result(mb_executor* ex, const void* value, size_t sz, void* result_dev,
                 void* result_host) {
  if (result_dev) {
    memcpy(ex->host_pinned, value, sz);
    MB_CUDA(cudaMemcpyAsync(result_dev, ex->host_pinned, sz, cudaMemcpyHostToDevice, ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
  }
  if (result_host) memcpy(result_host, value, sz);
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_reduce(mb_executor* ex, const mb_src* in, int op, const void* init, void* result_dev,
              void* result_host) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, in, "input"));
  if (!init) return set_error(MB_ERR_LAUNCH, "reduce needs an init value");
  const int ct = compute_type(in->vtype);
  if (!op_valid_for(op, ct)) return set_error(MB_ERR_LAUNCH, "operator not defined for this type");
  const size_t sz = dtype_size(in->vtype);
  uint64_t init_wide = 0;
  {
    uint64_t raw = 0;
    memcpy(&raw, init, sz);
    switch (in->vtype) {
      case MB_I8: init_wide = (uint64_t)(int64_t)(int8_t)raw; break;
      case MB_I16: init_wide = (uint64_t)(int64_t)(int16_t)raw; break;
      default: init_wide = raw; break;
    }
  }
  const uint64_t n = in->len;
  if (n == 0 || op == MB_OP_TAKE_LEFT) return write_result(ex, init, sz, result_dev, result_host);
  if (op == MB_OP_TAKE_RIGHT) {
    // The last element: a one-item copy of the reversed view.
    if (in->len_dev) return set_error(MB_ERR_LAUNCH, "TAKE_RIGHT reduce of a device-length view");
    Scratch tmp;
    MB_TRY(tmp.alloc(ex, n * sz));
    mb_col c{};
    c.data = tmp.ptr;
    c.dtype = in->vtype;
    c.len = n;
    MB_TRY(mb_copy(ex, in, c));
    if (result_dev)
      MB_CUDA(cudaMemcpyAsync(result_dev, (char*)tmp.ptr + (n - 1) * sz, sz,
                              cudaMemcpyDeviceToDevice, ex->stream));
    if (result_host) {
      MB_CUDA(cudaMemcpyAsync(ex->host_pinned, (char*)tmp.ptr + (n - 1) * sz, sz,
                              cudaMemcpyDeviceToHost, ex->stream));
      MB_CUDA(cudaStreamSynchronize(ex->stream));
      memcpy(result_host, ex->host_pinned, sz);
    }
    return MB_OK;
  }
  if (sz < 4) {
    // Narrow types reduce in their 32-bit compute type; the low bytes are
    // the narrow result.
    Scratch tmp;
    MB_TRY(tmp.alloc(ex, 16));
    uint64_t wide_host = 0;
    int st = ct == MB_U32
                 ? reduce_run<uint32_t>(ex, *in, op, &init_wide, tmp.ptr, result_host ? &wide_host : nullptr)
                 : reduce_run<int32_t>(ex, *in, op, &init_wide, tmp.ptr, result_host ? &wide_host : nullptr);
    if (st != MB_OK) return st;
    if (result_dev)
      MB_CUDA(cudaMemcpyAsync(result_dev, tmp.ptr, sz, cudaMemcpyDeviceToDevice, ex->stream));
    if (result_host) memcpy(result_host, &wide_host, sz);
    return MB_OK;
  }
  MB_DISPATCH_CTYPE(ct, reduce_run, ex, *in, op, &init_wide, result_dev, result_host);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

}  // extern "C"
