// scatter_reduce.cu -- vector::scatter_reduce.
//
// massively (massively/src/api/algorithm/scatter.rs:332-420, core
// massively/src/core/scatter_reduce.rs:388-403) reduces every group of
// proposals aimed at one destination -- `init op v_first op ... op v_last`
// -- and combines the result with the destination, `out[d] op reduced`
// (scatter_reduce.rs:179); destinations no index names keep their value.
// The op must be associative and commutative and the proposals of a group
// are reduced in an unspecified order.  massively gets there by a stable sort
// of the indices, a gather, head flags, a reduce-by-heads and one writer per
// destination.
//
// Here each proposal is folded straight into its destination with one
// atomic read-modify-write: hardware atomics for ADD (all types), MIN / MAX
// and the bit ops (integers), a compare-and-swap loop for MUL, float MIN /
// MAX and 1- / 2-byte columns (CAS on the aligned 32-bit word that holds the
// element).  Because the op is associative and commutative,
// `out[d] op v_1 op ... op v_k op init` equals massively's result exactly for
// the integer ops; `init` is folded in afterwards, once per destination that
// received a proposal (a bitmap records them), and only when it is not the
// op's identity.  Float ADD results depend on the arrival order, as the
// contract allows.  An index at or past the output's end is skipped and
// raises MB_DEV_ERR_BOUNDS (reported as a launch error at the next sync).

#include <algorithm>

#include "common.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kCasLimit = 1u << 22;  // CAS retries before reporting an error

unsigned grid_for_items(mb_executor* ex, uint64_t n) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t want = std::max<uint64_t>(1, (n + kThreads - 1) / kThreads);
  return (unsigned)std::min<uint64_t>(want, (uint64_t)sms * 16);
}

// Element of a 1-, 2-, 4- or 8-byte column as compute type T.
template <class T>
__device__ __forceinline__ T elem_from_bits(int dtype, uint64_t bits) {
  return map_to<T>(MB_UN_IDENTITY, dtype, bits);
}

template <class T>
__device__ __forceinline__ uint64_t elem_to_bits(int dtype, T v) {
  switch (dtype) {
    case MB_U8: case MB_I8: return (uint8_t)v;
    case MB_U16: case MB_I16: return (uint16_t)v;
    case MB_U32: case MB_I32: return (uint32_t)v;
    case MB_F32: return __float_as_uint((float)v);
    case MB_F64: return (uint64_t)__double_as_longlong((double)v);
    default: return (uint64_t)v;
  }
}

// out[j] = out[j] op v, atomically.  Returns false if a compare-and-swap
// loop gave up (it cannot starve: each failed swap is another thread's
// success; the limit only bounds a pathological case).
template <class T, int OP>
__device__ __forceinline__ bool atomic_combine(void* out, int dtype, uint64_t j, T v) {
  const size_t esize = dtype == MB_U8 || dtype == MB_I8 ? 1
                       : dtype == MB_U16 || dtype == MB_I16 ? 2
                       : dtype == MB_U64 || dtype == MB_I64 || dtype == MB_F64 ? 8 : 4;
  if (esize == sizeof(T)) {
    if constexpr (std::is_same<T, float>::value || std::is_same<T, double>::value) {
      if constexpr (OP == MB_OP_ADD) {
        atomicAdd((T*)out + j, v);
        return true;
      }
    } else if constexpr (sizeof(T) == 4) {
      using A = typename std::conditional<std::is_signed<T>::value, int, unsigned>::type;
      A* p = (A*)out + j;
      if constexpr (OP == MB_OP_ADD) { atomicAdd((unsigned*)p, (unsigned)v); return true; }
      if constexpr (OP == MB_OP_MIN) { atomicMin(p, (A)v); return true; }
      if constexpr (OP == MB_OP_MAX) { atomicMax(p, (A)v); return true; }
      if constexpr (OP == MB_OP_BIT_AND) { atomicAnd((unsigned*)p, (unsigned)v); return true; }
      if constexpr (OP == MB_OP_BIT_OR) { atomicOr((unsigned*)p, (unsigned)v); return true; }
      if constexpr (OP == MB_OP_BIT_XOR) { atomicXor((unsigned*)p, (unsigned)v); return true; }
    } else {
      using A = typename std::conditional<std::is_signed<T>::value, long long,
                                          unsigned long long>::type;
      A* p = (A*)out + j;
      using U = unsigned long long;
      if constexpr (OP == MB_OP_ADD) { atomicAdd((U*)p, (U)v); return true; }
      if constexpr (OP == MB_OP_MIN) { atomicMin(p, (A)v); return true; }
      if constexpr (OP == MB_OP_MAX) { atomicMax(p, (A)v); return true; }
      if constexpr (OP == MB_OP_BIT_AND) { atomicAnd((U*)p, (U)v); return true; }
      if constexpr (OP == MB_OP_BIT_OR) { atomicOr((U*)p, (U)v); return true; }
      if constexpr (OP == MB_OP_BIT_XOR) { atomicXor((U*)p, (U)v); return true; }
    }
    // compare-and-swap on the element itself
    if constexpr (sizeof(T) == 4) {
      unsigned* p = (unsigned*)out + j;
      unsigned old = *(volatile unsigned*)p;
      for (uint32_t k = 0; k < kCasLimit; ++k) {
        const unsigned want = (unsigned)to_bits64<T>(op_apply_rt<T>(OP, from_bits64<T>(old), v));
        const unsigned seen = atomicCAS(p, old, want);
        if (seen == old) return true;
        old = seen;
      }
    } else {
      unsigned long long* p = (unsigned long long*)out + j;
      unsigned long long old = *(volatile unsigned long long*)p;
      for (uint32_t k = 0; k < kCasLimit; ++k) {
        const unsigned long long want =
            (unsigned long long)to_bits64<T>(op_apply_rt<T>(OP, from_bits64<T>(old), v));
        const unsigned long long seen = atomicCAS(p, old, want);
        if (seen == old) return true;
        old = seen;
      }
    }
    return false;
  }
  // 1- or 2-byte element: swap the aligned 32-bit word around it
  const uintptr_t addr = (uintptr_t)out + j * esize;
  unsigned* w = (unsigned*)(addr & ~(uintptr_t)3);
  const unsigned shift = (unsigned)(addr & 3) * 8;
  const unsigned mask = (esize == 1 ? 0xFFu : 0xFFFFu) << shift;
  unsigned old = *(volatile unsigned*)w;
  for (uint32_t k = 0; k < kCasLimit; ++k) {
    const T cur = elem_from_bits<T>(dtype, (old & mask) >> shift);
    const unsigned nb = (unsigned)elem_to_bits<T>(dtype, op_apply_rt<T>(OP, cur, v));
    const unsigned want = (old & ~mask) | ((nb << shift) & mask);
    const unsigned seen = atomicCAS(w, old, want);
    if (seen == old) return true;
    old = seen;
  }
  return false;
}

template <class T, int OP>
__global__ void __launch_bounds__(kThreads)
    scatter_reduce_kernel(Src values, Src idx, void* out, int dtype, uint64_t nout,
                          uint32_t* __restrict__ touched, uint32_t* status) {
  const uint64_t n = src_len(values);
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += step) {
    const uint64_t j = src_load<uint32_t>(idx, i);
    if (j >= nout) {
      raise_device_error(status, MB_DEV_ERR_BOUNDS);
      continue;
    }
    if (!atomic_combine<T, OP>(out, dtype, j, src_load<T>(values, i)))
      raise_device_error(status, MB_DEV_ERR_LOOKBACK);
    if (touched) atomicOr(touched + (j >> 5), 1u << (j & 31));
  }
}

// out[d] = out[d] op init for every destination that received a proposal
// (one writer per destination).
template <class T, int OP>
__global__ void __launch_bounds__(kThreads)
    scatter_reduce_init_kernel(void* out, int dtype, uint64_t nout, T init,
                               const uint32_t* __restrict__ touched) {
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (uint64_t d = blockIdx.x * (uint64_t)kThreads + threadIdx.x; d < nout; d += step) {
    if (!((touched[d >> 5] >> (d & 31)) & 1u)) continue;
    const T cur = elem_from_bits<T>(dtype, ld_bits(dtype, out, d));
    st_cast<T>(dtype, out, d, op_apply_rt<T>(OP, cur, init));
  }
}

// The identity of `op` in the element type `dtype`, as its bit pattern.
bool identity_bits(int op, int dtype, uint64_t* bits) {
  const size_t sz = dtype_size(dtype);
  const uint64_t all = sz == 8 ? ~0ull : ((1ull << (8 * sz)) - 1);
  const uint64_t sign = 1ull << (8 * sz - 1);
  switch (op) {
    case MB_OP_ADD: case MB_OP_BIT_OR: case MB_OP_BIT_XOR:
      *bits = 0;  // +0.0 for floats
      return true;
    case MB_OP_BIT_AND: *bits = all; return true;
    case MB_OP_MUL:
      *bits = dtype == MB_F32 ? 0x3F800000ull : dtype == MB_F64 ? 0x3FF0000000000000ull : 1;
      return true;
    case MB_OP_MIN:  // the greatest value
      if (dtype == MB_F32) *bits = 0x7F800000ull;
      else if (dtype == MB_F64) *bits = 0x7FF0000000000000ull;
      else *bits = dtype_is_signed(dtype) ? all >> 1 : all;
      return true;
    case MB_OP_MAX:  // the least value
      if (dtype == MB_F32) *bits = 0xFF800000ull;
      else if (dtype == MB_F64) *bits = 0xFFF0000000000000ull;
      else *bits = dtype_is_signed(dtype) ? sign : 0;
      return true;
    default: return false;
  }
}

// Host value of compute type T from an element's bit pattern.
template <class T>
T host_elem(int dtype, uint64_t bits) {
  switch (dtype) {
    case MB_I8: return (T)(int8_t)bits;
    case MB_I16: return (T)(int16_t)bits;
    case MB_I32: return (T)(int32_t)bits;
    case MB_I64: return (T)(int64_t)bits;
    case MB_U8: return (T)(uint8_t)bits;
    case MB_U16: return (T)(uint16_t)bits;
    case MB_U32: return (T)(uint32_t)bits;
    case MB_F32: { float f; uint32_t b = (uint32_t)bits; memcpy(&f, &b, 4); return (T)f; }
    case MB_F64: { double f; memcpy(&f, &bits, 8); return (T)f; }
    default: return (T)bits;
  }
}

template <class T>
int scatter_column(mb_executor* ex, const mb_src& values, const mb_src& indices, int op,
                   uint64_t init_bits, bool fold_init, const mb_col& out, uint32_t* touched,
                   bool mark) {
  const Src v = to_src(values), ix = to_src(indices);
  const unsigned g = grid_for_items(ex, values.len);
  uint32_t* t = mark ? touched : nullptr;
#define MB_SR(OPV)                                                                      \
  scatter_reduce_kernel<T, OPV><<<g, kThreads, 0, ex->stream>>>(v, ix, out.data, out.dtype, \
                                                                out.len, t, ex->status_dev); \
  if (fold_init)                                                                        \
    scatter_reduce_init_kernel<T, OPV><<<grid_for_items(ex, out.len), kThreads, 0,        \
                                         ex->stream>>>(out.data, out.dtype, out.len,      \
                                                       host_elem<T>(out.dtype, init_bits), \
                                                       touched);                          \
  break;
  switch (op) {
    case MB_OP_ADD: MB_SR(MB_OP_ADD)
    case MB_OP_MUL: MB_SR(MB_OP_MUL)
    case MB_OP_MIN: MB_SR(MB_OP_MIN)
    case MB_OP_MAX: MB_SR(MB_OP_MAX)
    case MB_OP_BIT_AND:
      if constexpr (!std::is_floating_point<T>::value) { MB_SR(MB_OP_BIT_AND) }
      break;
    case MB_OP_BIT_OR:
      if constexpr (!std::is_floating_point<T>::value) { MB_SR(MB_OP_BIT_OR) }
      break;
    case MB_OP_BIT_XOR:
      if constexpr (!std::is_floating_point<T>::value) { MB_SR(MB_OP_BIT_XOR) }
      break;
    default: return set_error(MB_ERR_LAUNCH, "scatter_reduce needs an associative, commutative op");
  }
#undef MB_SR
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_scatter_reduce(mb_executor* ex, const mb_src* values, int nvals, const mb_src* indices,
                      const int* ops, const uint64_t* inits, const mb_col* out) {
  MB_TRY(check_exec(ex));
  if (nvals < 1 || !values || !ops || !inits || !out)
    return set_error(MB_ERR_UNBOUND_COLUMN, "scatter_reduce needs at least one value column");
  MB_TRY(check_src(ex, indices, "indices"));
  if (indices->vtype != MB_U32) return set_error(MB_ERR_LAUNCH, "indices must be u32 (MIndex)");
  MB_TRY(check_len_u32(indices->len));
  for (int c = 0; c < nvals; ++c) {
    MB_TRY(check_src(ex, &values[c], "values"));
    MB_TRY(check_col(ex, out[c], "output"));
    if (values[c].len != indices->len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "values and indices lengths differ",
                       values[c].len, indices->len);
    if (values[c].vtype != out[c].dtype)
      return set_error(MB_ERR_LAUNCH, "output element type differs from the values'");
    if (!op_valid_for(ops[c], compute_type(out[c].dtype)) || !op_commutative(ops[c]))
      return set_error(MB_ERR_LAUNCH, "scatter_reduce needs an associative, commutative op");
  }
  if (indices->len == 0) return MB_OK;
  // init is folded in only where it is not the op's identity
  bool any_init = false;
  std::vector<bool> fold(nvals);
  for (int c = 0; c < nvals; ++c) {
    uint64_t id = 0;
    const size_t sz = dtype_size(out[c].dtype);
    const uint64_t m = sz == 8 ? ~0ull : ((1ull << (8 * sz)) - 1);
    fold[c] = !identity_bits(ops[c], out[c].dtype, &id) || ((inits[c] & m) != id);
    any_init = any_init || fold[c];
  }
  Scratch touched;
  uint32_t* tb = nullptr;
  if (any_init) {
    uint64_t nout = 0;
    for (int c = 0; c < nvals; ++c) nout = std::max<uint64_t>(nout, out[c].len);
    const size_t bytes = ((nout + 31) / 32) * 4 + 16;
    MB_TRY(touched.alloc(ex, bytes));
    tb = touched.as<uint32_t>();
    MB_CUDA(cudaMemsetAsync(tb, 0, bytes, ex->stream));
  }
  for (int c = 0; c < nvals; ++c) {
    // every column's kernel marks: the output lengths may differ
    const bool mark = fold[c];
    if (fold[c] && c > 0)
      MB_CUDA(cudaMemsetAsync(tb, 0, ((out[c].len + 31) / 32) * 4 + 16, ex->stream));
    const int ct = compute_type(out[c].dtype);
    int st;
    switch (ct) {
      case MB_U32: st = scatter_column<uint32_t>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      case MB_I32: st = scatter_column<int32_t>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      case MB_U64: st = scatter_column<uint64_t>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      case MB_I64: st = scatter_column<int64_t>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      case MB_F32: st = scatter_column<float>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      case MB_F64: st = scatter_column<double>(ex, values[c], *indices, ops[c], inits[c], fold[c], out[c], tb, mark); break;
      default: return set_error(MB_ERR_LAUNCH, "unsupported element type");
    }
    MB_TRY(st);
  }
  return MB_OK;
}

}  // extern "C"
