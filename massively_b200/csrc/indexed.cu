// indexed.cu -- element-wise kernels: materialise a lazy view (copy / map),
// fill, gather / scatter (with optional stencil) and the PCG random streams.
//
// Replaces massively's indexed_copy_a13 (massively/src/core/indexed.rs:
// 16-190), materialize_a13 (massively/src/core/transform.rs:19-74) and the
// uniform random views (massively/src/api/util/random.rs:331-385).  Plain
// same-type columns move with 128-bit streaming loads and stores; lazy views
// are evaluated per item inside the load.  Grids are a multiple of the SM
// count with grid-stride loops.

#include "common.cuh"
#include "dispatch.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;

int sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

unsigned stride_grid(uint64_t work_items) {
  uint64_t want = (work_items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)sm_count() * 8;
  if (want < 1) want = 1;
  return (unsigned)(want < cap ? want : cap);
}

// out[i] = view[i]; T = the output's compute type.
template <class T>
__global__ void __launch_bounds__(kThreads) copy_view_kernel(Src in, void* out, int out_dtype,
                                                             uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < n; i += step) st_cast<T>(out_dtype, out, i, src_load<T>(in, i));
}

// The same for a 4-byte output of the view's own compute type, 16-byte
// aligned: four items per thread and one 16-byte store (views such as
// counting, constant or repeat_each compute their items, so stores dominate).
// KIND: MB_SRC_COUNTING / MB_SRC_STRIDE of the output's own type with no map
// (the item's bits are a + i*b, computed inline), or -1 for any view.
template <class T, int KIND>
__device__ __forceinline__ T view_item(const Src& in, uint64_t i) {
  if constexpr (KIND == MB_SRC_COUNTING) {
    const uint32_t b = (uint32_t)(in.a + i);
    T x;
    memcpy(&x, &b, 4);
    return x;
  } else if constexpr (KIND == MB_SRC_STRIDE) {
    const uint32_t b = (uint32_t)(in.a + i * in.b);
    T x;
    memcpy(&x, &b, 4);
    return x;
  } else {
    return src_load<T>(in, i);
  }
}

template <class T, int KIND>
__global__ void __launch_bounds__(kThreads) copy_view4_kernel(Src in, uint4* out, uint64_t n) {
  static_assert(sizeof(T) == 4, "4-byte items");
  const uint64_t nvec = n / 4;
  uint64_t v = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; v < nvec; v += step) {
    T x[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = view_item<T, KIND>(in, 4 * v + k);
    uint4 u;
    memcpy(&u, x, 16);
    __stcs(out + v, u);
  }
  for (uint64_t i = nvec * 4 + blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n; i += step)
    reinterpret_cast<T*>(out)[i] = view_item<T, KIND>(in, i);
}

// 16-byte vector copy of a plain column (same element type both sides).
__global__ void __launch_bounds__(kThreads) copy_vec_kernel(const uint4* in, uint4* out,
                                                            uint64_t nvec) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < nvec; i += step) __stcs(out + i, __ldcs(in + i));
}

__global__ void __launch_bounds__(kThreads) fill_kernel(void* out, int size, uint64_t bits,
                                                        uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < n; i += step) {
    switch (size) {
      case 1: ((uint8_t*)out)[i] = (uint8_t)bits; break;
      case 2: ((uint16_t*)out)[i] = (uint16_t)bits; break;
      case 4: ((uint32_t*)out)[i] = (uint32_t)bits; break;
      default: ((uint64_t*)out)[i] = bits; break;
    }
  }
}

// replace_where: out[i] = value where stencil[i] != 0 (massively's
// ReplaceWhereOperation, core/selection.rs:471-513: a gather of the value
// into the selected indices).  Items past the stencil's logical length (a
// device count) are left alone.
__global__ void __launch_bounds__(kThreads) replace_where_kernel(void* out, int size,
                                                                 uint64_t bits, Src stencil,
                                                                 uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  const uint64_t lim = src_len(stencil) < n ? src_len(stencil) : n;
  for (; i < lim; i += step) {
    if (src_load<uint32_t>(stencil, i) == 0) continue;
    switch (size) {
      case 1: ((uint8_t*)out)[i] = (uint8_t)bits; break;
      case 2: ((uint16_t*)out)[i] = (uint16_t)bits; break;
      case 4: ((uint32_t*)out)[i] = (uint32_t)bits; break;
      default: ((uint64_t*)out)[i] = bits; break;
    }
  }
}

// transform_where: out[i] = view[i] (the view's map is the operator) where
// stencil[i] != 0 (massively's TransformWhereInput, core/selection.rs:
// 515-578); T = the output's compute type.
template <class T>
__global__ void __launch_bounds__(kThreads) transform_where_kernel(Src in, Src stencil, void* out,
                                                                   int out_dtype, uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  uint64_t lim = src_len(stencil) < n ? src_len(stencil) : n;
  if (src_len(in) < lim) lim = src_len(in);
  for (; i < lim; i += step)
    if (src_load<uint32_t>(stencil, i) != 0) st_cast<T>(out_dtype, out, i, src_load<T>(in, i));
}

template <class T>
int transform_where_run(mb_executor* ex, const mb_src& in, const mb_src& stencil,
                        const mb_col& out) {
  transform_where_kernel<T><<<stride_grid(in.len), kThreads, 0, ex->stream>>>(
      to_src(in), to_src(stencil), out.data, out.dtype, in.len);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int transform_where_col(mb_executor* ex, const mb_src& in, const mb_src& stencil,
                        const mb_col& out) {
  MB_DISPATCH_CTYPE(compute_type(out.dtype), transform_where_run, ex, in, stencil, out);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

// gather: out[i] = values[idx[i]] where stencil (if any) is set.  Rows of
// `size` bytes move as raw bits (no conversion), like massively's copy.
template <int SIZE>
__global__ void __launch_bounds__(kThreads) gather_kernel(Src values, Src idx, Src stencil,
                                                          bool has_stencil, void* out,
                                                          uint64_t n, uint64_t nvalues,
                                                          uint32_t* status) {
  using W = typename std::conditional<SIZE == 1, uint8_t,
            typename std::conditional<SIZE == 2, uint16_t,
            typename std::conditional<SIZE == 4, uint32_t, uint64_t>::type>::type>::type;
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  const uint64_t lim = src_len(idx) < n ? src_len(idx) : n;  // the indices' logical length
  for (; i < lim; i += step) {
    if (has_stencil && src_load<uint32_t>(stencil, i) == 0) continue;
    const uint64_t j = src_load<uint32_t>(idx, i);
    if (j >= nvalues) { raise_device_error(status, MB_DEV_ERR_BOUNDS); continue; }
    ((W*)out)[i] = (W)src_load_bits(values, j);
  }
}

template <int SIZE>
__global__ void __launch_bounds__(kThreads) scatter_kernel(Src values, Src idx, Src stencil,
                                                           bool has_stencil, void* out,
                                                           uint64_t n, uint64_t nout,
                                                           uint32_t* status) {
  using W = typename std::conditional<SIZE == 1, uint8_t,
            typename std::conditional<SIZE == 2, uint16_t,
            typename std::conditional<SIZE == 4, uint32_t, uint64_t>::type>::type>::type;
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < n; i += step) {
    if (has_stencil && src_load<uint32_t>(stencil, i) == 0) continue;
    const uint64_t j = src_load<uint32_t>(idx, i);
    if (j >= nout) { raise_device_error(status, MB_DEV_ERR_BOUNDS); continue; }
    ((W*)out)[j] = (W)src_load_bits(values, i);
  }
}

// PCG hash of massively/src/api/util/random.rs:331-336.
__device__ __forceinline__ uint32_t pcg_hash32(uint32_t input) {
  uint32_t state = input * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// uniform_u32_value (random.rs:376-385); index = offset + i in u32.
__global__ void __launch_bounds__(kThreads) uniform_u32_kernel(uint32_t* out, uint64_t n,
                                                               uint32_t mn, uint32_t span,
                                                               uint32_t key, uint64_t offset) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < n; i += step) {
    uint32_t v = pcg_hash32((uint32_t)(offset + i) ^ key);
    out[i] = span == 0xFFFFFFFFu ? v : mn + v % (span + 1u);
  }
}

// uniform_u64_value (random.rs:343-348, 387-396).
__global__ void __launch_bounds__(kThreads) uniform_u64_kernel(uint64_t* out, uint64_t n,
                                                               uint64_t mn, uint64_t span,
                                                               uint32_t key, uint64_t offset) {
  uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x;
  const uint64_t step = (uint64_t)gridDim.x * kThreads;
  for (; i < n; i += step) {
    uint32_t idx = (uint32_t)(offset + i);
    uint64_t lo = pcg_hash32(idx ^ key);
    uint64_t hi = pcg_hash32(idx ^ key ^ 0x9e3779b9u);
    uint64_t v = lo | (hi << 32);
    out[i] = span == ~0ull ? v : mn + v % (span + 1ull);
  }
}

uint32_t pcg_hash32_host(uint32_t input) {
  uint32_t state = input * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

// seed_key of random.rs:18-22.
uint32_t seed_key(uint64_t seed) {
  return pcg_hash32_host((uint32_t)seed ^ pcg_hash32_host((uint32_t)(seed >> 32)));
}

template <class T>
int copy_run(mb_executor* ex, const mb_src& in, const mb_col& out) {
  const uint64_t n = in.len;
  if constexpr (sizeof(T) == 4) {
    if (out.dtype == DTypeOf<T>::value && (uintptr_t)out.data % 16 == 0 && !in.len_dev) {
      const unsigned g = stride_grid((n + 3) / 4);
      const bool own = in.map == MB_UN_IDENTITY && in.vtype == out.dtype && in.dtype == out.dtype;
      if (own && in.kind == MB_SRC_COUNTING)
        copy_view4_kernel<T, MB_SRC_COUNTING><<<g, kThreads, 0, ex->stream>>>(to_src(in),
                                                                           (uint4*)out.data, n);
      else if (own && in.kind == MB_SRC_STRIDE)
        copy_view4_kernel<T, MB_SRC_STRIDE><<<g, kThreads, 0, ex->stream>>>(to_src(in),
                                                                         (uint4*)out.data, n);
      else
        copy_view4_kernel<T, -1><<<g, kThreads, 0, ex->stream>>>(to_src(in), (uint4*)out.data, n);
      MB_CUDA(cudaGetLastError());
      return MB_OK;
    }
  }
  copy_view_kernel<T><<<stride_grid(n), kThreads, 0, ex->stream>>>(to_src(in), out.data,
                                                                    out.dtype, n);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int launch_indexed(mb_executor* ex, const mb_src* values, const mb_src* indices,
                   const mb_src* stencil, const mb_col& out, bool is_gather) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_src(ex, indices, "indices"));
  MB_TRY(check_col(ex, out, "output"));
  if (stencil) MB_TRY(check_src(ex, stencil, "stencil"));
  if (compute_type(indices->vtype) != MB_U32 || dtype_size(indices->vtype) != 4)
    return set_error(MB_ERR_LAUNCH, "indices must be u32 (MIndex)");
  if (dtype_size(values->vtype) != dtype_size(out.dtype))
    return set_error(MB_ERR_LAUNCH, "output element type differs from the values'");
  const uint64_t n = is_gather ? indices->len : values->len;
  if (!is_gather && indices->len != values->len)
    return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", values->len, indices->len);
  if (stencil && stencil->len != indices->len)
    return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", indices->len, stencil->len);
  if (is_gather && out.len < n)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out.len);
  if (n == 0) return MB_OK;
  Src v = to_src(*values), ix = to_src(*indices);
  Src st = stencil ? to_src(*stencil) : Src{};
  const bool hs = stencil != nullptr;
  const unsigned g = stride_grid(n);
  const uint64_t bound = is_gather ? values->len : out.len;
  switch (dtype_size(out.dtype)) {
#define MB_IDX_CASE(S)                                                                       \
  case S:                                                                                    \
    if (is_gather)                                                                           \
      gather_kernel<S><<<g, kThreads, 0, ex->stream>>>(v, ix, st, hs, out.data, n, bound,   \
                                                        ex->status_dev);                     \
    else                                                                                     \
      scatter_kernel<S><<<g, kThreads, 0, ex->stream>>>(v, ix, st, hs, out.data, n, bound,  \
                                                         ex->status_dev);                    \
    break;
    MB_IDX_CASE(1) MB_IDX_CASE(2) MB_IDX_CASE(4) MB_IDX_CASE(8)
#undef MB_IDX_CASE
    default: return set_error(MB_ERR_LAUNCH, "unsupported element size");
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

}  // namespace

// Internal: dst[i] = src[idx[i]] for plain columns of `esize`-byte elements.
int gather_raw(mb_executor* ex, const void* src, size_t esize, uint64_t nsrc,
               const uint32_t* idx, uint64_t n, void* dst, const uint32_t* n_dev) {
  if (n == 0) return MB_OK;
  Src v{};
  v.kind = MB_SRC_COLUMN;
  v.dtype = v.vtype = esize == 1 ? MB_U8 : esize == 2 ? MB_U16 : esize == 4 ? MB_U32 : MB_U64;
  v.map = MB_UN_IDENTITY;
  v.data = src;
  v.len = nsrc;
  Src ix{};
  ix.kind = MB_SRC_COLUMN;
  ix.dtype = ix.vtype = MB_U32;
  ix.map = MB_UN_IDENTITY;
  ix.data = idx;
  ix.len = n;
  ix.len_dev = n_dev;  // only the first *n_dev indices when given
  const unsigned g = stride_grid(n);
  switch (esize) {
    case 1: gather_kernel<1><<<g, kThreads, 0, ex->stream>>>(v, ix, Src{}, false, dst, n, nsrc, ex->status_dev); break;
    case 2: gather_kernel<2><<<g, kThreads, 0, ex->stream>>>(v, ix, Src{}, false, dst, n, nsrc, ex->status_dev); break;
    case 4: gather_kernel<4><<<g, kThreads, 0, ex->stream>>>(v, ix, Src{}, false, dst, n, nsrc, ex->status_dev); break;
    default: gather_kernel<8><<<g, kThreads, 0, ex->stream>>>(v, ix, Src{}, false, dst, n, nsrc, ex->status_dev); break;
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// Internal: materialises a view into a plain column of its vtype.
int materialize(mb_executor* ex, const mb_src& in, void* dst) {
  mb_col out{};
  out.data = dst;
  out.dtype = in.vtype;
  out.len = in.len;
  return mb_copy(ex, &in, out);
}

}  // namespace mb

using namespace mb;

extern "C" {

int mb_copy(mb_executor* ex, const mb_src* in, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, in, "input"));
  MB_TRY(check_col(ex, out, "output"));
  if (out.len < in->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", in->len, out.len);
  if (in->len == 0) return MB_OK;
  // Plain column of the same type, both 16-byte aligned: raw vector copy.
  if (in->kind == MB_SRC_COLUMN && in->map == MB_UN_IDENTITY && in->dtype == out.dtype &&
      in->vtype == out.dtype && in->len_dev == nullptr) {
    const uint64_t bytes = in->len * dtype_size(out.dtype);
    if ((uintptr_t)in->data % 16 == 0 && (uintptr_t)out.data % 16 == 0 && bytes % 16 == 0) {
      copy_vec_kernel<<<stride_grid(bytes / 16), kThreads, 0, ex->stream>>>(
          (const uint4*)in->data, (uint4*)out.data, bytes / 16);
      MB_CUDA(cudaGetLastError());
      return MB_OK;
    }
    MB_CUDA(cudaMemcpyAsync(out.data, in->data, bytes, cudaMemcpyDeviceToDevice, ex->stream));
    return MB_OK;
  }
  const int ct = compute_type(out.dtype);
  MB_DISPATCH_CTYPE(ct, copy_run, ex, *in, out);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int mb_fill(mb_executor* ex, const void* value, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_col(ex, out, "output"));
  if (!value) return set_error(MB_ERR_LAUNCH, "null fill value");
  if (out.len == 0) return MB_OK;
  uint64_t bits = 0;
  memcpy(&bits, value, dtype_size(out.dtype));
  fill_kernel<<<stride_grid(out.len), kThreads, 0, ex->stream>>>(
      out.data, (int)dtype_size(out.dtype), bits, out.len);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mb_replace_where(mb_executor* ex, const uint64_t* values, const mb_src* stencil,
                     const mb_col* out, int ncols) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, stencil, "stencil"));
  if (!out || !values || ncols < 1 || ncols > 12)
    return set_error(MB_ERR_LAUNCH, "replace_where takes 1 to 12 output columns and values");
  for (int c = 0; c < ncols; ++c) {
    MB_TRY(check_col(ex, out[c], "output"));
    if (stencil->len != out[c].len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "stencil and output lengths differ", stencil->len,
                       out[c].len);
  }
  if (stencil->len == 0) return MB_OK;
  const Src st = to_src(*stencil);
  for (int c = 0; c < ncols; ++c) {
    replace_where_kernel<<<stride_grid(out[c].len), kThreads, 0, ex->stream>>>(
        out[c].data, (int)dtype_size(out[c].dtype), values[c], st, out[c].len);
    MB_CUDA(cudaGetLastError());
  }
  return MB_OK;
}

int mb_transform_where(mb_executor* ex, const mb_src* in, int ncols, const mb_src* stencil,
                       const mb_col* out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, stencil, "stencil"));
  if (!in || !out || ncols < 1 || ncols > 12)
    return set_error(MB_ERR_LAUNCH, "transform_where takes 1 to 12 columns");
  for (int c = 0; c < ncols; ++c) {
    MB_TRY(check_src(ex, &in[c], "input"));
    MB_TRY(check_col(ex, out[c], "output"));
    if (in[c].len != stencil->len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input and stencil lengths differ", in[c].len,
                       stencil->len);
    if (in[c].len != out[c].len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input and output lengths differ", in[c].len,
                       out[c].len);
  }
  if (stencil->len == 0) return MB_OK;
  for (int c = 0; c < ncols; ++c) MB_TRY(transform_where_col(ex, in[c], *stencil, out[c]));
  return MB_OK;
}

int mb_gather(mb_executor* ex, const mb_src* values, const mb_src* indices, const mb_src* stencil,
              mb_col out) {
  return launch_indexed(ex, values, indices, stencil, out, true);
}

int mb_scatter(mb_executor* ex, const mb_src* values, const mb_src* indices,
               const mb_src* stencil, mb_col out) {
  return launch_indexed(ex, values, indices, stencil, out, false);
}

int mb_random_uniform_u32(mb_executor* ex, uint32_t mn, uint32_t mx, uint64_t seed,
                          uint64_t offset, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_col(ex, out, "output"));
  if (out.dtype != MB_U32) return set_error(MB_ERR_LAUNCH, "output must be u32");
  if (mn > mx) return set_error(MB_ERR_LAUNCH, "random distribution range must satisfy min <= max");
  if (out.len == 0) return MB_OK;
  uniform_u32_kernel<<<stride_grid(out.len), kThreads, 0, ex->stream>>>(
      (uint32_t*)out.data, out.len, mn, mx - mn, seed_key(seed), offset);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mb_random_uniform_u64(mb_executor* ex, uint64_t mn, uint64_t mx, uint64_t seed,
                          uint64_t offset, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_col(ex, out, "output"));
  if (out.dtype != MB_U64) return set_error(MB_ERR_LAUNCH, "output must be u64");
  if (mn > mx) return set_error(MB_ERR_LAUNCH, "random distribution range must satisfy min <= max");
  if (out.len == 0) return MB_OK;
  uniform_u64_kernel<<<stride_grid(out.len), kThreads, 0, ex->stream>>>(
      (uint64_t*)out.data, out.len, mn, mx - mn, seed_key(seed), offset);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

}  // extern "C"
