// seg_transform.cu -- per-segment transforms: Reverse, AdjacentDifference,
// and the length-changing Filter, Take and Unique.
//
// massively's ForEachSegment(Reverse / AdjacentDifference(op) / Filter(pred)
// / Take(k) / Unique(equal)) (massively/src/seg/mod.rs:161-209; oracle
// verification/oracle/src/seg.rs:41-46, 90-153).  One warp per segment:
//   Reverse             out[lo + len - 1 - l] = x[lo + l];
//   AdjacentDifference  out[lo] = x[lo], out[lo + l] = op(x[lo + l - 1], x[lo + l]);
//   Filter / Take / Unique keep a subsequence of every segment: a first pass
//     counts each segment's kept items (ballots) into new_offsets[s + 1], an
//     in-place inclusive scan turns the counts into the new offsets, and a
//     second pass writes each kept item at new_offsets[s] + its rank among
//     the segment's kept items (ballot prefix counts) -- stable, segments in
//     order.  Unique keeps an item when it is the segment's first or differs
//     from its predecessor, which for `==` equals massively's comparison with
//     the last kept item.

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

extern "C" int mb_inclusive_scan(mb_executor* ex, const mb_src* in, int op, mb_col out);

namespace mb {
namespace {

constexpr int kThreads = 256;

enum SegKind : int { kFilter = 0, kTake = 1, kUnique = 2 };

template <class T>
__device__ __forceinline__ bool keep_item(int kind, int param, const Src& v, uint64_t lo,
                                          uint32_t l, T x) {
  if (kind == kFilter)
    return map_to<uint32_t>(param, DTypeOf<T>::value, to_bits64<T>(x)) != 0;
  if (kind == kTake) return l < (uint32_t)param;
  return l == 0 || !(src_load<T>(v, lo + l - 1) == x);
}

__device__ __forceinline__ void seg_bounds(const uint32_t* off, uint64_t s, uint64_t n,
                                           uint64_t& lo, uint32_t& len) {
  uint64_t a = off[s], b = off[s + 1];
  b = min(b, n);
  a = min(a, b);
  lo = a;
  len = (uint32_t)(b - a);
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    seg_reverse_kernel(Src v, const uint32_t* __restrict__ off, uint64_t nseg, int out_dtype,
                       void* out, int op, int adjacent) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (kThreads / 32);
  const uint64_t n = src_len(v);
  for (uint64_t s = blockIdx.x * (uint64_t)(kThreads / 32) + (threadIdx.x >> 5); s < nseg;
       s += warps) {
    uint64_t lo;
    uint32_t len;
    seg_bounds(off, s, n, lo, len);
    for (uint32_t l = lane; l < len; l += 32) {
      const T x = src_load<T>(v, lo + l);
      if (adjacent) {
        const T y = l == 0 ? x : op_apply_rt<T>(op, src_load<T>(v, lo + l - 1), x);
        st_cast<T>(out_dtype, out, lo + l, y);
      } else {
        st_cast<T>(out_dtype, out, lo + (len - 1 - l), x);
      }
    }
  }
}

// Pass 1: kept items per segment into counts[s] (counts = new_offsets + 1).
template <class T>
__global__ void __launch_bounds__(kThreads)
    seg_keep_count_kernel(Src v, const uint32_t* __restrict__ off, uint64_t nseg, int kind,
                          int param, uint32_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (kThreads / 32);
  const uint64_t n = src_len(v);
  for (uint64_t s = blockIdx.x * (uint64_t)(kThreads / 32) + (threadIdx.x >> 5); s < nseg;
       s += warps) {
    uint64_t lo;
    uint32_t len;
    seg_bounds(off, s, n, lo, len);
    uint32_t c = 0;
    if (kind == kTake) {
      c = min(len, (uint32_t)param);
    } else {
      for (uint32_t b = 0; b < len; b += 32) {
        const uint32_t l = b + lane;
        bool k = false;
        if (l < len) k = keep_item<T>(kind, param, v, lo, l, src_load<T>(v, lo + l));
        c += __popc(__ballot_sync(0xFFFFFFFFu, k));
      }
    }
    if (lane == 0) counts[s] = c;
  }
}

// Pass 2: kept items to new_off[s] + rank.
template <class T>
__global__ void __launch_bounds__(kThreads)
    seg_keep_write_kernel(Src v, const uint32_t* __restrict__ off, uint64_t nseg, int kind,
                          int param, const uint32_t* __restrict__ new_off, int out_dtype,
                          void* out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (kThreads / 32);
  const uint64_t n = src_len(v);
  const uint32_t below = (1u << lane) - 1u;
  for (uint64_t s = blockIdx.x * (uint64_t)(kThreads / 32) + (threadIdx.x >> 5); s < nseg;
       s += warps) {
    uint64_t lo;
    uint32_t len;
    seg_bounds(off, s, n, lo, len);
    const uint64_t dst = new_off[s];
    const uint32_t limit = kind == kTake ? min(len, (uint32_t)param) : len;
    uint32_t done = 0;
    for (uint32_t b = 0; b < limit; b += 32) {
      const uint32_t l = b + lane;
      bool k = false;
      T x{};
      if (l < limit) {
        x = src_load<T>(v, lo + l);
        k = kind == kTake || keep_item<T>(kind, param, v, lo, l, x);
      }
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, k);
      if (k) st_cast<T>(out_dtype, out, dst + done + __popc(bal & below), x);
      done += __popc(bal);
    }
  }
}

unsigned warp_grid(mb_executor* ex, uint64_t nseg) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  return (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((nseg + kThreads / 32 - 1) / (kThreads / 32), (uint64_t)sms * 8));
}

template <class T>
int reverse_run(mb_executor* ex, const mb_src& values, const uint32_t* off, uint64_t nseg,
                const mb_col& out, int op, int adjacent) {
  seg_reverse_kernel<T><<<warp_grid(ex, nseg), kThreads, 0, ex->stream>>>(
      to_src(values), off, nseg, out.dtype, out.data, op, adjacent);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T>
int keep_run(mb_executor* ex, const mb_src& values, const uint32_t* off, uint64_t nseg, int kind,
             int param, const mb_col& out, uint32_t* new_off) {
  const Src v = to_src(values);
  const unsigned g = warp_grid(ex, nseg);
  MB_CUDA(cudaMemsetAsync(new_off, 0, 4, ex->stream));
  seg_keep_count_kernel<T><<<g, kThreads, 0, ex->stream>>>(v, off, nseg, kind, param,
                                                           new_off + 1);
  MB_CUDA(cudaGetLastError());
  // counts -> offsets, in place (each tile is read before it is written)
  mb_src cs{};
  cs.kind = MB_SRC_COLUMN;
  cs.dtype = cs.vtype = MB_U32;
  cs.map = MB_UN_IDENTITY;
  cs.data = new_off + 1;
  cs.len = nseg;
  mb_col co{};
  co.data = new_off + 1;
  co.dtype = MB_U32;
  co.len = nseg;
  MB_TRY(mb_inclusive_scan(ex, &cs, MB_OP_ADD, co));
  seg_keep_write_kernel<T><<<g, kThreads, 0, ex->stream>>>(v, off, nseg, kind, param, new_off,
                                                           out.dtype, out.data);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int check_common(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                 const mb_col& out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_col(ex, out, "output"));
  MB_TRY(check_len_u32(values->len));
  if (!offsets) return set_error(MB_ERR_INVALID_SEGMENTATION, "missing offsets");
  if (compute_type(out.dtype) != compute_type(values->vtype))
    return set_error(MB_ERR_LAUNCH, "output element type differs from the values'");
  if (out.len < values->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than the values", values->len,
                     out.len);
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_seg_reverse(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                   uint64_t segment_count, mb_col out) {
  MB_TRY(check_common(ex, values, offsets, out));
  if (segment_count == 0 || values->len == 0) return MB_OK;
  MB_DISPATCH_CTYPE(compute_type(values->vtype), reverse_run, ex, *values, offsets,
                    segment_count, out, 0, 0);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int mb_seg_adjacent_difference(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                               uint64_t segment_count, int op, mb_col out) {
  MB_TRY(check_common(ex, values, offsets, out));
  if (!op_valid_for(op, compute_type(values->vtype)))
    return set_error(MB_ERR_LAUNCH, "operator not defined for this type");
  if (segment_count == 0 || values->len == 0) return MB_OK;
  MB_DISPATCH_CTYPE(compute_type(values->vtype), reverse_run, ex, *values, offsets,
                    segment_count, out, op, 1);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int mb_seg_keep(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                uint64_t segment_count, int kind, int param, mb_col out, uint32_t* new_offsets,
                uint32_t* count_dev, uint32_t* count_host) {
  MB_TRY(check_common(ex, values, offsets, out));
  if (!new_offsets) return set_error(MB_ERR_UNBOUND_COLUMN, "missing new offsets");
  const int ct = compute_type(values->vtype);
  if (kind == kFilter) {
    if (param != MB_UN_IS_TRUE && param != MB_UN_IS_FALSE && param != MB_UN_IS_EVEN &&
        param != MB_UN_IS_ODD && param != MB_UN_IS_NEGATIVE && param != MB_UN_IS_POSITIVE)
      return set_error(MB_ERR_LAUNCH, "filter takes an IS_* predicate");
    if (dtype_is_float(ct) && (param == MB_UN_IS_EVEN || param == MB_UN_IS_ODD))
      return set_error(MB_ERR_LAUNCH, "IS_EVEN / IS_ODD take integer items");
  } else if (kind == kTake) {
    if (param < 0) return set_error(MB_ERR_LAUNCH, "take count must not be negative");
  } else if (kind == kUnique) {
    if (param != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "unique takes EQUAL");
  } else {
    return set_error(MB_ERR_LAUNCH, "unknown segment selection");
  }
  if (segment_count == 0) {
    MB_CUDA(cudaMemsetAsync(new_offsets, 0, 4, ex->stream));
  } else {
    const int st = [&]() -> int {
      MB_DISPATCH_CTYPE(ct, keep_run, ex, *values, offsets, segment_count, kind, param, out,
                        new_offsets);
      return set_error(MB_ERR_LAUNCH, "unsupported element type");
    }();
    MB_TRY(st);
  }
  if (count_dev)
    MB_CUDA(cudaMemcpyAsync(count_dev, new_offsets + segment_count, 4, cudaMemcpyDeviceToDevice,
                            ex->stream));
  if (count_host) MB_TRY(read_u32(ex, new_offsets + segment_count, count_host));
  return MB_OK;
}

}  // extern "C"
