// seg_query.cu -- per-segment predicates and first-index queries.
//
// massively's ForEachSegment(CountIf / FindIf / AdjacentFind / AllOf / AnyOf
// / NoneOf / IsSorted / IsSortedUntil) (massively/src/seg/mod.rs:211-245,
// oracle verification/oracle/src/seg.rs:171-283): one u32 per segment --
// a count, a local index (the segment's length when nothing qualifies) or an
// MFlag.
//
// CountIf is the segmented reduction (ADD) of the predicate's 0 / 1 flags,
// read through a lazy map.  The other queries: one warp per segment walks it
// 128 items at a time (four 32-item rounds loaded together), takes the first
// qualifying local index from a ballot and stops there.  AllOf is "the
// first failing item is past the end", AnyOf / NoneOf compare the first
// passing item with the length, IsSorted compares IsSortedUntil with it.
// Offsets are canonical (validated when the segmentation was built); reads
// are still clamped to the values' length.

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

extern "C" int mb_seg_reduce(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                             uint64_t segment_count, int op, const void* init, mb_col out);

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kRounds = 4;

template <class T>
__device__ __forceinline__ bool pass_of(int pred, T v) {
  return map_to<uint32_t>(pred, DTypeOf<T>::value, to_bits64<T>(v)) != 0;
}

template <class T, int LESS>
__device__ __forceinline__ bool lt(T a, T b) {
  if constexpr (LESS == MB_GREATER) return b < a;
  else if constexpr (LESS == MB_TOTAL_LESS) return radix_enc<T>(a) < radix_enc<T>(b);
  else return a < b;
}

// What a warp looks for in a segment.
enum Look : int { kPass = 0, kFail = 1, kAdjEqual = 2, kDescent = 3, kCount = 4 };

template <class T, int LOOK, int LESS>
__global__ void __launch_bounds__(kThreads)
    seg_query_kernel(Src values, const uint32_t* __restrict__ offsets, uint64_t nseg, int pred,
                     int query, uint32_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (kThreads / 32);
  const uint64_t n = src_len(values);
  for (uint64_t s = blockIdx.x * (uint64_t)(kThreads / 32) + (threadIdx.x >> 5); s < nseg;
       s += warps) {
    uint64_t lo = offsets[s], hi = offsets[s + 1];
    hi = min(hi, n);
    lo = min(lo, hi);
    const uint32_t len = (uint32_t)(hi - lo);
    uint32_t found = len;  // first qualifying local index
    uint32_t count = 0;
    for (uint32_t c = 0; c < len; c += 32 * kRounds) {
      bool q[kRounds];
#pragma unroll
      for (int r = 0; r < kRounds; ++r) {
        const uint32_t l = c + r * 32 + lane;
        bool ok = false;
        if (l < len) {
          const T x = src_load<T>(values, lo + l);
          if constexpr (LOOK == kPass || LOOK == kCount) ok = pass_of<T>(pred, x);
          else if constexpr (LOOK == kFail) ok = !pass_of<T>(pred, x);
          else if constexpr (LOOK == kAdjEqual) ok = l + 1 < len && x == src_load<T>(values, lo + l + 1);
          else ok = l >= 1 && lt<T, LESS>(x, src_load<T>(values, lo + l - 1));
        }
        q[r] = ok;
      }
      uint32_t hit = 0xFFFFFFFFu;
#pragma unroll
      for (int r = kRounds - 1; r >= 0; --r) {
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, q[r]);
        if constexpr (LOOK == kCount) count += __popc(b);
        else if (b) hit = c + r * 32 + (__ffs(b) - 1);
      }
      if constexpr (LOOK != kCount) {
        if (hit != 0xFFFFFFFFu) {  // warp-uniform
          found = hit;
          break;
        }
      }
    }
    if (lane == 0) {
      uint32_t r;
      switch (query) {
        case MB_SEG_COUNT_IF: r = count; break;
        case MB_SEG_ALL_OF: case MB_SEG_NONE_OF: case MB_SEG_IS_SORTED: r = found == len; break;
        case MB_SEG_ANY_OF: r = found < len; break;
        default: r = found; break;  // FIND_IF, ADJACENT_FIND, IS_SORTED_UNTIL
      }
      out[s] = r;
    }
  }
}

template <class T>
int seg_query_run(mb_executor* ex, const mb_src& values, const uint32_t* offsets, uint64_t nseg,
                  int query, int op, uint32_t* out) {
  const Src v = to_src(values);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const unsigned g = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((nseg + kThreads / 32 - 1) / (kThreads / 32), (uint64_t)sms * 8));
#define MB_SQ(LOOK, L) \
  seg_query_kernel<T, LOOK, L><<<g, kThreads, 0, ex->stream>>>(v, offsets, nseg, op, query, out)
  switch (query) {
    case MB_SEG_COUNT_IF: MB_SQ(kCount, MB_LESS); break;
    case MB_SEG_FIND_IF: case MB_SEG_ANY_OF: case MB_SEG_NONE_OF: MB_SQ(kPass, MB_LESS); break;
    case MB_SEG_ALL_OF: MB_SQ(kFail, MB_LESS); break;
    case MB_SEG_ADJACENT_FIND: MB_SQ(kAdjEqual, MB_LESS); break;
    default:  // IS_SORTED_UNTIL, IS_SORTED
      if (op == MB_GREATER) MB_SQ(kDescent, MB_GREATER);
      else if (op == MB_TOTAL_LESS) MB_SQ(kDescent, MB_TOTAL_LESS);
      else MB_SQ(kDescent, MB_LESS);
      break;
  }
#undef MB_SQ
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

bool is_predicate(int p) {
  return p == MB_UN_IS_TRUE || p == MB_UN_IS_FALSE || p == MB_UN_IS_EVEN || p == MB_UN_IS_ODD ||
         p == MB_UN_IS_NEGATIVE || p == MB_UN_IS_POSITIVE;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_seg_query(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                 uint64_t segment_count, int query, int op, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_col(ex, out, "output"));
  MB_TRY(check_len_u32(values->len));
  if (!offsets) return set_error(MB_ERR_INVALID_SEGMENTATION, "missing offsets");
  if (out.dtype != MB_U32 && out.dtype != MB_I32)
    return set_error(MB_ERR_LAUNCH, "segment query results are u32 (MIndex / MFlag)");
  if (out.len < segment_count)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than the segment count",
                     segment_count, out.len);
  const int ct = compute_type(values->vtype);
  switch (query) {
    case MB_SEG_COUNT_IF: case MB_SEG_FIND_IF: case MB_SEG_ALL_OF: case MB_SEG_ANY_OF:
    case MB_SEG_NONE_OF:
      if (!is_predicate(op)) return set_error(MB_ERR_LAUNCH, "takes an IS_* predicate");
      if (dtype_is_float(ct) && (op == MB_UN_IS_EVEN || op == MB_UN_IS_ODD))
        return set_error(MB_ERR_LAUNCH, "IS_EVEN / IS_ODD take integer items");
      break;
    case MB_SEG_ADJACENT_FIND:
      if (op != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "adjacent_find takes EQUAL");
      break;
    case MB_SEG_IS_SORTED_UNTIL: case MB_SEG_IS_SORTED:
      if (op != MB_LESS && op != MB_GREATER && op != MB_TOTAL_LESS)
        return set_error(MB_ERR_LAUNCH, "takes LESS, GREATER or TOTAL_LESS");
      break;
    default: return set_error(MB_ERR_LAUNCH, "unknown segment query");
  }
  if (segment_count == 0) return MB_OK;
  if (query == MB_SEG_COUNT_IF && values->map == MB_UN_IDENTITY &&
      values->vtype == values->dtype && values->kind != MB_SRC_ADJACENT) {
    // a segmented sum of the predicate's 0 / 1 flags: the tiled segmented
    // reduction, item-parallel, instead of a warp per segment
    mb_src flags = *values;
    flags.map = op;
    flags.vtype = MB_U32;
    const uint32_t zero = 0;
    mb_col o = out;
    o.dtype = MB_U32;
    return mb_seg_reduce(ex, &flags, offsets, segment_count, MB_OP_ADD, &zero, o);
  }
  MB_DISPATCH_CTYPE(ct, seg_query_run, ex, *values, offsets, segment_count, query, op,
                    (uint32_t*)out.data);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

}  // extern "C"
