// predicate.cu -- first-index searches and index-carrying extrema.
//
// massively's find_if / is_partitioned (massively/src/api/algorithm/
// predicate.rs:218, core/predicate.rs:204-223), adjacent_find /
// is_sorted_until / is_sorted / min_element / max_element / minmax_element
// (api/algorithm/ordering.rs:107, 213, 256, 300-380, core/arg_reduce.rs) and
// find_first_of / equal / mismatch / lexicographical_compare
// (api/algorithm/search.rs:33, 175, 231, 289), with the results of the
// sequential definitions in verification/oracle/src/vector.rs:212-218,
// 317-378, 428-481.
//
// First-index searches.  massively reduces a per-item candidate index
// (MIndex::MAX where the item does not qualify) with a minimum over every
// item.  Here blocks walk tiles of 2048 items in increasing order, offer the
// first qualifying index of a tile to one device word with atomicMin, and
// stop once that word lies before their next tile -- so an early hit ends
// the pass after a few tiles instead of after the whole input.  A one-thread
// kernel then turns the word into the API's value (None, the length, a flag)
// on the device, so the result needs no host round trip.
//
// Extrema.  The sequential definitions keep the first minimum
// (min_element), the first maximum (max_element and minmax's maximum) and the
// last minimum (minmax's minimum: it moves on `!less(x[min], x[i])`).  For a
// strict weak order these are the extrema under (value, index) with the tie
// broken toward the lower or higher index, a commutative and associative
// choice, so per-thread folds, a block tree and a one-block pass over the
// block partials give the sequential answer.  Under the IEEE `<` (and `>`) a
// NaN is not ordered and the sequential scan behaves as follows, which the
// kernels reproduce exactly:
//   * first minimum / first maximum: a NaN at index 0 is kept forever
//     (nothing compares below or above it); a NaN anywhere else is never
//     taken.  So: 0 when x[0] is NaN, else the extremum of the non-NaN items.
//   * last minimum: a NaN at the current minimum or at item i both make
//     `!less` true, so the scan restarts after the last NaN q: the answer is
//     the last minimum of the items after q, or q itself when q is last.  The
//     first pass records q (atomicMax); a second pass, whose kernels return at
//     once when no NaN was seen, redoes the minimum over (q, n).

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr uint32_t kNone = 0xFFFFFFFFu;  // MIndex::MAX: no index
constexpr int kNeedleSmem = 2048;        // needles staged in shared memory

enum FindKind : int {
  kFindIf = 0,
  kPartitioned = 1,
  kAdjacentFind = 2,
  kSortedUntil = 3,
  kMismatch = 4,
  kEqual = 5,
  kLexicographic = 6,
  kFirstOf = 7,
};

template <class T, int LESS>
__device__ __forceinline__ bool lt(T a, T b) {
  if constexpr (LESS == MB_GREATER) return b < a;
  else if constexpr (LESS == MB_TOTAL_LESS) return radix_enc<T>(a) < radix_enc<T>(b);
  else return a < b;
}

template <class T>
__device__ __forceinline__ uint64_t bits_of(T v) {
  return to_bits64<T>(v);
}

template <class T>
__device__ __forceinline__ T from_bits(uint64_t b) {
  return from_bits64<T>(b);
}

// A built-in predicate (an mb_unary IS_* map) on a value of compute type T.
template <class T>
__device__ __forceinline__ bool pred_holds(int pred, T v) {
  return map_to<uint32_t>(pred, DTypeOf<T>::value, bits_of(v)) != 0;
}

__device__ __forceinline__ uint32_t ld_word(const uint32_t* p) {
  return *(const volatile uint32_t*)p;
}

// The tile walk shared by every first-index search.  `hit(i)` tells whether
// item i < n qualifies.  All exits are block-uniform.
template <class HIT>
__device__ __forceinline__ void first_hit_tiles(uint64_t n, uint32_t* best, HIT hit) {
  for (uint64_t base = blockIdx.x * (uint64_t)kTile; base < n;
       base += (uint64_t)gridDim.x * kTile) {
    if (__syncthreads_or(base >= (uint64_t)ld_word(best))) return;
    bool h[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
      h[j] = i < n && hit(i);
    }
    uint32_t first = kNone;
#pragma unroll
    for (int j = kItems - 1; j >= 0; --j)
      if (h[j]) first = (uint32_t)(base + (uint64_t)j * kThreads + threadIdx.x);
    if (first != kNone) atomicMin(best, first);
    if (__syncthreads_or(first != kNone)) return;
  }
}

__device__ __forceinline__ uint64_t pair_len(const Src& a, const Src& b) {
  const uint64_t la = src_len(a), lb = src_len(b);
  return la < lb ? la : lb;
}

template <class T, int KIND, int LESS>
__global__ void __launch_bounds__(kThreads)
    find_first_kernel(Src a, Src b, int pred, uint32_t* __restrict__ best) {
  if constexpr (KIND == kFindIf) {
    first_hit_tiles(src_len(a), best,
                    [&](uint64_t i) { return pred_holds<T>(pred, src_load<T>(a, i)); });
  } else if constexpr (KIND == kPartitioned) {
    // the first passing item that follows a failing one
    first_hit_tiles(src_len(a), best, [&](uint64_t i) {
      return i >= 1 && pred_holds<T>(pred, src_load<T>(a, i)) &&
             !pred_holds<T>(pred, src_load<T>(a, i - 1));
    });
  } else if constexpr (KIND == kAdjacentFind) {
    const uint64_t n = src_len(a);
    first_hit_tiles(n, best, [&](uint64_t i) {
      return i + 1 < n && src_load<T>(a, i) == src_load<T>(a, i + 1);
    });
  } else if constexpr (KIND == kSortedUntil) {
    first_hit_tiles(src_len(a), best, [&](uint64_t i) {
      return i >= 1 && lt<T, LESS>(src_load<T>(a, i), src_load<T>(a, i - 1));
    });
  } else if constexpr (KIND == kMismatch || KIND == kEqual) {
    first_hit_tiles(pair_len(a, b), best,
                    [&](uint64_t i) { return !(src_load<T>(a, i) == src_load<T>(b, i)); });
  } else {
    first_hit_tiles(pair_len(a, b), best, [&](uint64_t i) {
      const T x = src_load<T>(a, i), y = src_load<T>(b, i);
      return lt<T, LESS>(x, y) || lt<T, LESS>(y, x);
    });
  }
}

// find_first_of: needles staged once per block in shared memory (the first
// kNeedleSmem of them; any beyond are read from global memory).
template <class T>
__global__ void __launch_bounds__(kThreads)
    find_first_of_kernel(Src a, Src needles, uint32_t* __restrict__ best) {
  __shared__ T s_need[kNeedleSmem];
  const uint64_t m = src_len(needles);
  const int ms = m < (uint64_t)kNeedleSmem ? (int)m : kNeedleSmem;
  for (int k = threadIdx.x; k < ms; k += kThreads) s_need[k] = src_load<T>(needles, k);
  __syncthreads();
  first_hit_tiles(src_len(a), best, [&](uint64_t i) {
    const T x = src_load<T>(a, i);
    bool any = false;
    for (int k = 0; k < ms && !any; ++k) any = x == s_need[k];
    for (uint64_t k = ms; k < m && !any; ++k) any = x == src_load<T>(needles, k);
    return any;
  });
}

// The API value of a search from its first-hit word.
template <class T, int KIND, int LESS>
__global__ void find_finish_kernel(Src a, Src b, const uint32_t* __restrict__ best,
                                   uint32_t* __restrict__ out) {
  const uint32_t h = *best;
  uint32_t r = h;
  if constexpr (KIND == kSortedUntil) {
    r = h == kNone ? (uint32_t)src_len(a) : h;
  } else if constexpr (KIND == kPartitioned) {
    r = h == kNone ? 1u : 0u;
  } else if constexpr (KIND == kMismatch) {
    if (h == kNone) r = src_len(a) == src_len(b) ? kNone : (uint32_t)pair_len(a, b);
  } else if constexpr (KIND == kEqual) {
    r = src_len(a) == src_len(b) && h == kNone ? 1u : 0u;
  } else if constexpr (KIND == kLexicographic) {
    r = h == kNone ? (src_len(a) < src_len(b) ? 1u : 0u)
                   : (lt<T, LESS>(src_load<T>(a, h), src_load<T>(b, h)) ? 1u : 0u);
  }
  *out = r;
}

unsigned grid_of(mb_executor* ex, uint64_t n) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t tiles = (n + kTile - 1) / kTile;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)sms * 8));
}

template <class T, int KIND, int LESS>
int find_launch(mb_executor* ex, const Src& a, const Src& b, uint64_t cap, int pred,
                uint32_t* best, uint32_t* out) {
  if (cap) {
    if constexpr (KIND == kFirstOf) {
      find_first_of_kernel<T><<<grid_of(ex, cap), kThreads, 0, ex->stream>>>(a, b, best);
    } else {
      find_first_kernel<T, KIND, LESS><<<grid_of(ex, cap), kThreads, 0, ex->stream>>>(a, b, pred,
                                                                                    best);
    }
    MB_CUDA(cudaGetLastError());
  }
  find_finish_kernel<T, KIND, LESS><<<1, 1, 0, ex->stream>>>(a, b, best, out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T>
int find_run(mb_executor* ex, int kind, const mb_src& a, const mb_src& b, uint64_t cap, int op,
             uint32_t* best, uint32_t* out) {
  const Src sa = to_src(a), sb = to_src(b);
#define MB_FIND(K, L) return find_launch<T, K, L>(ex, sa, sb, cap, op, best, out)
#define MB_FIND_LESS(K)                            \
  switch (op) {                                    \
    case MB_GREATER: MB_FIND(K, MB_GREATER);       \
    case MB_TOTAL_LESS: MB_FIND(K, MB_TOTAL_LESS); \
    default: MB_FIND(K, MB_LESS);                  \
  }
  switch (kind) {
    case kFindIf: MB_FIND(kFindIf, MB_LESS);
    case kPartitioned: MB_FIND(kPartitioned, MB_LESS);
    case kAdjacentFind: MB_FIND(kAdjacentFind, MB_LESS);
    case kSortedUntil: MB_FIND_LESS(kSortedUntil);
    case kMismatch: MB_FIND(kMismatch, MB_LESS);
    case kEqual: MB_FIND(kEqual, MB_LESS);
    case kLexicographic: MB_FIND_LESS(kLexicographic);
    default: MB_FIND(kFirstOf, MB_LESS);
  }
#undef MB_FIND_LESS
#undef MB_FIND
}

bool is_predicate(int p) {
  return p == MB_UN_IS_TRUE || p == MB_UN_IS_FALSE || p == MB_UN_IS_EVEN || p == MB_UN_IS_ODD ||
         p == MB_UN_IS_NEGATIVE || p == MB_UN_IS_POSITIVE;
}

bool is_order(int less) { return less == MB_LESS || less == MB_GREATER || less == MB_TOTAL_LESS; }

// Validates, runs the search and delivers the u32 result to `out_dev`
// and / or `out_host`.
int find_entry(mb_executor* ex, int kind, const mb_src* a, const mb_src* b, int op,
               uint32_t* out_dev, uint32_t* out_host) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, a, "input"));
  const bool two =
      kind == kMismatch || kind == kEqual || kind == kLexicographic || kind == kFirstOf;
  if (two) {
    MB_TRY(check_src(ex, b, kind == kFirstOf ? "needles" : "right"));
    if (compute_type(a->vtype) != compute_type(b->vtype))
      return set_error(MB_ERR_LAUNCH, "the two inputs' element types differ");
    MB_TRY(check_len_u32(b->len));
  }
  MB_TRY(check_len_u32(a->len));
  if ((kind == kFindIf || kind == kPartitioned) && dtype_is_float(compute_type(a->vtype)) &&
      (op == MB_UN_IS_EVEN || op == MB_UN_IS_ODD))
    return set_error(MB_ERR_LAUNCH, "IS_EVEN / IS_ODD take integer items");
  uint64_t cap = a->len;
  if (kind == kMismatch || kind == kEqual || kind == kLexicographic)
    cap = std::min<uint64_t>(a->len, b->len);
  if (kind == kFirstOf && b->len == 0) cap = 0;
  Scratch word;
  MB_TRY(word.alloc(ex, 16));
  uint32_t* best = word.as<uint32_t>();
  uint32_t* out = out_dev ? out_dev : best + 1;
  MB_CUDA(cudaMemsetAsync(best, 0xFF, 4, ex->stream));
  {
    TimedLaunch tl(ex, MB_KF_SEARCH);
    const mb_src& bb = two ? *b : *a;
    const int st = [&]() -> int {
      MB_DISPATCH_CTYPE(compute_type(a->vtype), find_run, ex, kind, *a, bb, cap, op, best, out);
      return set_error(MB_ERR_LAUNCH, "unsupported element type");
    }();
    MB_TRY(st);
  }
  if (out_host) MB_TRY(read_u32(ex, out, out_host));
  return MB_OK;
}

// ------------------------------------------------------------- extrema --

enum ArgKind : int { kMinFirst = 0, kMaxFirst = 1, kMinMax = 2 };

// A (value, index) candidate; i == kNone marks "none".
template <class T>
struct Cand {
  T v;
  uint32_t i;
};

template <class T, int LESS>
__device__ __forceinline__ Cand<T> pick_min(Cand<T> x, Cand<T> y, bool last) {
  if (x.i == kNone) return y;
  if (y.i == kNone) return x;
  const bool take =
      lt<T, LESS>(y.v, x.v) || (!lt<T, LESS>(x.v, y.v) && (last ? y.i > x.i : y.i < x.i));
  return take ? y : x;
}

template <class T, int LESS>
__device__ __forceinline__ Cand<T> pick_max(Cand<T> x, Cand<T> y) {
  if (x.i == kNone) return y;
  if (y.i == kNone) return x;
  const bool take = lt<T, LESS>(x.v, y.v) || (!lt<T, LESS>(y.v, x.v) && y.i < x.i);
  return take ? y : x;
}

template <class T>
__device__ __forceinline__ Cand<T> shfl_cand(Cand<T> c, int d) {
  Cand<T> r;
  r.v = from_bits<T>(__shfl_down_sync(0xFFFFFFFFu, (unsigned long long)bits_of(c.v), d));
  r.i = __shfl_down_sync(0xFFFFFFFFu, c.i, d);
  return r;
}

// IEEE orders (LESS, GREATER) on floating types leave NaN unordered.
template <class T, int LESS>
constexpr bool kNanAware = std::is_floating_point<T>::value && LESS != MB_TOTAL_LESS;

template <class T>
struct ArgAcc {
  Cand<T> mn, mx;
  uint32_t q;  // last NaN index + 1 (0: none)
};

// Block-wide combination; the result is valid in thread 0.
template <class T, int LESS, int KIND>
__device__ ArgAcc<T> block_combine(ArgAcc<T> acc) {
  constexpr bool kLast = KIND == kMinMax;
  __shared__ uint64_t s_mv[kThreads / 32], s_xv[kThreads / 32];
  __shared__ uint32_t s_mi[kThreads / 32], s_xi[kThreads / 32], s_q[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // (a lane past the end of the warp reads its own candidate back: a tie
  // with the same index, which every pick resolves to the candidate itself)
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    if constexpr (KIND != kMaxFirst)
      acc.mn = pick_min<T, LESS>(acc.mn, shfl_cand(acc.mn, d), kLast);
    if constexpr (KIND != kMinFirst) acc.mx = pick_max<T, LESS>(acc.mx, shfl_cand(acc.mx, d));
    acc.q = max(acc.q, __shfl_down_sync(0xFFFFFFFFu, acc.q, d));
  }
  if (lane == 0) {
    s_mv[warp] = bits_of(acc.mn.v);
    s_mi[warp] = acc.mn.i;
    s_xv[warp] = bits_of(acc.mx.v);
    s_xi[warp] = acc.mx.i;
    s_q[warp] = acc.q;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w) {
      if constexpr (KIND != kMaxFirst)
        acc.mn = pick_min<T, LESS>(acc.mn, Cand<T>{from_bits<T>(s_mv[w]), s_mi[w]}, kLast);
      if constexpr (KIND != kMinFirst)
        acc.mx = pick_max<T, LESS>(acc.mx, Cand<T>{from_bits<T>(s_xv[w]), s_xi[w]});
      acc.q = max(acc.q, s_q[w]);
    }
  }
  return acc;
}

// Per-block extrema of items [lo, n), lo = *lo_word when lo_word is given
// (the pass after the last NaN; the kernel returns at once if there was
// none).  Partials per block: the minimum's and the maximum's value bits
// (pv[2b], pv[2b+1]) and indices (pi[2b], pi[2b+1]).
template <class T, int LESS, int KIND>
__global__ void __launch_bounds__(kThreads)
    arg_partial_kernel(Src a, const uint32_t* __restrict__ lo_word, uint64_t* __restrict__ pv,
                       uint32_t* __restrict__ pi, uint32_t* __restrict__ q_word) {
  constexpr bool kLast = KIND == kMinMax;
  uint64_t lo = 0;
  if (lo_word) {
    lo = *lo_word;
    if (lo == 0) return;
  }
  const uint64_t n = src_len(a);
  ArgAcc<T> acc{{T(0), kNone}, {T(0), kNone}, 0};
  for (uint64_t base = lo + blockIdx.x * (uint64_t)kTile; base < n;
       base += (uint64_t)gridDim.x * kTile) {
    T v[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
      v[j] = i < n ? src_load<T>(a, i) : T(0);
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
      if (i >= n) break;
      if constexpr (kNanAware<T, LESS>) {
        if (v[j] != v[j]) {
          acc.q = (uint32_t)i + 1;
          continue;
        }
      }
      // this thread's items arrive in increasing index order
      const Cand<T> c{v[j], (uint32_t)i};
      if constexpr (KIND != kMaxFirst) {
        if (acc.mn.i == kNone || lt<T, LESS>(c.v, acc.mn.v) ||
            (kLast && !lt<T, LESS>(acc.mn.v, c.v)))
          acc.mn = c;
      }
      if constexpr (KIND != kMinFirst) {
        if (acc.mx.i == kNone || lt<T, LESS>(acc.mx.v, c.v)) acc.mx = c;
      }
    }
  }
  acc = block_combine<T, LESS, KIND>(acc);
  if (threadIdx.x == 0) {
    pv[2 * blockIdx.x] = bits_of(acc.mn.v);
    pi[2 * blockIdx.x] = acc.mn.i;
    pv[2 * blockIdx.x + 1] = bits_of(acc.mx.v);
    pi[2 * blockIdx.x + 1] = acc.mx.i;
    if (q_word && acc.q) atomicMax(q_word, acc.q);
  }
}

// Folds the block partials into out[0] (the minimum's or the maximum's
// index) and, for minmax, out[1] (the maximum's).  With lo_word given this
// is the pass after the last NaN q: it rewrites out[0] with the last minimum
// after q, or q when nothing follows it.
template <class T, int LESS, int KIND>
__global__ void __launch_bounds__(kThreads)
    arg_final_kernel(Src a, const uint64_t* __restrict__ pv, const uint32_t* __restrict__ pi,
                     int parts, const uint32_t* __restrict__ lo_word, uint32_t* __restrict__ out) {
  constexpr bool kLast = KIND == kMinMax;
  if (lo_word && *lo_word == 0) return;
  ArgAcc<T> acc{{T(0), kNone}, {T(0), kNone}, 0};
  for (int b = threadIdx.x; b < parts; b += kThreads) {
    if constexpr (KIND != kMaxFirst)
      acc.mn = pick_min<T, LESS>(acc.mn, Cand<T>{from_bits<T>(pv[2 * b]), pi[2 * b]}, kLast);
    if constexpr (KIND != kMinFirst)
      acc.mx = pick_max<T, LESS>(acc.mx, Cand<T>{from_bits<T>(pv[2 * b + 1]), pi[2 * b + 1]});
  }
  acc = block_combine<T, LESS, KIND>(acc);
  if (threadIdx.x != 0) return;
  if (lo_word) {
    out[0] = acc.mn.i != kNone ? acc.mn.i : *lo_word - 1;
    return;
  }
  if (src_len(a) == 0) {
    out[0] = kNone;
    if (KIND == kMinMax) out[1] = kNone;
    return;
  }
  bool nan0 = false;
  if constexpr (kNanAware<T, LESS>) {
    const T x0 = src_load<T>(a, 0);
    nan0 = x0 != x0;
  }
  // a NaN at index 0 is the first minimum and the first maximum
  if constexpr (KIND == kMinFirst) {
    out[0] = nan0 ? 0u : acc.mn.i;
  } else if constexpr (KIND == kMaxFirst) {
    out[0] = nan0 ? 0u : acc.mx.i;
  } else {
    out[0] = acc.mn.i;  // rewritten by the pass after the last NaN, if any
    out[1] = nan0 ? 0u : acc.mx.i;
  }
}

template <class T, int LESS, int KIND>
int arg_launch(mb_executor* ex, const mb_src& a, uint32_t* out) {
  const unsigned g = grid_of(ex, a.len);
  Scratch part;
  MB_TRY(part.alloc(ex, (size_t)g * 24 + 64));
  uint64_t* pv = part.as<uint64_t>();
  uint32_t* pi = (uint32_t*)(pv + 2 * (size_t)g);
  uint32_t* q = pi + 2 * (size_t)g;
  const Src s = to_src(a);
  constexpr bool kSecond = KIND == kMinMax && kNanAware<T, LESS>;
  if constexpr (kSecond) MB_CUDA(cudaMemsetAsync(q, 0, 4, ex->stream));
  arg_partial_kernel<T, LESS, KIND><<<g, kThreads, 0, ex->stream>>>(s, nullptr, pv, pi,
                                                                   kSecond ? q : nullptr);
  arg_final_kernel<T, LESS, KIND><<<1, kThreads, 0, ex->stream>>>(s, pv, pi, (int)g, nullptr, out);
  if constexpr (kSecond) {
    arg_partial_kernel<T, LESS, kMinMax><<<g, kThreads, 0, ex->stream>>>(s, q, pv, pi, nullptr);
    arg_final_kernel<T, LESS, kMinMax><<<1, kThreads, 0, ex->stream>>>(s, pv, pi, (int)g, q, out);
  }
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T>
int arg_run(mb_executor* ex, int kind, const mb_src& a, int less, uint32_t* out) {
#define MB_ARG(K)                                                           \
  switch (less) {                                                           \
    case MB_GREATER: return arg_launch<T, MB_GREATER, K>(ex, a, out);       \
    case MB_TOTAL_LESS: return arg_launch<T, MB_TOTAL_LESS, K>(ex, a, out); \
    default: return arg_launch<T, MB_LESS, K>(ex, a, out);                  \
  }
  switch (kind) {
    case kMaxFirst: MB_ARG(kMaxFirst);
    case kMinMax: MB_ARG(kMinMax);
    default: MB_ARG(kMinFirst);
  }
#undef MB_ARG
}

// Writes 1 u32 result (2 for minmax: minimum, maximum) to out_dev and / or
// out_host.
int arg_entry(mb_executor* ex, int kind, const mb_src* a, int less, uint32_t* out_dev,
              uint32_t* out_host) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, a, "input"));
  MB_TRY(check_len_u32(a->len));
  if (!is_order(less)) return set_error(MB_ERR_LAUNCH, "takes LESS, GREATER or TOTAL_LESS");
  if (out_host && ex->capturing)
    return set_error(MB_ERR_LAUNCH, "a host-valued result cannot be read inside graph capture");
  const int count = kind == kMinMax ? 2 : 1;
  Scratch word;
  MB_TRY(word.alloc(ex, 16));
  uint32_t* out = out_dev ? out_dev : word.as<uint32_t>();
  {
    TimedLaunch tl(ex, MB_KF_SEARCH);
    const int st = [&]() -> int {
      MB_DISPATCH_CTYPE(compute_type(a->vtype), arg_run, ex, kind, *a, less, out);
      return set_error(MB_ERR_LAUNCH, "unsupported element type");
    }();
    MB_TRY(st);
  }
  if (out_host) {
    MB_CUDA(cudaMemcpyAsync(ex->host_pinned, out, 4 * count, cudaMemcpyDeviceToHost, ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
    for (int k = 0; k < count; ++k) out_host[k] = ex->host_pinned[k];
  }
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_find_if(mb_executor* ex, const mb_src* input, int pred, uint32_t* index_dev,
               uint32_t* index_host) {
  if (!is_predicate(pred)) return set_error(MB_ERR_LAUNCH, "find_if takes an IS_* predicate");
  return find_entry(ex, kFindIf, input, nullptr, pred, index_dev, index_host);
}

int mb_is_partitioned(mb_executor* ex, const mb_src* input, int pred, uint32_t* flag_dev,
                      uint32_t* flag_host) {
  if (!is_predicate(pred))
    return set_error(MB_ERR_LAUNCH, "is_partitioned takes an IS_* predicate");
  return find_entry(ex, kPartitioned, input, nullptr, pred, flag_dev, flag_host);
}

int mb_adjacent_find(mb_executor* ex, const mb_src* input, int equal, uint32_t* index_dev,
                     uint32_t* index_host) {
  if (equal != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "adjacent_find takes EQUAL");
  return find_entry(ex, kAdjacentFind, input, nullptr, 0, index_dev, index_host);
}

int mb_is_sorted_until(mb_executor* ex, const mb_src* input, int less, uint32_t* index_dev,
                       uint32_t* index_host) {
  if (!is_order(less))
    return set_error(MB_ERR_LAUNCH, "is_sorted_until takes LESS, GREATER or TOTAL_LESS");
  return find_entry(ex, kSortedUntil, input, nullptr, less, index_dev, index_host);
}

int mb_find_first_of(mb_executor* ex, const mb_src* source, const mb_src* needles, int equal,
                     uint32_t* index_dev, uint32_t* index_host) {
  if (equal != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "find_first_of takes EQUAL");
  return find_entry(ex, kFirstOf, source, needles, 0, index_dev, index_host);
}

int mb_mismatch(mb_executor* ex, const mb_src* left, const mb_src* right, int equal,
                uint32_t* index_dev, uint32_t* index_host) {
  if (equal != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "mismatch takes EQUAL");
  return find_entry(ex, kMismatch, left, right, 0, index_dev, index_host);
}

int mb_equal(mb_executor* ex, const mb_src* left, const mb_src* right, int equal,
             uint32_t* flag_dev, uint32_t* flag_host) {
  if (equal != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "equal takes EQUAL");
  return find_entry(ex, kEqual, left, right, 0, flag_dev, flag_host);
}

int mb_lexicographical_compare(mb_executor* ex, const mb_src* left, const mb_src* right, int less,
                               uint32_t* flag_dev, uint32_t* flag_host) {
  if (!is_order(less))
    return set_error(MB_ERR_LAUNCH, "lexicographical_compare takes LESS, GREATER or TOTAL_LESS");
  return find_entry(ex, kLexicographic, left, right, less, flag_dev, flag_host);
}

int mb_min_element(mb_executor* ex, const mb_src* input, int less, uint32_t* index_dev,
                   uint32_t* index_host) {
  return arg_entry(ex, kMinFirst, input, less, index_dev, index_host);
}

int mb_max_element(mb_executor* ex, const mb_src* input, int less, uint32_t* index_dev,
                   uint32_t* index_host) {
  return arg_entry(ex, kMaxFirst, input, less, index_dev, index_host);
}

int mb_minmax_element(mb_executor* ex, const mb_src* input, int less, uint32_t* index_dev,
                      uint32_t* index_host) {
  return arg_entry(ex, kMinMax, input, less, index_dev, index_host);
}

}  // extern "C"
