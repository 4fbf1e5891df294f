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

// Tile geometry.  On a plain, 16-byte-aligned column a thread reads VECS
// 16-byte vectors per tile (vector v of thread t covers items
// base + (v * kThreads + t) * VEC ...  + VEC - 1, so a warp's loads are
// contiguous); other views and the last, partial tile are read item by item
// (item j of thread t: base + j * kThreads + t).  Either way a thread's items
// of a tile come in increasing index order.
template <class T>
struct Geo {
  static constexpr int VEC = 16 / (int)sizeof(T);
  static constexpr int VECS = 4;
  static constexpr int ITEMS = VEC * VECS;       // per thread and tile
  static constexpr int TILE = kThreads * ITEMS;  // 4096 4-byte or 2048 8-byte items
};

template <class T>
__device__ __forceinline__ uint64_t vec_index(uint64_t base, int v, int e) {
  return base + ((uint64_t)v * kThreads + threadIdx.x) * Geo<T>::VEC + e;
}

template <class T>
__device__ __forceinline__ void load_vecs(const T* __restrict__ p, uint64_t base,
                                          T (&x)[Geo<T>::VECS][Geo<T>::VEC]) {
#pragma unroll
  for (int v = 0; v < Geo<T>::VECS; ++v) {
    const uint4 u = __ldcs(reinterpret_cast<const uint4*>(p + base) + v * kThreads + threadIdx.x);
    memcpy(x[v], &u, 16);
  }
}

template <class T>
__device__ __forceinline__ T shfl_t(T v, int src_lane) {
  if constexpr (sizeof(T) == 8)
    return from_bits64<T>(__shfl_sync(0xFFFFFFFFu, (unsigned long long)to_bits64<T>(v), src_lane));
  else
    return from_bits64<T>(__shfl_sync(0xFFFFFFFFu, (unsigned)to_bits64<T>(v), src_lane));
}

template <int KIND>
constexpr bool kTwoInputs = KIND == kMismatch || KIND == kEqual || KIND == kLexicographic;

__device__ __forceinline__ uint64_t pair_len(const Src& a, const Src& b) {
  const uint64_t la = src_len(a), lb = src_len(b);
  return la < lb ? la : lb;
}

// Whether item i qualifies, from its value x, its neighbour (the previous
// item for is_sorted_until / is_partitioned, the next for adjacent_find) and
// the right input's item y.
template <class T, int KIND, int LESS>
__device__ __forceinline__ bool qualifies(int pred, T x, T nb, T y) {
  if constexpr (KIND == kFindIf) return pred_holds<T>(pred, x);
  else if constexpr (KIND == kPartitioned) return pred_holds<T>(pred, x) && !pred_holds<T>(pred, nb);
  else if constexpr (KIND == kAdjacentFind) return x == nb;
  else if constexpr (KIND == kSortedUntil) return lt<T, LESS>(x, nb);
  else if constexpr (KIND == kMismatch || KIND == kEqual) return !(x == y);
  else return lt<T, LESS>(x, y) || lt<T, LESS>(y, x);
}

// KIND uses the previous item (+1 -> the next item, 0 -> none).
template <int KIND>
constexpr int kNeighbour = KIND == kAdjacentFind ? 1
                           : (KIND == kSortedUntil || KIND == kPartitioned) ? -1 : 0;

// One full tile of a plain column: the first qualifying index of this
// thread's items, or kNone.
template <class T, int KIND, int LESS>
__device__ __forceinline__ uint32_t plain_tile(const T* __restrict__ a, const T* __restrict__ b,
                                               uint64_t n, uint64_t base, int pred) {
  using G = Geo<T>;
  constexpr int NB = kNeighbour<KIND>;
  T x[G::VECS][G::VEC], y[G::VECS][G::VEC];
  load_vecs<T>(a, base, x);
  if constexpr (kTwoInputs<KIND>) load_vecs<T>(b, base, y);
  // neighbours across vector edges: the next lane's first item / the
  // previous lane's last item; across warp edges, one scalar load
  T edge[G::VECS];
  const int lane = threadIdx.x & 31;
  if constexpr (NB != 0) {
#pragma unroll
    for (int v = 0; v < G::VECS; ++v) {
      if constexpr (NB > 0) {
        edge[v] = shfl_t<T>(x[v][0], (lane + 1) & 31);
        const uint64_t j = vec_index<T>(base, v, G::VEC - 1) + 1;
        if (lane == 31 && j < n) edge[v] = a[j];
      } else {
        edge[v] = shfl_t<T>(x[v][G::VEC - 1], (lane + 31) & 31);
        const uint64_t i0 = vec_index<T>(base, v, 0);
        if (lane == 0 && i0 >= 1) edge[v] = a[i0 - 1];
      }
    }
  }
  uint32_t first = kNone;
#pragma unroll
  for (int v = 0; v < G::VECS; ++v) {
#pragma unroll
    for (int e = 0; e < G::VEC; ++e) {
      const uint64_t i = vec_index<T>(base, v, e);
      T nb = x[v][e];
      if constexpr (NB > 0) nb = e + 1 < G::VEC ? x[v][e + 1] : edge[v];
      if constexpr (NB < 0) nb = e > 0 ? x[v][e - 1] : edge[v];
      bool ok = true;
      if constexpr (NB > 0) ok = i + 1 < n;
      if constexpr (NB < 0) ok = i >= 1;
      const T yy = kTwoInputs<KIND> ? y[v][e] : x[v][e];
      if (first == kNone && ok && qualifies<T, KIND, LESS>(pred, x[v][e], nb, yy))
        first = (uint32_t)i;
    }
  }
  return first;
}

// Any tile of any view (and the partial last tile of a plain column).
template <class T, int KIND, int LESS>
__device__ __forceinline__ uint32_t view_tile(const Src& a, const Src& b, uint64_t n,
                                              uint64_t base, int pred) {
  constexpr int NB = kNeighbour<KIND>;
  uint32_t first = kNone;
#pragma unroll 4
  for (int j = 0; j < Geo<T>::ITEMS; ++j) {
    const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
    if (i >= n) break;
    if constexpr (NB > 0) {
      if (i + 1 >= n) continue;
    }
    if constexpr (NB < 0) {
      if (i == 0) continue;
    }
    const T x = src_load<T>(a, i);
    T nb = x, y = x;
    if constexpr (NB != 0) nb = src_load<T>(a, NB > 0 ? i + 1 : i - 1);
    if constexpr (kTwoInputs<KIND>) y = src_load<T>(b, i);
    if (qualifies<T, KIND, LESS>(pred, x, nb, y)) {
      first = (uint32_t)i;
      break;
    }
  }
  return first;
}

// Blocks walk tiles in increasing order, offer each tile's first hit to
// `best` and stop once `best` lies before their next tile.  The barrier at
// the top of every tile makes the exit block-uniform (and lets this block's
// own hit, offered before it, end the walk).
template <class T, int KIND, int LESS, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    find_first_kernel(Src a, Src b, int pred, uint32_t* __restrict__ best) {
  using G = Geo<T>;
  const uint64_t n = kTwoInputs<KIND> ? pair_len(a, b) : src_len(a);
  for (uint64_t base = blockIdx.x * (uint64_t)G::TILE; base < n;
       base += (uint64_t)gridDim.x * G::TILE) {
    if (__syncthreads_or(base >= (uint64_t)ld_word(best))) return;
    uint32_t first;
    if (PLAIN && base + G::TILE <= n)
      first = plain_tile<T, KIND, LESS>((const T*)a.data, (const T*)b.data, n, base, pred);
    else
      first = view_tile<T, KIND, LESS>(a, b, n, base, pred);
    if (first != kNone) atomicMin(best, first);
  }
}

// The walk of find_first_of (one item at a time; the needle loop dominates).
template <class HIT>
__device__ __forceinline__ void first_hit_tiles(uint64_t n, uint32_t* best, HIT hit) {
  for (uint64_t base = blockIdx.x * (uint64_t)kTile; base < n;
       base += (uint64_t)gridDim.x * kTile) {
    if (__syncthreads_or(base >= (uint64_t)ld_word(best))) return;
    uint32_t first = kNone;
    for (int j = 0; j < kItems; ++j) {
      const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
      if (i < n && hit(i)) {
        first = (uint32_t)i;
        break;
      }
    }
    if (first != kNone) atomicMin(best, first);
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

unsigned grid_of(mb_executor* ex, uint64_t n, uint64_t tile) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t tiles = (n + tile - 1) / tile;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)sms * 8));
}

template <class T, int KIND, int LESS>
int find_launch(mb_executor* ex, const Src& a, const Src& b, uint64_t cap, int pred, bool plain,
                uint32_t* best, uint32_t* out) {
  if (cap) {
    if constexpr (KIND == kFirstOf) {
      find_first_of_kernel<T><<<grid_of(ex, cap, kTile), kThreads, 0, ex->stream>>>(a, b, best);
    } else {
      const unsigned g = grid_of(ex, cap, Geo<T>::TILE);
      if (plain)
        find_first_kernel<T, KIND, LESS, true><<<g, kThreads, 0, ex->stream>>>(a, b, pred, best);
      else
        find_first_kernel<T, KIND, LESS, false><<<g, kThreads, 0, ex->stream>>>(a, b, pred, best);
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
  constexpr int ct = DTypeOf<T>::value;
  const bool two = kind == kMismatch || kind == kEqual || kind == kLexicographic;
  const bool plain = src_plain(a, ct) && (uintptr_t)a.data % 16 == 0 &&
                     (!two || (src_plain(b, ct) && (uintptr_t)b.data % 16 == 0));
#define MB_FIND(K, L) return find_launch<T, K, L>(ex, sa, sb, cap, op, plain, best, out)
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
// Folds one item into a thread's accumulator; a thread's items arrive in
// increasing index order.
template <class T, int LESS, int KIND>
__device__ __forceinline__ void arg_take(ArgAcc<T>& acc, T v, uint32_t i) {
  constexpr bool kLast = KIND == kMinMax;
  if constexpr (kNanAware<T, LESS>) {
    if (v != v) {
      acc.q = i + 1;
      return;
    }
  }
  if constexpr (KIND != kMaxFirst) {
    if (acc.mn.i == kNone || lt<T, LESS>(v, acc.mn.v) || (kLast && !lt<T, LESS>(acc.mn.v, v)))
      acc.mn = Cand<T>{v, i};
  }
  if constexpr (KIND != kMinFirst) {
    if (acc.mx.i == kNone || lt<T, LESS>(acc.mx.v, v)) acc.mx = Cand<T>{v, i};
  }
}

template <class T, int LESS, int KIND, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    arg_partial_kernel(Src a, const uint32_t* __restrict__ lo_word, uint64_t* __restrict__ pv,
                       uint32_t* __restrict__ pi, uint32_t* __restrict__ q_word) {
  using G = Geo<T>;
  uint64_t lo = 0;
  if (lo_word) {
    lo = *lo_word;
    if (lo == 0) return;
  }
  // vector loads need tiles that start on a 16-byte boundary
  const bool vec = PLAIN && lo % G::VEC == 0;
  const uint64_t n = src_len(a);
  ArgAcc<T> acc{{T(0), kNone}, {T(0), kNone}, 0};
  for (uint64_t base = lo + blockIdx.x * (uint64_t)G::TILE; base < n;
       base += (uint64_t)gridDim.x * G::TILE) {
    if (vec && base + G::TILE <= n) {
      T x[G::VECS][G::VEC];
      load_vecs<T>((const T*)a.data, base, x);
#pragma unroll
      for (int v = 0; v < G::VECS; ++v)
#pragma unroll
        for (int e = 0; e < G::VEC; ++e)
          arg_take<T, LESS, KIND>(acc, x[v][e], (uint32_t)vec_index<T>(base, v, e));
    } else {
#pragma unroll 4
      for (int j = 0; j < G::ITEMS; ++j) {
        const uint64_t i = base + (uint64_t)j * kThreads + threadIdx.x;
        if (i >= n) break;
        arg_take<T, LESS, KIND>(acc, src_load<T>(a, i), (uint32_t)i);
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
  const unsigned g = grid_of(ex, a.len, Geo<T>::TILE);
  const bool plain = src_plain(a, DTypeOf<T>::value) && (uintptr_t)a.data % 16 == 0;
  Scratch part;
  MB_TRY(part.alloc(ex, (size_t)g * 24 + 64));
  uint64_t* pv = part.as<uint64_t>();
  uint32_t* pi = (uint32_t*)(pv + 2 * (size_t)g);
  uint32_t* q = pi + 2 * (size_t)g;
  const Src s = to_src(a);
  constexpr bool kSecond = KIND == kMinMax && kNanAware<T, LESS>;
  if constexpr (kSecond) MB_CUDA(cudaMemsetAsync(q, 0, 4, ex->stream));
  if (plain)
    arg_partial_kernel<T, LESS, KIND, true><<<g, kThreads, 0, ex->stream>>>(
        s, nullptr, pv, pi, kSecond ? q : nullptr);
  else
    arg_partial_kernel<T, LESS, KIND, false><<<g, kThreads, 0, ex->stream>>>(
        s, nullptr, pv, pi, kSecond ? q : nullptr);
  arg_final_kernel<T, LESS, KIND><<<1, kThreads, 0, ex->stream>>>(s, pv, pi, (int)g, nullptr, out);
  if constexpr (kSecond) {
    // (rare: only after a NaN; items one by one)
    arg_partial_kernel<T, LESS, kMinMax, false><<<g, kThreads, 0, ex->stream>>>(s, q, pv, pi,
                                                                               nullptr);
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
