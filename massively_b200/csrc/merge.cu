// merge.cu -- merge-path merge / merge_by_key and the multiset set
// operations.
//
// Merge (massively/src/core/merge.rs:24-1230: a merge-path control kernel
// of 64 threads x 4 items writing a permutation, then a separate apply pass
// for the payload) becomes two: a small kernel finds the merge-path split of
// every tile boundary (all binary searches at once), then every block reads
// its two splits, stages its slice of both inputs in shared memory, each
// thread finds its own split there and merges kItems outputs serially (an
// odd count, so the threads' strided shared-memory accesses fall in distinct
// banks), and the block writes keys and payload columns with coalesced
// stores.  Ties take the left element first (vector.rs:493-513 of massively's
// oracle: the right element is taken only when strictly less).
//
// Set operations (massively/src/core/set.rs:14-401) keep massively's
// occurrence-rank rule: the k-th copy of a value in one input is kept by
// intersection when the other input holds more than k copies, by difference
// when it holds at most k; union is the merge of the left input with the
// right input's extra copies.  Ranks and counts come from binary searches;
// the kept elements are compacted by the single-pass selection kernel and the
// result count stays on the device.

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"

namespace mb {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 9;  // odd: conflict-free strided shared-memory access
constexpr int kTile = kThreads * kItems;
constexpr int kMaxPay = 12;

template <class T>
__device__ __forceinline__ bool cmp_less(int less, T a, T b) {
  switch (less) {
    case MB_GREATER: return b < a;
    case MB_TOTAL_LESS: return radix_enc<T>(a) < radix_enc<T>(b);
    default: return a < b;
  }
}

// The comparison with the predicate fixed at compile time (hot kernels).
template <class T, int LESS>
__device__ __forceinline__ bool cmp_ct(T a, T b) {
  if constexpr (LESS == MB_GREATER) return b < a;
  else if constexpr (LESS == MB_TOTAL_LESS) return radix_enc<T>(a) < radix_enc<T>(b);
  else return a < b;
}

// Element i of an input: a direct load for plain columns of type T, the
// lazy-view loader otherwise.
template <class T, bool PLAIN>
__device__ __forceinline__ T merge_load(const Src& s, uint64_t i) {
  if constexpr (PLAIN) return ((const T*)s.data)[i];
  else return src_load<T>(s, i);
}

// Number of left elements among the first d outputs of the stable merge.
template <class T, int LESS, bool PLAIN>
__device__ uint64_t merge_path(const Src& L, const Src& R, uint64_t nl, uint64_t nr, uint64_t d) {
  uint64_t lo = d > nr ? d - nr : 0;
  uint64_t hi = d < nl ? d : nl;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    const T l = merge_load<T, PLAIN>(L, mid);
    const T r = merge_load<T, PLAIN>(R, d - 1 - mid);
    if (!cmp_ct<T, LESS>(r, l)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

struct Payload {
  int ncols;
  Src left[kMaxPay];
  Src right[kMaxPay];
  void* out[kMaxPay];
  int esize[kMaxPay];
};

__device__ __forceinline__ void st_raw_pay(void* p, uint64_t i, int esize, uint64_t bits) {
  switch (esize) {
    case 1: ((uint8_t*)p)[i] = (uint8_t)bits; break;
    case 2: ((uint16_t*)p)[i] = (uint16_t)bits; break;
    case 4: ((uint32_t*)p)[i] = (uint32_t)bits; break;
    default: ((uint64_t*)p)[i] = bits; break;
  }
}

constexpr uint32_t kFromRight = 0x80000000u;

// The merge-path split of every tile boundary, one thread per boundary (all
// binary searches in flight together rather than one dependent search at the
// start of each tile).
template <class T, int LESS, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    merge_splits_kernel(Src L, Src R, uint64_t tiles, uint64_t* __restrict__ splits) {
  const uint64_t nl = src_len(L), nr = src_len(R), n = nl + nr;
  for (uint64_t b = blockIdx.x * (uint64_t)kThreads + threadIdx.x; b <= tiles;
       b += (uint64_t)gridDim.x * kThreads)
    splits[b] = merge_path<T, LESS, PLAIN>(L, R, nl, nr, min(b * (uint64_t)kTile, n));
}

template <class T, int LESS, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    merge_kernel(Src L, Src R, void* out, int out_dtype, Payload pay,
                 uint32_t* count_dev, const uint64_t* __restrict__ splits) {
  __shared__ T s_keys[kTile];
  __shared__ T s_out[kTile];
  __shared__ uint32_t s_src[kTile];
  __shared__ uint64_t s_split[2];
  const uint64_t nl = src_len(L), nr = src_len(R), n = nl + nr;
  if (blockIdx.x == 0 && threadIdx.x == 0 && count_dev) *count_dev = (uint32_t)n;
  const uint64_t d0 = (uint64_t)blockIdx.x * kTile;
  if (d0 >= n) return;
  const uint64_t d1 = min(d0 + (uint64_t)kTile, n);
  if (threadIdx.x < 2) s_split[threadIdx.x] = splits[blockIdx.x + threadIdx.x];
  __syncthreads();
  const uint64_t i0 = s_split[0], i1 = s_split[1];
  const uint64_t j0 = d0 - i0, j1 = d1 - i1;
  const int la = (int)(i1 - i0), lb = (int)(j1 - j0);
  for (int t = threadIdx.x; t < la; t += kThreads) s_keys[t] = merge_load<T, PLAIN>(L, i0 + t);
  for (int t = threadIdx.x; t < lb; t += kThreads) s_keys[la + t] = merge_load<T, PLAIN>(R, j0 + t);
  __syncthreads();
  const int total = la + lb;
  const int dt = min((int)threadIdx.x * kItems, total);
  // Per-thread split inside the tile.
  int lo = dt > lb ? dt - lb : 0, hi = dt < la ? dt : la;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (!cmp_ct<T, LESS>(s_keys[la + dt - 1 - mid], s_keys[mid])) lo = mid + 1;
    else hi = mid;
  }
  // Serial merge with the two heads in registers: one shared-memory read per
  // output.
  int a = lo, b = dt - lo;
  T ka = a < la ? s_keys[a] : T(0);
  T kb = b < lb ? s_keys[la + b] : T(0);
  const bool pay_on = pay.ncols != 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    if (dt + k >= total) break;
    const bool take_left = b >= lb || (a < la && !cmp_ct<T, LESS>(kb, ka));
    s_out[dt + k] = take_left ? ka : kb;
    if (pay_on) s_src[dt + k] = take_left ? (uint32_t)a : (kFromRight | (uint32_t)b);
    if (take_left) {
      ++a;
      ka = a < la ? s_keys[a] : ka;
    } else {
      ++b;
      kb = b < lb ? s_keys[la + b] : kb;
    }
  }
  __syncthreads();
  const bool same_type = out_dtype == DTypeOf<T>::value;
  for (int t = threadIdx.x; t < total; t += kThreads) {
    if (out) {
      if (same_type) __stcs((T*)out + d0 + t, s_out[t]);
      else st_cast<T>(out_dtype, out, d0 + t, s_out[t]);
    }
    if (pay.ncols) {
      const uint32_t s = s_src[t];
      const bool right = s & kFromRight;
      const uint64_t idx = right ? j0 + (s & ~kFromRight) : i0 + s;
      for (int c = 0; c < pay.ncols; ++c) {
        const uint64_t bits = src_load_bits(right ? pay.right[c] : pay.left[c], idx);
        st_raw_pay(pay.out[c], d0 + t, pay.esize[c], bits);
      }
    }
  }
}

// Occurrence-rank flags of `own` against `other` (set.rs:18-46 rules).
// mode 1 (keep if rank < count in other): intersection;
// mode 2 (keep if rank >= count in other): difference and union extras.
template <class T>
__global__ void __launch_bounds__(kThreads)
    set_flags_kernel(Src own, Src other, int less, int mode, uint32_t* flags) {
  const uint64_t n = src_len(own), m = src_len(other);
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * kThreads) {
    const T v = src_load<T>(own, i);
    // first position in own whose element is not less than v
    uint64_t lo = 0, hi = i;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (cmp_less<T>(less, src_load<T>(own, mid), v)) lo = mid + 1;
      else hi = mid;
    }
    const uint64_t rank = i - lo;
    uint64_t a = 0, b = m;
    while (a < b) {
      const uint64_t mid = (a + b) >> 1;
      if (cmp_less<T>(less, src_load<T>(other, mid), v)) a = mid + 1;
      else b = mid;
    }
    uint64_t c = a, e = m;
    while (c < e) {
      const uint64_t mid = (c + e) >> 1;
      if (!cmp_less<T>(less, v, src_load<T>(other, mid))) c = mid + 1;
      else e = mid;
    }
    const uint64_t cnt = c - a;
    flags[i] = mode == 1 ? (rank < cnt) : (rank >= cnt);
  }
}

__global__ void add_counts_kernel(const uint32_t* a, uint64_t b, uint32_t* out) {
  *out = *a + (uint32_t)b;
}

unsigned grid_n(uint64_t n) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 16));
}

template <class T, int LESS, bool PLAIN>
int merge_launch(mb_executor* ex, const mb_src& l, const mb_src& r, void* out, int out_dtype,
                 const Payload& pay, uint32_t* count_dev) {
  const uint64_t cap = l.len + r.len;
  const uint64_t tiles = std::max<uint64_t>(1, (cap + kTile - 1) / kTile);
  Scratch splits;
  MB_TRY(splits.alloc(ex, (tiles + 1) * sizeof(uint64_t)));
  const uint64_t sblocks = std::min<uint64_t>((tiles + kThreads) / kThreads, 4096);
  merge_splits_kernel<T, LESS, PLAIN><<<(unsigned)sblocks, kThreads, 0, ex->stream>>>(
      to_src(l), to_src(r), tiles, splits.as<uint64_t>());
  MB_CUDA(cudaGetLastError());
  merge_kernel<T, LESS, PLAIN><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
      to_src(l), to_src(r), out, out_dtype, pay, count_dev, splits.as<uint64_t>());
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T, int LESS>
int merge_less(mb_executor* ex, const mb_src& l, const mb_src& r, void* out, int out_dtype,
               const Payload& pay, uint32_t* count_dev) {
  const int ct = DTypeOf<T>::value;
  if (src_plain(l, ct) && src_plain(r, ct))
    return merge_launch<T, LESS, true>(ex, l, r, out, out_dtype, pay, count_dev);
  return merge_launch<T, LESS, false>(ex, l, r, out, out_dtype, pay, count_dev);
}

template <class T>
int merge_run(mb_executor* ex, const mb_src& l, const mb_src& r, int less, void* out,
              int out_dtype, const Payload& pay, uint32_t* count_dev) {
  switch (less) {
    case MB_GREATER: return merge_less<T, MB_GREATER>(ex, l, r, out, out_dtype, pay, count_dev);
    case MB_TOTAL_LESS:
      return merge_less<T, MB_TOTAL_LESS>(ex, l, r, out, out_dtype, pay, count_dev);
    default: return merge_less<T, MB_LESS>(ex, l, r, out, out_dtype, pay, count_dev);
  }
}

template <class T>
int set_flags_run(mb_executor* ex, const mb_src& own, const mb_src& other, int less, int mode,
                  uint32_t* flags) {
  if (own.len == 0) return MB_OK;
  set_flags_kernel<T><<<grid_n(own.len), kThreads, 0, ex->stream>>>(to_src(own), to_src(other),
                                                                    less, mode, flags);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int merge_dispatch(mb_executor* ex, const mb_src& l, const mb_src& r, int less, void* out,
                   int out_dtype, const Payload& pay, uint32_t* count_dev) {
  const int ct = compute_type(l.vtype);
  MB_DISPATCH_CTYPE(ct, merge_run, ex, l, r, less, out, out_dtype, pay, count_dev);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int flags_dispatch(mb_executor* ex, const mb_src& own, const mb_src& other, int less, int mode,
                   uint32_t* flags) {
  const int ct = compute_type(own.vtype);
  MB_DISPATCH_CTYPE(ct, set_flags_run, ex, own, other, less, mode, flags);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int check_pair(mb_executor* ex, const mb_src* l, const mb_src* r, int less) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, l, "left"));
  MB_TRY(check_src(ex, r, "right"));
  if (compute_type(l->vtype) != compute_type(r->vtype))
    return set_error(MB_ERR_LAUNCH, "left and right element types differ");
  if (less < MB_LESS || less > MB_TOTAL_LESS)
    return set_error(MB_ERR_LAUNCH, "takes LESS, GREATER or TOTAL_LESS");
  return MB_OK;
}

// Set operation: mode 1 intersection, 2 difference, 0 union.
int set_op(mb_executor* ex, const mb_src* l, const mb_src* r, int less, mb_col out,
           uint32_t* count_dev, uint32_t* count_host, int mode) {
  MB_TRY(check_pair(ex, l, r, less));
  MB_TRY(check_col(ex, out, "output"));
  const uint64_t need = mode == 0 ? l->len + r->len : l->len;
  if (out.len < need) return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", need, out.len);
  if (dtype_size(out.dtype) != dtype_size(l->vtype))
    return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  Scratch cnt;
  if (!count_dev) {
    MB_TRY(cnt.alloc(ex, 16));
    count_dev = cnt.as<uint32_t>();
  }
  const mb_src& own = mode == 0 ? *r : *l;
  const mb_src& other = mode == 0 ? *l : *r;
  Scratch flags;
  MB_TRY(flags.alloc(ex, std::max<uint64_t>(16, own.len * 4)));
  MB_TRY(flags_dispatch(ex, own, other, less, mode == 1 ? 1 : 2, flags.as<uint32_t>()));
  mb_src st{};
  st.kind = MB_SRC_COLUMN;
  st.dtype = st.vtype = MB_U32;
  st.map = MB_UN_IDENTITY;
  st.data = flags.ptr;
  st.len = own.len;
  if (mode != 0) {
    MB_TRY(mb_copy_where(ex, l, 1, &st, &out, count_dev, nullptr));
  } else {
    // Union: merge left with the right input's extra copies.
    Scratch extras, ecount;
    MB_TRY(extras.alloc(ex, std::max<uint64_t>(16, r->len * dtype_size(r->vtype))));
    MB_TRY(ecount.alloc(ex, 16));
    mb_col ec{};
    ec.data = extras.ptr;
    ec.dtype = r->vtype;
    ec.len = r->len;
    MB_TRY(mb_copy_where(ex, r, 1, &st, &ec, ecount.as<uint32_t>(), nullptr));
    mb_src es{};
    es.kind = MB_SRC_COLUMN;
    es.dtype = es.vtype = r->vtype;
    es.map = MB_UN_IDENTITY;
    es.data = extras.ptr;
    es.len = r->len;
    es.len_dev = ecount.as<uint32_t>();
    Payload none{};
    MB_TRY(merge_dispatch(ex, *l, es, less, out.data, out.dtype, none, nullptr));
    add_counts_kernel<<<1, 1, 0, ex->stream>>>(ecount.as<uint32_t>(), l->len, count_dev);
    MB_CUDA(cudaGetLastError());
  }
  if (count_host) MB_TRY(read_u32(ex, count_dev, count_host));
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_merge(mb_executor* ex, const mb_src* left, const mb_src* right, int less, mb_col out) {
  MB_TRY(check_pair(ex, left, right, less));
  MB_TRY(check_col(ex, out, "output"));
  const uint64_t n = left->len + right->len;
  MB_TRY(check_len_u32(n));
  if (out.len < n) return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out.len);
  if (compute_type(out.dtype) != compute_type(left->vtype))
    return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  if (n == 0) return MB_OK;
  Payload none{};
  return merge_dispatch(ex, *left, *right, less, out.data, out.dtype, none, nullptr);
}

int mb_merge_by_key(mb_executor* ex, const mb_src* left_keys, const mb_src* left_values,
                    const mb_src* right_keys, const mb_src* right_values, int nvals, int less,
                    mb_col out_keys, const mb_col* out_values) {
  MB_TRY(check_pair(ex, left_keys, right_keys, less));
  if (nvals < 0 || nvals > kMaxPay) return set_error(MB_ERR_LAUNCH, "values take 0 to 12 columns");
  const uint64_t n = left_keys->len + right_keys->len;
  MB_TRY(check_len_u32(n));
  Payload pay{};
  pay.ncols = nvals;
  for (int c = 0; c < nvals; ++c) {
    MB_TRY(check_src(ex, &left_values[c], "left values"));
    MB_TRY(check_src(ex, &right_values[c], "right values"));
    MB_TRY(check_col(ex, out_values[c], "value output"));
    if (left_values[c].len != left_keys->len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", left_keys->len, left_values[c].len);
    if (right_values[c].len != right_keys->len)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", right_keys->len, right_values[c].len);
    if (out_values[c].len < n)
      return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out_values[c].len);
    pay.left[c] = to_src(left_values[c]);
    pay.right[c] = to_src(right_values[c]);
    pay.out[c] = out_values[c].data;
    pay.esize[c] = (int)dtype_size(left_values[c].vtype);
  }
  if (out_keys.data) {
    MB_TRY(check_col(ex, out_keys, "key output"));
    if (out_keys.len < n) return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out_keys.len);
  }
  if (n == 0) return MB_OK;
  return merge_dispatch(ex, *left_keys, *right_keys, less, out_keys.data, out_keys.dtype, pay,
                        nullptr);
}

int mb_set_union(mb_executor* ex, const mb_src* left, const mb_src* right, int less, mb_col out,
                 uint32_t* count_dev, uint32_t* count_host) {
  return set_op(ex, left, right, less, out, count_dev, count_host, 0);
}

int mb_set_intersection(mb_executor* ex, const mb_src* left, const mb_src* right, int less,
                        mb_col out, uint32_t* count_dev, uint32_t* count_host) {
  return set_op(ex, left, right, less, out, count_dev, count_host, 1);
}

int mb_set_difference(mb_executor* ex, const mb_src* left, const mb_src* right, int less,
                      mb_col out, uint32_t* count_dev, uint32_t* count_host) {
  return set_op(ex, left, right, less, out, count_dev, count_host, 2);
}

}  // extern "C"
