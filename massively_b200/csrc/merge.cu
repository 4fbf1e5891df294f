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
#include "lookback.cuh"

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

// ------------------------------------------------------ set operations --
//
// One pass over the stable merge M of the two inputs (ties: left first).
// Equivalent items (neither less than the other) form one run of M: its
// left copies, then its right copies.  With rs / re the run's first and
// one-past-last merged positions and lr the position of its first right
// copy (cl = lr - rs left copies, cr = re - lr right copies), massively's
// multiset rule (core/set.rs:18-46; the two-pointer walk of its oracle,
// verification/oracle/src/vector.rs:595-664) keeps, for the item at p:
//   intersection: a left copy with p - rs <  cr;
//   difference:   a left copy with p - rs >= cr;
//   union:        every left copy, and a right copy with p - lr >= cl.
// A tile of M (its merge-path split) merges its two slices in shared
// memory, finds every position's run with block-wide scans of the run heads
// and of the left / right positions, and takes the runs that cross its
// edges from the run of each boundary's item (four binary searches per
// boundary, for all boundaries at once before the tile kernel).  It counts
// the kept items, gets the count of all earlier tiles by a decoupled
// look-back, and writes the kept items in order; the total stays on the
// device.  The inputs must be sorted under a strict weak order (no NaN
// under LESS / GREATER; TOTAL_LESS orders every float).

struct SetRun {
  uint32_t lbl, ubl, lbr, ubr;  // the run's bounds in the left and in the right input
};

template <class T, int LESS>
__device__ __forceinline__ bool equiv_ct(T a, T b) {
  return !cmp_ct<T, LESS>(a, b) && !cmp_ct<T, LESS>(b, a);
}

// First index in [0, n) whose item is not less than v (UPPER: that v is
// less than).
template <class T, int LESS, bool PLAIN, bool UPPER>
__device__ uint64_t bound_of(const Src& s, uint64_t n, T v) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    const T x = merge_load<T, PLAIN>(s, mid);
    const bool before = UPPER ? !cmp_ct<T, LESS>(v, x) : cmp_ct<T, LESS>(x, v);
    if (before) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Per tile boundary b: the merge-path split, the item at merged position
// b * kTile and the bounds of its run in both inputs.
template <class T, int LESS, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    set_bounds_kernel(Src L, Src R, uint64_t tiles, uint64_t* __restrict__ splits,
                      SetRun* __restrict__ runs, T* __restrict__ vals) {
  const uint64_t nl = src_len(L), nr = src_len(R), n = nl + nr;
  for (uint64_t b = blockIdx.x * (uint64_t)kThreads + threadIdx.x; b <= tiles;
       b += (uint64_t)gridDim.x * kThreads) {
    const uint64_t d = min(b * (uint64_t)kTile, n);
    const uint64_t i = merge_path<T, LESS, PLAIN>(L, R, nl, nr, d);
    splits[b] = i;
    if (d >= n) continue;
    const uint64_t j = d - i;
    const bool from_left =
        i < nl && (j >= nr || !cmp_ct<T, LESS>(merge_load<T, PLAIN>(R, j),
                                               merge_load<T, PLAIN>(L, i)));
    const T v = from_left ? merge_load<T, PLAIN>(L, i) : merge_load<T, PLAIN>(R, j);
    vals[b] = v;
    SetRun r;
    r.lbl = (uint32_t)bound_of<T, LESS, PLAIN, false>(L, nl, v);
    r.ubl = (uint32_t)bound_of<T, LESS, PLAIN, true>(L, nl, v);
    r.lbr = (uint32_t)bound_of<T, LESS, PLAIN, false>(R, nr, v);
    r.ubr = (uint32_t)bound_of<T, LESS, PLAIN, true>(R, nr, v);
    runs[b] = r;
  }
}

constexpr int kNone = 0x7FFFFFFF;

// Exclusive block-wide scans over the threads' chunk summaries: a running
// maximum of (a, b) from the left, and a running minimum of (c, d) from the
// right (each thread gets the extremes of the chunks before / after it).
__device__ __forceinline__ void set_block_scans(int& a, int& b, int& c, int& d, int* s_tmp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int W = kThreads / 32;
  int ia = a, ib = b, ic = c, id = d;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int oa = __shfl_up_sync(kFull, ia, off), ob = __shfl_up_sync(kFull, ib, off);
    const int oc = __shfl_down_sync(kFull, ic, off), od = __shfl_down_sync(kFull, id, off);
    if (lane >= off) { ia = max(ia, oa); ib = max(ib, ob); }
    if (lane + off < 32) { ic = min(ic, oc); id = min(id, od); }
  }
  if (lane == 31) { s_tmp[warp] = ia; s_tmp[W + warp] = ib; }
  if (lane == 0) { s_tmp[2 * W + warp] = ic; s_tmp[3 * W + warp] = id; }
  __syncthreads();
  int ca = -1, cb = -1, cc = kNone, cd = kNone;
  for (int w = 0; w < warp; ++w) { ca = max(ca, s_tmp[w]); cb = max(cb, s_tmp[W + w]); }
  for (int w = warp + 1; w < W; ++w) { cc = min(cc, s_tmp[2 * W + w]); cd = min(cd, s_tmp[3 * W + w]); }
  const int pa = __shfl_up_sync(kFull, ia, 1), pb = __shfl_up_sync(kFull, ib, 1);
  const int pc = __shfl_down_sync(kFull, ic, 1), pd = __shfl_down_sync(kFull, id, 1);
  a = lane > 0 ? max(ca, pa) : ca;
  b = lane > 0 ? max(cb, pb) : cb;
  c = lane < 31 ? min(cc, pc) : cc;
  d = lane < 31 ? min(cd, pd) : cd;
}

// MODE: 0 union, 1 intersection, 2 difference.
template <class T, int LESS, bool PLAIN>
__global__ void __launch_bounds__(kThreads, 4)
    set_tile_kernel(int MODE, Src L, Src R, void* out, int out_esize, uint32_t* count_dev,
                    const uint64_t* __restrict__ splits, const SetRun* __restrict__ runs,
                    const T* __restrict__ vals, uint32_t* counter, TileState<uint32_t, true> st,
                    DevErr err) {
  __shared__ T s_keys[kTile];
  __shared__ T s_out[kTile];
  __shared__ uint8_t s_right[kTile];
  __shared__ int s_tmp[4 * (kThreads / 32)];
  __shared__ uint32_t s_wcount[kThreads / 32];
  __shared__ uint32_t s_tile, s_excl, s_tile_kept;
  __shared__ uint64_t s_split[2];
  const uint64_t nl = src_len(L), nr = src_len(R), n = nl + nr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(counter, 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t d0 = tile * (uint64_t)kTile;
  if (d0 >= n) return;
  const uint64_t d1 = min(d0 + (uint64_t)kTile, n);
  if (tid < 2) s_split[tid] = splits[tile + tid];
  __syncthreads();
  const uint64_t i0 = s_split[0], i1 = s_split[1];
  const uint64_t j0 = d0 - i0, j1 = d1 - i1;
  const int la = (int)(i1 - i0), lb = (int)(j1 - j0);
  for (int t = tid; t < la; t += kThreads) s_keys[t] = merge_load<T, PLAIN>(L, i0 + t);
  for (int t = tid; t < lb; t += kThreads) s_keys[la + t] = merge_load<T, PLAIN>(R, j0 + t);
  __syncthreads();
  const int total = la + lb;
  const int dt = min(tid * kItems, total);
  {
    int lo = dt > lb ? dt - lb : 0, hi = dt < la ? dt : la;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (!cmp_ct<T, LESS>(s_keys[la + dt - 1 - mid], s_keys[mid])) lo = mid + 1;
      else hi = mid;
    }
    int a = lo, b = dt - lo;
    T ka = a < la ? s_keys[a] : T(0);
    T kb = b < lb ? s_keys[la + b] : T(0);
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      if (dt + k >= total) break;
      const bool take_left = b >= lb || (a < la && !cmp_ct<T, LESS>(kb, ka));
      s_out[dt + k] = take_left ? ka : kb;
      s_right[dt + k] = take_left ? 0 : 1;
      if (take_left) {
        ++a;
        ka = a < la ? s_keys[a] : ka;
      } else {
        ++b;
        kb = b < lb ? s_keys[la + b] : kb;
      }
    }
  }
  __syncthreads();

  // Chunk summaries: last head, last left position (forward); first head,
  // first right position (backward).  Position 0 is a head of the tile.
  const int cnt = min(kItems, total - dt);
  bool head[kItems], right[kItems];
  int lastH = -1, lastL = -1, firstH = kNone, firstR = kNone;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int t = dt + k;
    head[k] = false;
    right[k] = false;
    if (k < cnt) {
      head[k] = t == 0 || !equiv_ct<T, LESS>(s_out[t - 1], s_out[t]);
      right[k] = s_right[t] != 0;
      if (head[k]) { lastH = t; if (firstH == kNone) firstH = t; }
      if (right[k]) { if (firstR == kNone) firstR = t; } else { lastL = t; }
    }
  }
  int eh = lastH, el = lastL, fh = firstH, fr = firstR;
  set_block_scans(eh, el, fh, fr, s_tmp);
  // rs / last left (at or before t) forward; re (head after t) / first right
  // (at or after t) backward -- tile positions.
  int rs[kItems], ll[kItems], re[kItems], rr[kItems];
  {
    int h = eh, l = el;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      if (k < cnt) {
        if (head[k]) h = dt + k;
        if (!right[k]) l = dt + k;
      }
      rs[k] = h;
      ll[k] = l;
    }
    int nh = fh, nrp = fr;
#pragma unroll
    for (int k = kItems - 1; k >= 0; --k) {
      re[k] = nh;
      if (k < cnt) {
        if (right[k]) nrp = dt + k;
        if (head[k]) nh = dt + k;
      }
      rr[k] = nrp;
    }
  }
  // Runs that cross the tile's edges: the first (when it started before
  // d0) from boundary `tile`, the last (when it goes on past d1) from
  // boundary `tile + 1`.
  const SetRun r0 = runs[tile];
  const uint64_t rs0 = (uint64_t)r0.lbl + r0.lbr;
  const bool first_open = rs0 < d0;
  bool last_open = false;
  SetRun r1{};
  if (d1 < n) {
    r1 = runs[tile + 1];
    last_open = equiv_ct<T, LESS>(s_out[total - 1], vals[tile + 1]);
  }
  // Tile position of the last run's head (every thread reads the same).
  __shared__ int s_last_rs;
  if (tid == 0) s_last_rs = -1;
  __syncthreads();
  if (cnt > 0 && dt + cnt == total) s_last_rs = rs[cnt - 1];
  __syncthreads();
  const int last_rs = s_last_rs;

  bool keep[kItems];
  uint32_t kept = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    keep[k] = false;
    if (k >= cnt) continue;
    const bool use0 = first_open && rs[k] == 0;
    const bool use1 = !use0 && last_open && rs[k] == last_rs;
    bool kp;
    if (use0 || use1) {  // a run crossing the tile's edge: global positions
      const SetRun x = use0 ? r0 : r1;
      const uint64_t g = d0 + dt + k;
      const uint64_t grs = (uint64_t)x.lbl + x.lbr;
      const uint64_t cl = x.ubl - x.lbl, cr = x.ubr - x.lbr;
      if (!right[k]) {
        const uint64_t rank = g - grs;
        kp = MODE == 0 || (MODE == 1 ? rank < cr : rank >= cr);
      } else {
        kp = MODE == 0 && g - (grs + cl) >= cl;
      }
    } else {  // a run inside the tile: tile positions
      const int t = dt + k;
      const int e = re[k] == kNone ? total : re[k];
      if (!right[k]) {
        const int lr = min(rr[k] == kNone ? total : rr[k], e);
        const int rank = t - rs[k], cr = e - lr;
        kp = MODE == 0 || (MODE == 1 ? rank < cr : rank >= cr);
      } else {
        const int lr = max(ll[k] + 1, rs[k]);
        kp = MODE == 0 && t - lr >= lr - rs[k];
      }
    }
    keep[k] = kp;
    kept += kp ? 1u : 0u;
  }

  // Output offsets: warp and block prefix of the kept counts, then the
  // counts of all earlier tiles by the look-back.
  uint32_t incl = kept;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t o = __shfl_up_sync(kFull, incl, off);
    if (lane >= off) incl += o;
  }
  if (lane == 31) s_wcount[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t c = lane < kThreads / 32 ? s_wcount[lane] : 0u;
    const uint32_t agg = __reduce_add_sync(kFull, c);
    const Op<uint32_t, MB_OP_ADD> add{MB_OP_ADD};
    uint32_t excl = 0;
    if (tile == 0) {
      if (lane == 0) st.publish(0, kFlagIncl, agg);
    } else {
      if (lane == 0) st.publish(tile, kFlagAgg, agg);
      excl = lookback_exclusive<uint32_t, Op<uint32_t, MB_OP_ADD>, false>(st, tile, add, err, 0u);
      if (lane == 0) st.publish(tile, kFlagIncl, excl + agg);
    }
    if (lane == 0) {
      s_excl = excl;
      s_tile_kept = agg;
      if (d1 == n && count_dev) *count_dev = excl + agg;
    }
  }
  // The kept items, compacted in tile order into s_keys (free since the
  // merge), then written with consecutive threads on consecutive addresses.
  uint32_t lpos = incl - kept;
  for (int w = 0; w < warp; ++w) lpos += s_wcount[w];
#pragma unroll
  for (int k = 0; k < kItems; ++k)
    if (keep[k]) s_keys[lpos++] = s_out[dt + k];
  __syncthreads();
  const uint64_t base = s_excl;
  const uint32_t tile_kept = s_tile_kept;
  const uint64_t cap = MODE == 0 ? n : nl;
  for (uint32_t i = tid; i < tile_kept; i += kThreads) {
    if (base + i < cap) st_raw_pay(out, base + i, out_esize, to_bits64(s_keys[i]));
    else raise_device_error(err, MB_DEV_ERR_BOUNDS);  // only after a failed look-back
  }
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

// Set operation over n = |l| + |r| > 0 merged items (mode 0 union, 1
// intersection, 2 difference); the kept count goes to count_dev.
template <class T, int LESS, bool PLAIN>
int set_launch(mb_executor* ex, const mb_src& l, const mb_src& r, int mode, const mb_col& out,
               uint32_t* count_dev) {
  const uint64_t n = l.len + r.len;
  const uint64_t tiles = (n + kTile - 1) / kTile;
  const size_t state_b = TileState<uint32_t, true>::bytes(tiles);
  const size_t splits_b = ((tiles + 1) * 8 + 255) / 256 * 256;
  const size_t runs_b = ((tiles + 1) * sizeof(SetRun) + 255) / 256 * 256;
  const size_t vals_b = ((tiles + 1) * sizeof(T) + 255) / 256 * 256;
  Scratch scratch;
  MB_TRY(scratch.alloc(ex, 256 + state_b + splits_b + runs_b + vals_b));
  char* base = scratch.as<char>();
  MB_CUDA(cudaMemsetAsync(base, 0, 256 + state_b, ex->stream));
  uint64_t* splits = (uint64_t*)(base + 256 + state_b);
  SetRun* runs = (SetRun*)(base + 256 + state_b + splits_b);
  T* vals = (T*)(base + 256 + state_b + splits_b + runs_b);
  const uint64_t sblocks = std::min<uint64_t>((tiles + kThreads) / kThreads, 4096);
  set_bounds_kernel<T, LESS, PLAIN><<<(unsigned)sblocks, kThreads, 0, ex->stream>>>(
      to_src(l), to_src(r), tiles, splits, runs, vals);
  MB_CUDA(cudaGetLastError());
  const DevErr err{ex->status_dev, (uint32_t*)base + 1};
  set_tile_kernel<T, LESS, PLAIN><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
      mode, to_src(l), to_src(r), out.data, (int)dtype_size(out.dtype), count_dev, splits, runs,
      vals,
      (uint32_t*)base, TileState<uint32_t, true>::make(base + 256, tiles), err);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T>
int set_run(mb_executor* ex, const mb_src& l, const mb_src& r, int less, int mode,
            const mb_col& out, uint32_t* count_dev) {
  const int ct = DTypeOf<T>::value;
  const bool plain = src_plain(l, ct) && src_plain(r, ct);
#define MB_SET_LESS(LESSID)                                                              \
  return plain ? set_launch<T, LESSID, true>(ex, l, r, mode, out, count_dev)             \
               : set_launch<T, LESSID, false>(ex, l, r, mode, out, count_dev)
  switch (less) {
    case MB_GREATER: MB_SET_LESS(MB_GREATER);
    case MB_TOTAL_LESS: MB_SET_LESS(MB_TOTAL_LESS);
    default: MB_SET_LESS(MB_LESS);
  }
#undef MB_SET_LESS
}

int merge_dispatch(mb_executor* ex, const mb_src& l, const mb_src& r, int less, void* out,
                   int out_dtype, const Payload& pay, uint32_t* count_dev) {
  const int ct = compute_type(l.vtype);
  MB_DISPATCH_CTYPE(ct, merge_run, ex, l, r, less, out, out_dtype, pay, count_dev);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

int set_dispatch(mb_executor* ex, const mb_src& l, const mb_src& r, int less, int mode,
                 const mb_col& out, uint32_t* count_dev) {
  const int ct = compute_type(l.vtype);
  MB_DISPATCH_CTYPE(ct, set_run, ex, l, r, less, mode, out, count_dev);
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
  MB_TRY(check_len_u32(l->len + r->len));
  Scratch cnt;
  if (!count_dev) {
    MB_TRY(cnt.alloc(ex, 16));
    count_dev = cnt.as<uint32_t>();
  }
  // Zero first: inputs whose device lengths are both 0 launch no tile that
  // writes the count.
  MB_CUDA(cudaMemsetAsync(count_dev, 0, 4, ex->stream));
  if (l->len + r->len > 0) MB_TRY(set_dispatch(ex, *l, *r, less, mode, out, count_dev));
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
