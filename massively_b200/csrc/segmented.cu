// segmented.cu -- single-pass segmented scan / reduce over a Segmentation,
// and the by-key algorithms (inclusive / exclusive scan_by_key,
// reduce_by_key), plus Segmentation construction kernels.
//
// Replaces massively's head-flag pipeline (massively/src/seg/control.rs:
// 223-285 heads fill + mark; massively/src/core/segmented_fixed.rs:22-707
// block segmented scan, recursive segmented prefix, exclusive fix-up and the
// per-segment tail pick; massively/src/seg/mod.rs:712-785 fill-with-init,
// selection scan and scatter of the per-head results; massively/src/core/
// by_key.rs:79-121 for reduce_by_key) with one kernel per call.
//
// Each tile marks its segment heads in a shared-memory bitmap -- from the
// offsets (the tile's first segment comes from a per-tile lower bound that a
// small kernel computes for all tiles in parallel, then one read per segment
// start) or, for the by-key algorithms, from adjacent key inequality -- and
// scans (head count, value) pairs under the segmented
// operator  (ha, a) . (hb, b) = (ha + hb, hb ? b : a op b),  which is
// associative, so the decoupled look-back of lookback.cuh carries segment
// boundaries across tiles.  Reductions stage the tile's inclusive pairs in
// shared memory and write one value per segment tail: init op inclusive
// (massively's init op v_head ... op v_tail); empty segments get init
// (massively/src/seg/mod.rs:728-729); run indices of reduce_by_key are the
// inclusive head counts, and the run count stays on the device.

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

namespace mb {

int materialize(mb_executor* ex, const mb_src& in, void* dst);

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kLoads = 4;
// Blocks per SM the segmented kernel is compiled for: at the compiler's
// natural 123 registers only two fit, and warps sit at the barrier while
// warp 0 looks back.
constexpr int kSegMinBlocks = 4;

// kReduceTiles: ForEachSegment(Reduce) over offsets without the cross-tile
// look-back -- each tile reduces the segments that start and end in it and
// leaves two partial folds for the segments that cross its edges, which
// seg_reduce_cross_kernel then folds in tile order.
// kScanInclTiles / kScanExclTiles: the segmented scans over offsets without
// the look-back -- every tile scans as if it started a segment and leaves
// its tail fold; seg_tile_carry_kernel scans those folds over the tiles
// (a segmented scan of one value per tile), and seg_scan_fix_kernel applies
// each tile's carry to the items before its first segment start.
// kReduceKeysTiles: reduce_by_key the same way -- a first pass counts every
// tile's run heads (seg_run_heads_kernel) and scans the counts into each
// tile's first run index (seg_run_base_kernel); each tile then reduces the
// runs that start and end in it and leaves its folds for the runs that cross
// its edges (seg_rbk_walk_kernel).  The run bases are computed once per call
// and shared by every value column of the same tile size.
enum SegMode : int {
  kScanIncl = 0,
  kScanExcl = 1,
  kReduce = 2,
  kReduceTiles = 3,
  kScanInclTiles = 4,
  kScanExclTiles = 5,
  kReduceKeysTiles = 6
};
enum HeadsSrc : int { kHeadsOffsets = 0, kHeadsKeys = 1 };

template <class V>
struct SegVal {
  uint32_t heads;
  V v;
};

}  // namespace

// A (head count, 4-byte value) pair packs into one status word with its flag:
// flag in bits 62-63, head count (below 2^30: at most one head per item) in
// bits 32-61, value bits in 0-31 -- one load per predecessor in the look-back.
template <class V>
struct StatePack<SegVal<V>> {
  static constexpr bool kPackable = sizeof(V) == 4;
  __device__ __forceinline__ static uint64_t pack(uint32_t flag, const SegVal<V>& x) {
    return ((uint64_t)flag << 62) | ((uint64_t)(x.heads & 0x3FFFFFFFu) << 32) | to_bits64(x.v);
  }
  __device__ __forceinline__ static uint32_t unpack(uint64_t w, SegVal<V>& x) {
    x.heads = (uint32_t)(w >> 32) & 0x3FFFFFFFu;
    x.v = from_bits64<V>(w & 0xFFFFFFFFull);
    return (uint32_t)(w >> 62);
  }
};

namespace {

template <class V, int OP>
struct SegOp {
  Op<V, OP> op;
  __device__ __forceinline__ SegVal<V> operator()(const SegVal<V>& a, const SegVal<V>& b) const {
    SegVal<V> r;
    r.heads = a.heads + b.heads;
    r.v = b.heads ? b.v : op(a.v, b.v);
    return r;
  }
};

template <class V>
struct SegCfg {
  static constexpr int VEC = 16 / sizeof(V);
  static constexpr int ITEMS = VEC * kLoads;
  static constexpr int WARP_ITEMS = 32 * ITEMS;
  static constexpr int TILE = kThreads * ITEMS;
};

template <class V>
struct SegParams {
  int op;
  int mode;
  int heads_src;
  int out_dtype;
  V init;
  const uint32_t* offsets;  // nseg + 1 entries
  uint64_t nseg;
  const uint32_t* tile_lb;  // per tile t: first segment starting at or after t * TILE
  Src keys;
  void* out;
  void* out_keys;
  int out_key_esize;
  uint32_t* count_dev;
  uint32_t* counter;
  DevErr err;
  // kReduceTiles: per tile, the fold before its first segment start
  // (part_head), the fold from its last segment start to its end
  // (part_tail), and the segment that starts at that last start when it goes
  // on past the tile (tail_seg, ~0u otherwise).
  V* part_head;
  V* part_tail;
  uint32_t* tail_seg;
  // kReduceKeysTiles: each tile's first run index (the heads before it) and
  // the position of its first head (the tile's length when it has none).
  const uint32_t* run_base;
  uint32_t* first_pos;
  // kReduceKeysTiles: every tile's run-head bitmap (TILE / 32 words per
  // tile), written by seg_run_heads_kernel, so the value passes need not
  // read the keys again.
  const uint32_t* head_bits;
};

__device__ __forceinline__ bool key_eq(int dtype, uint64_t a, uint64_t b) {
  if (dtype == MB_F32) return __uint_as_float((uint32_t)a) == __uint_as_float((uint32_t)b);
  if (dtype == MB_F64) return __longlong_as_double((long long)a) == __longlong_as_double((long long)b);
  return a == b;
}

// First index in [0, count) with offsets[idx] >= x (count if none).
__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* a, uint64_t count, uint64_t x) {
  uint64_t lo = 0, hi = count;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
// First index in [0, count) with offsets[idx] > x.
__device__ __forceinline__ uint64_t upper_bound_u32(const uint32_t* a, uint64_t count, uint64_t x) {
  uint64_t lo = 0, hi = count;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)a[mid] <= x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// tile_lb[t] = first s in [0, nseg] with offsets[s] >= t * tile, for every
// tile t in [0, tiles]: one thread per offset s fills the tiles whose first
// position lies in (offsets[s-1], offsets[s]] -- O(segments + tiles) work in
// parallel, instead of a dependent binary search per tile.
__global__ void __launch_bounds__(kThreads)
    seg_tile_bounds_kernel(const uint32_t* __restrict__ offsets, uint64_t nseg, uint64_t tile,
                           uint64_t tiles, uint32_t* __restrict__ tile_lb) {
  for (uint64_t s = blockIdx.x * (uint64_t)kThreads + threadIdx.x; s <= nseg;
       s += (uint64_t)gridDim.x * kThreads) {
    const uint64_t lo = s == 0 ? 0 : (uint64_t)offsets[s - 1] / tile + 1;
    const uint64_t hi = min((uint64_t)offsets[s] / tile, tiles);
    for (uint64_t t = lo; t <= hi; ++t) tile_lb[t] = (uint32_t)s;
  }
}

__device__ __forceinline__ void st_raw_bits(void* p, uint64_t i, int esize, uint64_t bits) {
  switch (esize) {
    case 1: ((uint8_t*)p)[i] = (uint8_t)bits; break;
    case 2: ((uint16_t*)p)[i] = (uint16_t)bits; break;
    case 4: ((uint32_t*)p)[i] = (uint32_t)bits; break;
    default: ((uint64_t*)p)[i] = bits; break;
  }
}

template <class V, int OP, bool PLAIN, bool PK>
__global__ void __launch_bounds__(kThreads, kSegMinBlocks)
    seg_kernel(Src in, uint64_t cap, SegParams<V> p, TileState<SegVal<V>, PK> st) {
  using C = SegCfg<V>;
  using T = SegVal<V>;
  constexpr int VEC = C::VEC;
  constexpr bool DET = std::is_floating_point<V>::value;
  extern __shared__ __align__(16) unsigned char seg_smem[];
  T* stage = reinterpret_cast<T*>(seg_smem);  // kReduce only: TILE entries
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_bits[C::TILE / 32];
  __shared__ T s_warp_total[kWarps];
  __shared__ T s_excl;
  __shared__ uint64_t s_seg[3];  // continuing segment, first start, end
  __shared__ uint32_t s_head_te;

  const int tid = threadIdx.x;
  if (tid == 0) s_tile = atomicAdd(p.counter, 1u);
  for (int w = tid; w < C::TILE / 32; w += kThreads) s_bits[w] = 0;
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t n = in.len_dev ? min((uint64_t)*in.len_dev, cap) : cap;
  const uint64_t tb = tile * (uint64_t)C::TILE;
  if (tb >= n) return;
  const uint64_t te = min(tb + (uint64_t)C::TILE, n);
  const bool last_tile = te == n;

  // ---- value loads, issued first so their latency overlaps the heads ----
  const SegOp<V, OP> op{Op<V, OP>{p.op}};
  const int warp = tid >> 5, lane = tid & 31;
  const uint64_t warp_base = tb + (uint64_t)warp * C::WARP_ITEMS;
  const bool full = tb + C::TILE <= n;
  V raw[kLoads][VEC];
  if (PLAIN && full) {
#pragma unroll
    for (int j = 0; j < kLoads; ++j) {
      uint4 u = __ldcs(reinterpret_cast<const uint4*>((const V*)in.data + warp_base +
                                                      (uint64_t)(j * 32 + lane) * VEC));
      memcpy(raw[j], &u, 16);
    }
  } else if (!PLAIN && full && in.kind == MB_SRC_COLUMN && (uintptr_t)in.data % 16 == 0 &&
             (sizeof(V) == 4 ? (in.dtype == MB_U32 || in.dtype == MB_I32 || in.dtype == MB_F32)
                             : (in.dtype == MB_U64 || in.dtype == MB_I64 || in.dtype == MB_F64))) {
    // A mapped or cast column of V's width (a predicate's 0 / 1 flags for
    // count_if, say): the same 16-byte loads, the map applied per element.
#pragma unroll
    for (int j = 0; j < kLoads; ++j) {
      uint4 u = __ldcs(reinterpret_cast<const uint4*>(
          (const char*)in.data + (warp_base + (uint64_t)(j * 32 + lane) * VEC) * sizeof(V)));
      if constexpr (sizeof(V) == 4) {
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < VEC; ++k) raw[j][k] = map_to<V>(in.map, in.dtype, w[k]);
      } else {
        const uint64_t w[2] = {((uint64_t)u.y << 32) | u.x, ((uint64_t)u.w << 32) | u.z};
#pragma unroll
        for (int k = 0; k < VEC; ++k) raw[j][k] = map_to<V>(in.map, in.dtype, w[k]);
      }
    }
  } else if (!PLAIN && in.kind == MB_SRC_CONSTANT) {
    // A constant column (the count of a group-by): one value, no loads.
    const V c = src_load<V>(in, 0);
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
#pragma unroll
      for (int k = 0; k < VEC; ++k)
        raw[j][k] = warp_base + (uint64_t)(j * 32 + lane) * VEC + k < n ? c : V(0);
  } else {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
#pragma unroll
      for (int k = 0; k < VEC; ++k) {
        const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
        if (i < n) {
          if constexpr (PLAIN) raw[j][k] = ((const V*)in.data)[i];
          else raw[j][k] = src_load<V>(in, i);
        } else {
          raw[j][k] = V(0);
        }
      }
  }

  // ---- heads ----
  if (p.heads_src == kHeadsOffsets) {
    // Every thread reads the tile's segment range (broadcast loads).
    const uint64_t sa = p.tile_lb[tile];  // first start >= tb
    const uint64_t sb = last_tile ? p.nseg : min((uint64_t)p.tile_lb[tile + 1], p.nseg);
    if (tid == 0) {
      // The segment before sa holds tb (and continues into this tile)
      // unless one starts exactly at tb.
      s_seg[0] = (sa > 0 && p.offsets[sa] > tb) ? sa - 1 : ~0ull;
      s_seg[1] = sa;
      s_seg[2] = sb;
    }
    for (uint64_t s = sa + tid; s < sb; s += kThreads) {
      const uint64_t start = p.offsets[s];
      if (start >= tb && start < te) atomicOr(&s_bits[(start - tb) >> 5], 1u << ((start - tb) & 31));
    }
  } else if (p.head_bits) {
    // The heads pass left this tile's bitmap (key changes and segment
    // starts); the next tile's first bit says whether te is a head.
    constexpr int W = C::TILE / 32;
    const uint32_t* hb = p.head_bits + tile * W;
    for (int w = tid; w < W; w += kThreads) s_bits[w] = hb[w];
    if (tid == 0) s_head_te = te < n ? (p.head_bits[(tile + 1) * W] & 1u) : 1u;
  } else {
    for (uint64_t i = tb + tid; i < te; i += kThreads) {
      bool h = i == 0;
      if (!h) h = !key_eq(p.keys.vtype, src_load_bits(p.keys, i - 1), src_load_bits(p.keys, i));
      if (h) atomicOr(&s_bits[(i - tb) >> 5], 1u << ((i - tb) & 31));
    }
    if (tid == 0) {
      uint32_t h = te < n ? !key_eq(p.keys.vtype, src_load_bits(p.keys, te - 1),
                                    src_load_bits(p.keys, te))
                          : 1u;
      if (p.offsets) {  // segment starts are run heads too
        s_seg[1] = p.tile_lb[tile];
        if (te < n) {
          const uint64_t at = p.tile_lb[tile + 1];  // first start >= te
          s_seg[2] = min(at, p.nseg);
          if (at < p.nseg && p.offsets[at] == te) h = 1u;
        } else {
          s_seg[2] = p.nseg;
        }
      }
      s_head_te = h;
    }
    if (p.offsets) {
      __syncthreads();
      for (uint64_t s = s_seg[1] + tid; s < s_seg[2]; s += kThreads) {
        const uint64_t start = p.offsets[s];
        if (start >= tb && start < te) atomicOr(&s_bits[(start - tb) >> 5], 1u << ((start - tb) & 31));
      }
    }
  }
  __syncthreads();

  // ---- (value, head) pairs ----
  T x[kLoads][VEC];
#pragma unroll
  for (int j = 0; j < kLoads; ++j)
#pragma unroll
    for (int k = 0; k < VEC; ++k) {
      const uint32_t pos = (uint32_t)(warp_base - tb) + (j * 32 + lane) * VEC + k;
      x[j][k].v = raw[j][k];
      x[j][k].heads = (s_bits[pos >> 5] >> (pos & 31)) & 1u;
    }

  // ---- tile scan (same structure as the plain scan kernel) ----
#pragma unroll
  for (int j = 0; j < kLoads; ++j)
#pragma unroll
    for (int k = 1; k < VEC; ++k) x[j][k] = op(x[j][k - 1], x[j][k]);
  T ge[kLoads], rowtot[kLoads];
#pragma unroll
  for (int j = 0; j < kLoads; ++j) {
    T g = x[j][VEC - 1];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T o = shfl_up(g, d);
      if (lane >= d) g = op(o, g);
    }
    rowtot[j] = shfl_idx(g, 31);
    ge[j] = shfl_up(g, 1);
  }
  T rp[kLoads];
  rp[0] = rowtot[0];
#pragma unroll
  for (int j = 1; j < kLoads; ++j) rp[j] = op(rp[j - 1], rowtot[j]);
  if (lane == 0) s_warp_total[warp] = rp[kLoads - 1];
  __syncthreads();
  // no look-back: every tile starts fresh
  const bool local = p.mode == kReduceTiles || p.mode >= kScanInclTiles;
  if (warp == 0 && !local) {
    T agg = s_warp_total[0];
#pragma unroll
    for (int w = 1; w < kWarps; ++w) agg = op(agg, s_warp_total[w]);
    if (tile == 0) {
      if (lane == 0) st.publish(0, kFlagIncl, agg);
    } else {
      if (lane == 0) st.publish(tile, kFlagAgg, agg);
      T excl;
      if constexpr (DET) {
        excl = lookback_grouped<T>(st, tile, op, p.err, agg, agg);
      } else {
        excl = lookback_exclusive<T, SegOp<V, OP>, false>(st, tile, op, p.err, agg);
        if (lane == 0) st.publish(tile, kFlagIncl, op(excl, agg));
      }
      if (lane == 0) s_excl = excl;
    }
  }
  __syncthreads();
  bool has_pre = tile > 0 && !local;
  T pre = has_pre ? s_excl : T{0, V(0)};
  for (int w = 0; w < warp; ++w) {
    T t = s_warp_total[w];
    pre = has_pre ? op(pre, t) : t;
    has_pre = true;
  }
  T y[kLoads][VEC];
#pragma unroll
  for (int j = 0; j < kLoads; ++j) {
    bool h = has_pre;
    T pj = pre;
    if (j > 0) { pj = h ? op(pj, rp[j - 1]) : rp[j - 1]; h = true; }
    if (lane > 0) { pj = h ? op(pj, ge[j]) : ge[j]; h = true; }
#pragma unroll
    for (int k = 0; k < VEC; ++k) y[j][k] = h ? op(pj, x[j][k]) : x[j][k];
  }

  const Op<V, OP> vop{p.op};
  if (p.mode == kScanIncl || p.mode == kScanExcl || p.mode == kScanInclTiles ||
      p.mode == kScanExclTiles) {
    V o[kLoads][VEC];
    if (p.mode == kScanIncl || p.mode == kScanInclTiles) {
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) o[j][k] = y[j][k].v;
    } else {
#pragma unroll
      for (int j = 0; j < kLoads; ++j) {
        V up = shfl_up(y[j][VEC - 1].v, 1);
        V wrap = shfl_idx(j > 0 ? y[j - 1][VEC - 1].v : y[0][VEC - 1].v, 31);
        const V prev0 = lane > 0 ? up : (j > 0 ? wrap : pre.v);
        // A head restarts at init; any other item is init op inclusive of
        // the item before it (which lies in the same segment).
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          const uint32_t pos = (uint32_t)(warp_base - tb) + (j * 32 + lane) * VEC + k;
          const bool hd = ((s_bits[pos >> 5] >> (pos & 31)) & 1u) || tb + pos == 0;
          const V prev = k == 0 ? prev0 : y[j][k - 1].v;
          // (without the look-back, the items of a segment that came in from
          // an earlier tile keep their tile-local inclusive value here;
          // seg_scan_fix_kernel turns it into the exclusive result)
          o[j][k] = local && y[j][k].heads == 0 ? y[j][k].v
                                                : (hd ? p.init : vop(p.init, prev));
        }
      }
    }
    if (local) {  // the tile's tail fold, for the carries of later tiles
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
          if (i + 1 == te) p.part_tail[tile] = y[j][k].v;
        }
    }
    if (PLAIN && full && p.out_dtype == DTypeOf<V>::value) {
#pragma unroll
      for (int j = 0; j < kLoads; ++j) {
        uint4 u;
        memcpy(&u, o[j], 16);
        __stcs(reinterpret_cast<uint4*>((V*)p.out + warp_base + (uint64_t)(j * 32 + lane) * VEC), u);
      }
    } else {
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
          if (i < n) st_cast<V>(p.out_dtype, p.out, i, o[j][k]);
        }
    }
    return;
  }

  // ---- reductions: stage inclusive pairs, write one value per tail ----
  // (kReduceTiles: the segments that start and end in this tile are written
  // here; the tile leaves its fold before its first segment start, its fold
  // from its last start to its end, and the segment that starts there when it
  // goes on past the tile, for seg_reduce_cross_kernel.  Writing by segment
  // index keeps the per-segment stores coalesced.)
#pragma unroll
  for (int j = 0; j < kLoads; ++j)
#pragma unroll
    for (int k = 0; k < VEC; ++k) {
      const uint32_t pos = (uint32_t)(warp_base - tb) + (j * 32 + lane) * VEC + k;
      stage[pos] = y[j][k];
    }
  __syncthreads();
  if (p.heads_src == kHeadsOffsets) {
    // Segment s is written by the tile holding its tail (non-empty) or its
    // start (empty; the last tile takes starts at n).
    auto write_seg = [&](uint64_t s) {
      const uint64_t start = p.offsets[s], end = p.offsets[s + 1];
      if (start == end) {
        if ((start >= tb && start < te) || (last_tile && start >= te))
          st_cast<V>(p.out_dtype, p.out, s, p.init);
      } else if (end - 1 >= tb && end - 1 < te) {
        if (!local || start >= tb)  // else: finished by seg_reduce_cross_kernel
          st_cast<V>(p.out_dtype, p.out, s, vop(p.init, stage[end - 1 - tb].v));
      } else if (local && start >= tb && start < te) {
        p.tail_seg[tile] = (uint32_t)s;  // goes on past this tile
      }
    };
    if (tid == 0 && s_seg[0] != ~0ull) write_seg(s_seg[0]);
    for (uint64_t s = s_seg[1] + tid; s < s_seg[2]; s += kThreads) write_seg(s);
    if (local) {
      __shared__ uint32_t s_first;  // the tile's first segment start
      if (tid == 0) s_first = (uint32_t)(te - tb);
      __syncthreads();
      if (tid < C::TILE / 32 && s_bits[tid])
        atomicMin(&s_first, (uint32_t)tid * 32 + __ffs(s_bits[tid]) - 1);
      __syncthreads();
      if (tid == 0) {
        p.part_head[tile] = s_first > 0 ? stage[s_first - 1].v : p.init;
        p.part_tail[tile] = stage[te - tb - 1].v;
      }
    }
  } else if (local) {
    // kReduceKeysTiles: run index = the tile's first run index + the tile-
    // local inclusive head count - 1.  Items before the tile's first head
    // belong to the run that came in from an earlier tile.
    // One thread per bitmap word visits only its heads (the keys) and its
    // tails (items followed by a head; the tile's last item when the item
    // after the tile is one): runs are usually far fewer than items.
    const uint32_t base = p.run_base[tile];
    const uint32_t len = (uint32_t)(te - tb);
    const int words = (int)((len + 31) / 32);
    for (int w = tid; w < words; w += kThreads) {
      const uint32_t hb = s_bits[w];
      const uint32_t lo = (uint32_t)w * 32;
      const uint32_t valid = len - lo >= 32 ? ~0u : ((1u << (len - lo)) - 1u);
      uint32_t nxt = 0;  // whether the item after this word's last is a head
      if (lo + 32 < len) nxt = s_bits[w + 1] & 1u;
      else if (lo + 32 == len) nxt = s_head_te != 0;
      uint32_t tails = ((hb >> 1) | (nxt << 31)) & valid;
      if (len - lo < 32 && s_head_te) tails |= 1u << (len - 1 - lo);  // the tile's last item
      if (p.out_keys)
        for (uint32_t b = hb & valid; b; b &= b - 1) {
          const uint32_t pos = lo + (uint32_t)(__ffs(b) - 1);
          st_raw_bits(p.out_keys, base + stage[pos].heads - 1, p.out_key_esize,
                      src_load_bits(p.keys, tb + pos));
        }
      for (uint32_t b = tails; b; b &= b - 1) {
        const uint32_t pos = lo + (uint32_t)(__ffs(b) - 1);
        const T yv = stage[pos];
        if (yv.heads == 0) p.part_head[tile] = yv.v;  // the incoming run ends here
        else st_cast<V>(p.out_dtype, p.out, base + yv.heads - 1, vop(p.init, yv.v));
      }
    }
    if (tid == 0) {
      const T yl = stage[len - 1];
      p.part_tail[tile] = yl.v;
      if (yl.heads == 0) p.part_head[tile] = yl.v;  // no head in the tile: all of it
      else if (!s_head_te) p.tail_seg[tile] = base + yl.heads - 1;  // goes on past this tile
    }
    __shared__ uint32_t s_fp;  // the tile's first head
    if (tid == 0) s_fp = (uint32_t)(te - tb);
    __syncthreads();
    if (tid < C::TILE / 32 && s_bits[tid])
      atomicMin(&s_fp, (uint32_t)tid * 32 + __ffs(s_bits[tid]) - 1);
    __syncthreads();
    if (tid == 0) p.first_pos[tile] = s_fp;
  } else {
    // Runs of equal keys: key at the head, value at the tail, index =
    // inclusive head count - 1.
    for (uint64_t i = tb + tid; i < te; i += kThreads) {
      const uint32_t pos = (uint32_t)(i - tb);
      const T yv = stage[pos];
      const bool head = (s_bits[pos >> 5] >> (pos & 31)) & 1u;
      if (head && p.out_keys)
        st_raw_bits(p.out_keys, yv.heads - 1, p.out_key_esize, src_load_bits(p.keys, i));
      const bool tail = (i + 1 == te) ? (s_head_te != 0)
                                      : (((s_bits[(pos + 1) >> 5] >> ((pos + 1) & 31)) & 1u) != 0);
      if (tail) {
        st_cast<V>(p.out_dtype, p.out, yv.heads - 1, vop(p.init, yv.v));
        if (i + 1 == n && p.count_dev) *p.count_dev = yv.heads;
      }
    }
  }
}

template <class V>
size_t seg_smem(int mode) {
  return mode == kReduce || mode == kReduceTiles || mode == kReduceKeysTiles
             ? sizeof(SegVal<V>) * SegCfg<V>::TILE
             : 0;
}

// kReduceTiles: the segments that cross tile edges, one thread per tile
// whose last segment goes on past it: init op (the fold from its start to
// its tile's end) op (the whole folds of the tiles it covers) op (the fold
// before the first start of the tile it ends in), left to right, so the
// result is the same from run to run.
template <class V>
__global__ void __launch_bounds__(kThreads)
    seg_reduce_cross_kernel(const uint32_t* __restrict__ offsets, uint64_t tiles,
                            uint64_t tile_items, int op, V init, const V* __restrict__ part_head,
                            const V* __restrict__ part_tail, const uint32_t* __restrict__ tail_seg,
                            void* out, int out_dtype) {
  for (uint64_t t = blockIdx.x * (uint64_t)kThreads + threadIdx.x; t < tiles;
       t += (uint64_t)gridDim.x * kThreads) {
    const uint32_t s = tail_seg[t];
    if (s == ~0u) continue;
    const uint64_t last = ((uint64_t)offsets[s + 1] - 1) / tile_items;  // tile of its last item
    V acc = part_tail[t];
    for (uint64_t u = t + 1; u <= last && u < tiles; ++u)
      acc = op_apply_rt<V>(op, acc, u < last ? part_tail[u] : part_head[u]);
    st_cast<V>(out_dtype, out, s, op_apply_rt<V>(op, init, acc));
  }
}

// One block scans per-tile values over all tiles (carries, run bases).
constexpr int kCarryThreads = 1024;

// kReduceKeysTiles, first pass: the run heads of every tile -- items whose
// key differs from the one before (massively's Equal; the first item is a
// head) and, for reduce_by_key_segmented, segment starts -- counted into
// head_count[tile].
__global__ void __launch_bounds__(kThreads)
    seg_run_heads_kernel(Src keys, uint64_t cap, const uint32_t* __restrict__ n_dev,
                         const uint32_t* __restrict__ offsets, uint64_t nseg,
                         const uint32_t* __restrict__ tile_lb, uint64_t tile_items,
                         uint32_t* __restrict__ head_count, uint32_t* __restrict__ head_bits) {
  constexpr int kMaxWords = 4096 / 32;  // the largest tile (4-byte values)
  __shared__ uint32_t s_bits[kMaxWords];
  __shared__ uint32_t s_cnt;
  const uint64_t tile = blockIdx.x;
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t tb = tile * tile_items;
  if (tb >= n) return;
  const uint64_t te = min(tb + tile_items, n);
  const int words = (int)(tile_items / 32);
  for (int w = threadIdx.x; w < words; w += kThreads) s_bits[w] = 0;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  // A warp's 32 lanes take 32 consecutive items: one ballot is one bitmap
  // word.  Plain 4-byte keys are read directly (the item before comes from
  // the same or the previous line).
  const bool plain4 = keys.kind == MB_SRC_COLUMN && keys.map == MB_UN_IDENTITY &&
                      keys.dtype == keys.vtype &&
                      (keys.dtype == MB_U32 || keys.dtype == MB_I32 || keys.dtype == MB_F32);
  const uint32_t* kp = (const uint32_t*)keys.data;
  for (uint64_t b = tb; b < te; b += kThreads) {
    const uint64_t i = b + threadIdx.x;
    bool h = false;
    if (i < te) {
      h = i == 0;
      if (!h) {
        if (plain4) h = !key_eq(keys.vtype, __ldg(kp + i - 1), __ldg(kp + i));
        else h = !key_eq(keys.vtype, src_load_bits(keys, i - 1), src_load_bits(keys, i));
      }
    }
    const uint32_t word = __ballot_sync(kFull, h);
    if ((threadIdx.x & 31) == 0 && word) atomicOr(&s_bits[(i - tb) >> 5], word);
  }
  if (offsets) {
    const uint64_t sa = tile_lb[tile];
    const uint64_t sb = te == n ? nseg : min((uint64_t)tile_lb[tile + 1], nseg);
    for (uint64_t s = sa + threadIdx.x; s < sb; s += kThreads) {
      const uint64_t start = offsets[s];
      if (start >= tb && start < te) atomicOr(&s_bits[(start - tb) >> 5], 1u << ((start - tb) & 31));
    }
  }
  __syncthreads();
  uint32_t c = 0;
  for (int w = threadIdx.x; w < words; w += kThreads) {
    c += __popc(s_bits[w]);
    head_bits[tile * words + w] = s_bits[w];
  }
  c = __reduce_add_sync(kFull, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) head_count[tile] = s_cnt;
}

// kReduceKeysTiles: head counts -> each tile's first run index (exclusive
// sum, in place over `counts`) and the run count to counts[live] and
// count_dev.  One block:
// each thread sums a contiguous run of tiles, a block scan joins them.
__global__ void __launch_bounds__(kCarryThreads)
    seg_run_base_kernel(uint32_t* __restrict__ counts, uint64_t tiles, uint64_t tile_items,
                        uint64_t cap, const uint32_t* __restrict__ n_dev,
                        uint32_t* __restrict__ count_dev) {
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t live = min((n + tile_items - 1) / tile_items, tiles);
  const uint64_t per = (live + blockDim.x - 1) / blockDim.x;
  const uint64_t u0 = threadIdx.x * per, u1 = min(u0 + per, live);
  uint32_t sum = 0;
  for (uint64_t u = u0; u < u1; ++u) sum += counts[u];
  __shared__ uint32_t s_v[kCarryThreads];
  s_v[threadIdx.x] = sum;
  __syncthreads();
  for (int d = 1; d < (int)blockDim.x; d <<= 1) {
    const uint32_t x = threadIdx.x >= (unsigned)d ? s_v[threadIdx.x - d] : 0u;
    __syncthreads();
    s_v[threadIdx.x] += x;
    __syncthreads();
  }
  uint32_t run = s_v[threadIdx.x] - sum;  // exclusive
  for (uint64_t u = u0; u < u1; ++u) {
    const uint32_t c = counts[u];
    counts[u] = run;
    run += c;
  }
  if (threadIdx.x == blockDim.x - 1) {
    counts[live] = s_v[threadIdx.x];  // the run count, after the last tile's base
    if (count_dev) *count_dev = s_v[threadIdx.x];
  }
}

// kReduceKeysTiles: the runs that cross tile edges.  One block scans
// (has a head, tail fold) over the tiles -- the segmented scan of
// seg_tile_carry_kernel -- so `run` is the fold of the run still open at the
// end of tile u - 1.  That run ends in the first later tile with a head
// (after the fold of the items before that head, part_head) or at the end of
// the data; it is written there unless it ended exactly at the end of a tile
// that wrote it itself (a head in tile u - 1 and one at the start of tile
// u).  Work is O(tiles) whatever the run lengths.
template <class V>
__global__ void __launch_bounds__(kCarryThreads)
    seg_rbk_walk_kernel(uint64_t tiles, uint64_t tile_items, uint64_t cap,
                        const uint32_t* __restrict__ n_dev, int op, V init,
                        const V* __restrict__ part_head, const V* __restrict__ part_tail,
                        const uint32_t* __restrict__ first_pos,
                        const uint32_t* __restrict__ run_base, void* out, int out_dtype) {
  using T = SegVal<V>;
  const SegOp<V, kOpDyn> sop{Op<V, kOpDyn>{op}};
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t live = min((n + tile_items - 1) / tile_items, tiles);
  if (live == 0) return;
  const uint64_t per = (live + kCarryThreads - 1) / kCarryThreads;
  const uint64_t u0 = threadIdx.x * per, u1 = min(u0 + per, live);
  auto has_head = [&](uint64_t u) -> bool {
    return (uint64_t)first_pos[u] < min(tile_items, n - u * tile_items);
  };
  T agg{0, V(0)};
  bool has = false;
  for (uint64_t u = u0; u < u1; ++u) {
    const T x{has_head(u) ? 1u : 0u, part_tail[u]};
    agg = has ? sop(agg, x) : x;
    has = true;
  }
  __shared__ T s_v[kCarryThreads];
  __shared__ int s_h[kCarryThreads];
  s_v[threadIdx.x] = agg;
  s_h[threadIdx.x] = has;
  __syncthreads();
  for (int d = 1; d < kCarryThreads; d <<= 1) {  // inclusive, in thread order
    T x{};
    int hx = 0;
    if (threadIdx.x >= d && s_h[threadIdx.x - d]) {
      x = s_h[threadIdx.x] ? sop(s_v[threadIdx.x - d], s_v[threadIdx.x]) : s_v[threadIdx.x - d];
      hx = 1;
    }
    __syncthreads();
    if (hx) {
      s_v[threadIdx.x] = x;
      s_h[threadIdx.x] = 1;
    }
    __syncthreads();
  }
  T run{0, V(0)};
  bool rh = threadIdx.x > 0 && s_h[threadIdx.x - 1];
  if (rh) run = s_v[threadIdx.x - 1];
  bool prev_head = u0 > 0 && u0 < u1 && has_head(u0 - 1);
  for (uint64_t u = u0; u < u1; ++u) {
    const bool hh = has_head(u);
    if (u > 0 && hh) {
      const uint32_t fp = first_pos[u];
      if (fp > 0 || !prev_head)
        st_cast<V>(out_dtype, out, run_base[u] - 1,
                   op_apply_rt<V>(op, init, fp > 0 ? op_apply_rt<V>(op, run.v, part_head[u])
                                                   : run.v));
    }
    const T x{hh ? 1u : 0u, part_tail[u]};
    run = rh ? sop(run, x) : x;
    rh = true;
    prev_head = hh;
  }
  // The last run, when no head in the last tile let that tile write it.
  if (u0 < u1 && u1 == live && !prev_head)
    st_cast<V>(out_dtype, out, run_base[live] - 1, op_apply_rt<V>(op, init, run.v));
}

// reduce_by_key of a constant integer column under ADD: every run's value is
// init + c * (its length), so no value pass is needed.  seg_run_starts_kernel
// turns the call's run-head bitmap (tiles of `tile_items`) and run bases into
// each run's first position, one block per tile; seg_const_runs_kernel writes
// the values.  Integer adds wrap, so c * length equals the repeated adds.
__global__ void __launch_bounds__(kThreads)
    seg_run_starts_kernel(const uint32_t* __restrict__ head_bits,
                          const uint32_t* __restrict__ run_base, uint64_t tile_items,
                          uint64_t cap, const uint32_t* __restrict__ n_dev,
                          uint32_t* __restrict__ starts) {
  __shared__ uint32_t s_wsum[kWarps];
  const uint64_t tile = blockIdx.x;
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t tb = tile * tile_items;
  if (tb >= n) return;
  const int words = (int)(tile_items / 32);  // at most kThreads
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t w = (int)threadIdx.x < words ? head_bits[tile * words + threadIdx.x] : 0u;
  const uint32_t c = (uint32_t)__popc(w);
  uint32_t incl = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(kFull, incl, d);
    if (lane >= d) incl += o;
  }
  if (lane == 31) s_wsum[warp] = incl;
  __syncthreads();
  uint32_t r = run_base[tile] + incl - c;
  for (int v = 0; v < warp; ++v) r += s_wsum[v];
  for (uint32_t bits = w; bits; bits &= bits - 1)
    starts[r++] = (uint32_t)(tb + threadIdx.x * 32u + (uint32_t)(__ffs(bits) - 1));
}

template <class V>
__global__ void __launch_bounds__(kThreads)
    seg_const_runs_kernel(const uint32_t* __restrict__ starts,
                          const uint32_t* __restrict__ run_base, uint64_t tile_items,
                          uint64_t cap, const uint32_t* __restrict__ n_dev, V init, V value,
                          void* out, int out_dtype) {
  using U = typename std::make_unsigned<V>::type;
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t runs = run_base[(n + tile_items - 1) / tile_items];
  for (uint64_t r = blockIdx.x * (uint64_t)kThreads + threadIdx.x; r < runs;
       r += (uint64_t)gridDim.x * kThreads) {
    const uint64_t end = r + 1 < runs ? (uint64_t)starts[r + 1] : n;
    const U len = (U)(end - starts[r]);
    st_cast<V>(out_dtype, out, r, (V)((U)init + (U)value * len));
  }
}

// Whether tile t (items [t * tile_items, te)) holds a segment start: the
// first start at or after its beginning lies before its end.
__device__ __forceinline__ bool tile_has_start(const uint32_t* offsets, const uint32_t* tile_lb,
                                               uint64_t t, uint64_t te) {
  return (uint64_t)offsets[tile_lb[t]] < te;
}


// kScan*Tiles: carry[t] = the fold of the segment that enters tile t over
// the items before t -- the value of an inclusive segmented scan, over the
// tiles, of (tile holds a start, its tail fold) at tile t - 1.  One block;
// each thread folds a contiguous run of tiles, a block scan (fixed shape)
// joins the runs, and the threads walk their runs again, so the result is
// the same from run to run.
template <class V>
__global__ void __launch_bounds__(kCarryThreads)
    seg_tile_carry_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ tile_lb,
                          uint64_t tiles, uint64_t tile_items, uint64_t cap,
                          const uint32_t* __restrict__ n_dev, int op,
                          const V* __restrict__ part_tail, V* __restrict__ carry) {
  using T = SegVal<V>;
  const SegOp<V, kOpDyn> sop{Op<V, kOpDyn>{op}};
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t live = (n + tile_items - 1) / tile_items < tiles ? (n + tile_items - 1) / tile_items
                                                                  : tiles;
  const uint64_t per = (live + kCarryThreads - 1) / kCarryThreads;
  const uint64_t u0 = threadIdx.x * per, u1 = min(u0 + per, live);
  auto item = [&](uint64_t u) -> T {
    const uint64_t te = min((u + 1) * tile_items, n);
    return T{tile_has_start(offsets, tile_lb, u, te) ? 1u : 0u, part_tail[u]};
  };
  T agg{0, V(0)};
  bool has = false;
  for (uint64_t u = u0; u < u1; ++u) {
    const T x = item(u);
    agg = has ? sop(agg, x) : x;
    has = true;
  }
  __shared__ T s_v[kCarryThreads];
  __shared__ int s_h[kCarryThreads];
  s_v[threadIdx.x] = agg;
  s_h[threadIdx.x] = has;
  __syncthreads();
  for (int d = 1; d < kCarryThreads; d <<= 1) {  // inclusive, in thread order
    T x{};
    int hx = 0;
    if (threadIdx.x >= d && s_h[threadIdx.x - d]) {
      x = s_h[threadIdx.x] ? sop(s_v[threadIdx.x - d], s_v[threadIdx.x]) : s_v[threadIdx.x - d];
      hx = 1;
    }
    __syncthreads();
    if (hx) {
      s_v[threadIdx.x] = x;
      s_h[threadIdx.x] = 1;
    }
    __syncthreads();
  }
  T run{0, V(0)};
  bool rh = threadIdx.x > 0 && s_h[threadIdx.x - 1];
  if (rh) run = s_v[threadIdx.x - 1];
  for (uint64_t u = u0; u < u1; ++u) {
    if (rh) carry[u] = run.v;
    const T x = item(u);
    run = rh ? sop(run, x) : x;
    rh = true;
  }
}

// kScan*Tiles: the items of tile t before its first segment start belong to
// a segment that began in an earlier tile; the tile kernel left their
// tile-local inclusive values in `out`.  Inclusive: carry op local;
// exclusive: init op (carry op local of the item before), init op carry for
// the tile's first item.  All loads come before the barrier, all stores
// after it.
template <class V>
__global__ void __launch_bounds__(kThreads)
    seg_scan_fix_kernel(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ tile_lb,
                        uint64_t tile_items, uint64_t cap, const uint32_t* __restrict__ n_dev,
                        int op, int exclusive, V init, const V* __restrict__ carry, void* out,
                        int out_dtype) {
  constexpr int MAXR = (int)(SegCfg<V>::TILE / kThreads);
  const uint64_t t = blockIdx.x + 1;  // tile 0 starts with a segment
  const uint64_t n = n_dev ? min((uint64_t)*n_dev, cap) : cap;
  const uint64_t tb = t * tile_items;
  if (tb >= n) return;
  const uint64_t te = min(tb + tile_items, n);
  const uint64_t first = min((uint64_t)offsets[tile_lb[t]], te);
  if (first == tb) return;
  const uint64_t len = first - tb;
  const V c = carry[t];
  Src o{};
  o.kind = MB_SRC_COLUMN;
  o.dtype = out_dtype;
  o.vtype = DTypeOf<V>::value;
  o.map = MB_UN_IDENTITY;
  o.data = out;
  o.len = cap;
  V x[MAXR], xp[MAXR];
#pragma unroll
  for (int r = 0; r < MAXR; ++r) {
    const uint64_t i = (uint64_t)r * kThreads + threadIdx.x;
    if (i < len) {
      x[r] = src_load<V>(o, tb + i);
      if (exclusive && i > 0) xp[r] = src_load<V>(o, tb + i - 1);
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < MAXR; ++r) {
    const uint64_t i = (uint64_t)r * kThreads + threadIdx.x;
    if (i >= len) continue;
    V v;
    if (!exclusive) v = op_apply_rt<V>(op, c, x[r]);
    else v = op_apply_rt<V>(op, init, i == 0 ? c : op_apply_rt<V>(op, c, xp[r]));
    st_cast<V>(out_dtype, out, tb + i, v);
  }
}

// kReduceKeysTiles: run bases shared by the value columns of one
// reduce_by_key call (`ptr` holds tiles + 1 words for the smallest tile;
// `tile` is the tile size they were computed for, 0 before the first).
struct RunBases {
  uint32_t* ptr = nullptr;
  uint32_t* bits = nullptr;  // the head bitmap: n / 32 + 256 words
  uint64_t tile = 0;
};

template <class V>
int seg_run(mb_executor* ex, const mb_src& in, SegParams<V> p, const void* init_wide,
            RunBases* rb) {
  using C = SegCfg<V>;
  const uint64_t cap = in.len;
  if (cap == 0) return MB_OK;
  memcpy(&p.init, init_wide, sizeof(V));
  const uint64_t tiles = (cap + C::TILE - 1) / C::TILE;
  using T = SegVal<V>;
  // Packed states when the pair fits one word beside its flag.
  const bool pk = StatePack<T>::kPackable && cap < (1ull << 30);
  const size_t state_b =
      pk ? TileState<T, true>::bytes(tiles) : TileState<T, false>::bytes(tiles);
  const size_t lb_b = p.offsets ? ((tiles + 1) * 4 + 255) / 256 * 256 : 0;
  // kReduceTiles: part_head, part_tail, tail_seg; kScan*Tiles: part_tail and
  // the carries (in the part_head slot).
  const bool scan_tiles = p.mode == kScanInclTiles || p.mode == kScanExclTiles;
  const bool keys_tiles = p.mode == kReduceKeysTiles;
  const bool tiles_mode = p.mode == kReduceTiles || scan_tiles || keys_tiles;
  const size_t part_b = tiles_mode ? (tiles * sizeof(V) + 255) / 256 * 256 : 0;
  const size_t tseg_b = tiles_mode ? (tiles * 4 + 255) / 256 * 256 : 0;
  // kReduceKeysTiles: run bases (tiles + 1 words) and first-head positions,
  // then the head bitmap (unless shared)
  const size_t keys_b = keys_tiles ? 2 * (((tiles + 1) * 4 + 255) / 256 * 256) : 0;
  const size_t bits_b = keys_tiles && !(rb && rb->ptr) ? (tiles + 1) * (C::TILE / 32) * 4 : 0;
  Scratch scratch;
  MB_TRY(scratch.alloc(ex, 256 + state_b + lb_b + 2 * part_b + tseg_b + keys_b + bits_b));
  MB_CUDA(cudaMemsetAsync(scratch.ptr, 0, 256 + state_b, ex->stream));
  p.counter = scratch.as<uint32_t>();
  p.err = DevErr{ex->status_dev, scratch.as<uint32_t>() + 1};
  if (tiles_mode) {
    char* q = scratch.as<char>() + 256 + state_b + lb_b;
    p.part_head = (V*)q;
    p.part_tail = (V*)(q + part_b);
    p.tail_seg = (uint32_t*)(q + 2 * part_b);
    MB_CUDA(cudaMemsetAsync(p.tail_seg, 0xFF, tiles * 4, ex->stream));
    if (keys_tiles) {
      uint32_t* base = (uint32_t*)(q + 2 * part_b + tseg_b);
      p.first_pos = (uint32_t*)((char*)base + keys_b / 2);
      uint32_t* bits = (uint32_t*)(q + 2 * part_b + tseg_b + keys_b);
      if (rb && rb->ptr) {
        base = rb->ptr;
        bits = rb->bits;
      }
      p.run_base = base;
      p.head_bits = bits;
      if (!rb || rb->tile != (uint64_t)C::TILE)
        MB_CUDA(cudaMemsetAsync(base, 0, (tiles + 1) * 4, ex->stream));
    }
  }
  if (p.offsets) {
    uint32_t* lb = (uint32_t*)(scratch.as<char>() + 256 + state_b);
    MB_CUDA(cudaMemsetAsync(lb, 0xFF, (tiles + 1) * 4, ex->stream));
    const uint64_t blocks = std::min<uint64_t>((p.nseg + kThreads) / kThreads, 4096);
    seg_tile_bounds_kernel<<<(unsigned)std::max<uint64_t>(1, blocks), kThreads, 0, ex->stream>>>(
        p.offsets, p.nseg, C::TILE, tiles, lb);
    MB_CUDA(cudaGetLastError());
    p.tile_lb = lb;
  }
  const bool plain = src_plain(in, DTypeOf<V>::value) && (uintptr_t)in.data % 16 == 0 &&
                     (p.mode == kReduce || p.mode == kReduceTiles || keys_tiles ||
                      (uintptr_t)p.out % 16 == 0);
  const Src s = to_src(in);
  if (keys_tiles && (!rb || rb->tile != (uint64_t)C::TILE)) {
    // Every tile's first run index, and the run count.
    if (rb && rb->ptr) rb->tile = C::TILE;
    seg_run_heads_kernel<<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
        p.keys, cap, in.len_dev, p.offsets, p.nseg, p.tile_lb, C::TILE, (uint32_t*)p.run_base,
        (uint32_t*)p.head_bits);
    MB_CUDA(cudaGetLastError());
    seg_run_base_kernel<<<1, kCarryThreads, 0, ex->stream>>>(
        (uint32_t*)p.run_base, tiles, C::TILE, cap, in.len_dev, p.count_dev);
    MB_CUDA(cudaGetLastError());
  }
  const size_t smem = seg_smem<V>(p.mode);
  char* state_base = scratch.as<char>() + 256;
  auto launch = [&](auto kern, auto st) -> int {
    if (smem > 48 * 1024)
      MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)tiles, kThreads, smem, ex->stream>>>(s, cap, p, st);
    return MB_OK;
  };
#define MB_SEG_LAUNCH(OPID)                                                           \
  do {                                                                                \
    if constexpr (StatePack<T>::kPackable) {                                          \
      if (pk) {                                                                       \
        auto st = TileState<T, true>::make(state_base, tiles);                        \
        MB_TRY(plain ? launch(seg_kernel<V, OPID, true, true>, st)                     \
                     : launch(seg_kernel<V, OPID, false, true>, st));                  \
        break;                                                                        \
      }                                                                               \
    }                                                                                 \
    auto st = TileState<T, false>::make(state_base, tiles);                           \
    MB_TRY(plain ? launch(seg_kernel<V, OPID, true, false>, st)                        \
                 : launch(seg_kernel<V, OPID, false, false>, st));                     \
  } while (0)
  switch (p.op) {
    case MB_OP_ADD: MB_SEG_LAUNCH(MB_OP_ADD); break;
    case MB_OP_MIN: MB_SEG_LAUNCH(MB_OP_MIN); break;
    case MB_OP_MAX: MB_SEG_LAUNCH(MB_OP_MAX); break;
    default: MB_SEG_LAUNCH(kOpDyn); break;
  }
#undef MB_SEG_LAUNCH
  MB_CUDA(cudaGetLastError());
  if (scan_tiles) {
    seg_tile_carry_kernel<V><<<1, kCarryThreads, 0, ex->stream>>>(
        p.offsets, p.tile_lb, tiles, C::TILE, cap, in.len_dev, p.op, p.part_tail, p.part_head);
    MB_CUDA(cudaGetLastError());
    if (tiles > 1) {
      seg_scan_fix_kernel<V><<<(unsigned)(tiles - 1), kThreads, 0, ex->stream>>>(
          p.offsets, p.tile_lb, C::TILE, cap, in.len_dev, p.op,
          p.mode == kScanExclTiles ? 1 : 0, p.init, p.part_head, p.out, p.out_dtype);
      MB_CUDA(cudaGetLastError());
    }
  } else if (keys_tiles) {
    seg_rbk_walk_kernel<V><<<1, kCarryThreads, 0, ex->stream>>>(
        tiles, C::TILE, cap, in.len_dev, p.op, p.init, p.part_head, p.part_tail, p.first_pos,
        p.run_base, p.out, p.out_dtype);
    MB_CUDA(cudaGetLastError());
  } else if (tiles_mode) {
    const unsigned g = (unsigned)std::min<uint64_t>((tiles + kThreads - 1) / kThreads, 4096);
    seg_reduce_cross_kernel<V><<<std::max(1u, g), kThreads, 0, ex->stream>>>(
        p.offsets, tiles, C::TILE, p.op, p.init, p.part_head, p.part_tail, p.tail_seg, p.out,
        p.out_dtype);
    MB_CUDA(cudaGetLastError());
  }
  return MB_OK;
}

// Common set-up of every segmented call.  `out` holds per-element results
// (scans) or per-segment / per-run results (reductions).
int seg_entry(mb_executor* ex, const mb_src* values, int op, int mode, const void* init,
              void* out, int out_dtype, const uint32_t* offsets, uint64_t nseg,
              const mb_src* keys, void* out_keys, int out_key_esize, uint32_t* count_dev,
              RunBases* rb = nullptr) {
  const int ct = compute_type(values->vtype);
  if (!op_valid_for(op, ct)) return set_error(MB_ERR_LAUNCH, "operator not defined for this type");
  uint64_t init_wide = 0;
  if (init) {
    uint64_t raw = 0;
    memcpy(&raw, init, dtype_size(values->vtype));
    switch (values->vtype) {
      case MB_I8: init_wide = (uint64_t)(int64_t)(int8_t)raw; break;
      case MB_I16: init_wide = (uint64_t)(int64_t)(int16_t)raw; break;
      default: init_wide = raw; break;
    }
  }
#define MB_SEG_DISPATCH(V)                                          \
  {                                                                 \
    SegParams<V> p{};                                               \
    p.op = op;                                                      \
    p.mode = mode;                                                  \
    p.heads_src = keys ? kHeadsKeys : kHeadsOffsets;                \
    p.out_dtype = out_dtype;                                        \
    p.offsets = offsets;                                            \
    p.nseg = nseg;                                                  \
    if (keys) p.keys = to_src(*keys);                               \
    p.out = out;                                                    \
    p.out_keys = out_keys;                                          \
    p.out_key_esize = out_key_esize;                                \
    p.count_dev = count_dev;                                        \
    return seg_run<V>(ex, *values, p, &init_wide, rb);              \
  }
  switch (ct) {
    case MB_U32: MB_SEG_DISPATCH(uint32_t)
    case MB_I32: MB_SEG_DISPATCH(int32_t)
    case MB_U64: MB_SEG_DISPATCH(uint64_t)
    case MB_I64: MB_SEG_DISPATCH(int64_t)
    case MB_F32: MB_SEG_DISPATCH(float)
    case MB_F64: MB_SEG_DISPATCH(double)
    default: break;
  }
#undef MB_SEG_DISPATCH
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

// ------------------------------------------------------ segmentation ----

__global__ void validate_offsets_kernel(const uint32_t* off, uint64_t count, uint32_t* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if ((i == 0 && off[0] != 0) || (i > 0 && off[i] < off[i - 1])) atomicMax(bad, 1u);
  }
}

// offsets[0] = 0, offsets[s+1] = prefix[s]; flags a total above u32.
__global__ void offsets_from_prefix_kernel(const uint64_t* prefix, uint64_t nseg, uint32_t* off,
                                           uint32_t* status) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= nseg;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (s == 0) { off[0] = 0; continue; }
    const uint64_t v = prefix[s - 1];
    if (v > 0xFFFFFFFFull) atomicMax(status, 1u);
    off[s] = (uint32_t)v;
    if (s == nseg) status[1] = (uint32_t)v;
  }
}

__global__ void lengths_kernel(const uint32_t* off, uint64_t nseg, uint32_t* len) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nseg;
       s += (uint64_t)gridDim.x * blockDim.x)
    len[s] = off[s + 1] - off[s];
}

__global__ void local_indices_kernel(const uint32_t* off, uint64_t nseg, uint32_t* local,
                                     uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    local[i] = (uint32_t)(i - off[upper_bound_u32(off, nseg + 1, i) - 1]);
}

// Segment ids of a chunk of kIdTile items per block, without a search per
// item: the chunk's segment starts (from the per-tile lower bounds) are
// counted per position in shared memory and scanned, so id(i) = (first
// segment starting in the chunk) - 1 + starts at or before i.  COMP writes
// the sort key (id << 32) | enc(value) of a 4-byte value instead of the id:
// enc orders unsigned (0), signed (1) or float (2, total order) bits as
// unsigned, complemented when `desc`; with `ieee`, -0 counts as +0.
constexpr int kIdItems = 16;
constexpr int kIdTile = kThreads * kIdItems;

template <bool COMP>
__global__ void __launch_bounds__(kThreads)
    seg_ids_kernel(const uint32_t* __restrict__ off, uint64_t nseg, uint64_t n,
                   const uint32_t* __restrict__ tile_lb, uint32_t* __restrict__ ids, Src values,
                   int enc, int desc, int ieee, uint64_t* __restrict__ comp) {
  __shared__ uint32_t cnt[kIdTile];
  __shared__ uint32_t wsum[kWarps];
  const uint64_t c0 = (uint64_t)blockIdx.x * kIdTile;
  if (c0 >= n) return;
  const uint64_t c1 = min(c0 + (uint64_t)kIdTile, n);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kIdTile; i += kThreads) cnt[i] = 0;
  __syncthreads();
  const uint64_t lb = tile_lb[blockIdx.x];  // first s with off[s] >= c0
  const uint64_t lbn = c1 < n ? (uint64_t)tile_lb[blockIdx.x + 1] : nseg + 1;
  for (uint64_t sg = max(lb, (uint64_t)1) + tid; sg < lbn; sg += kThreads) {
    const uint64_t o = off[sg];
    if (o < c1) atomicAdd(&cnt[o - c0], 1u);
  }
  __syncthreads();
  // Warp w scans positions [512 w, 512 w + 512) in rounds of 32.
  uint32_t carry = 0;
  uint32_t loc[kIdItems];
#pragma unroll
  for (int k = 0; k < kIdItems; ++k) {
    uint32_t v = cnt[warp * 32 * kIdItems + k * 32 + lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, v, d);
      if (lane >= d) v += o;
    }
    loc[k] = carry + v;
    carry += __shfl_sync(kFull, v, 31);
  }
  if (lane == 0) wsum[warp] = carry;
  __syncthreads();
  uint32_t base = lb >= 1 ? (uint32_t)(lb - 1) : 0u;
  for (int w = 0; w < warp; ++w) base += wsum[w];
#pragma unroll
  for (int k = 0; k < kIdItems; ++k) {
    const uint64_t i = c0 + (uint64_t)warp * 32 * kIdItems + k * 32 + lane;
    if (i >= c1) break;
    const uint32_t id = base + loc[k];
    if constexpr (COMP) {
      uint32_t u = (uint32_t)src_load_bits(values, i);
      if (ieee && (u & 0x7FFFFFFFu) == 0) u = 0;  // -0 == +0 under `<`
      if (enc == 1) u ^= 0x80000000u;
      else if (enc == 2) u = (u & 0x80000000u) ? ~u : (u ^ 0x80000000u);
      if (desc) u = ~u;
      comp[i] = ((uint64_t)id << 32) | u;
    } else {
      ids[i] = id;
    }
  }
}

// Inverse of the COMP encoding: the low 32 bits of a sorted key back to the
// value's bits.
__global__ void __launch_bounds__(kThreads)
    seg_decode_kernel(const uint64_t* __restrict__ comp, uint64_t n, int enc, int desc,
                      uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * kThreads) {
    uint32_t u = (uint32_t)comp[i];
    if (desc) u = ~u;
    if (enc == 1) u ^= 0x80000000u;
    else if (enc == 2) u = (u & 0x80000000u) ? (u ^ 0x80000000u) : ~u;
    out[i] = u;
  }
}

// ids must be non-decreasing and < nseg; bad[0] is set otherwise.
__global__ void validate_ids_kernel(Src ids, uint64_t n, uint64_t nseg, uint32_t* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = src_load<uint32_t>(ids, i);
    if (v >= nseg || (i > 0 && src_load<uint32_t>(ids, i - 1) > v)) atomicMax(bad, 1u);
  }
}

// offsets[s] = first index i with ids[i] >= s (massively's lower_bound of
// counting(0) against the ids).
__global__ void offsets_from_ids_kernel(Src ids, uint64_t n, uint64_t nseg, uint32_t* off) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= nseg;
       s += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if ((uint64_t)src_load<uint32_t>(ids, mid) < s) lo = mid + 1;
      else hi = mid;
    }
    off[s] = (uint32_t)lo;
  }
}

unsigned grid_for_n(uint64_t n) {
  uint64_t g = (n + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 8));
}

int check_values_out(mb_executor* ex, const mb_src* values, const mb_col& out, uint64_t need) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_col(ex, out, "output"));
  if (out.len < need)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", need, out.len);
  if (compute_type(out.dtype) != compute_type(values->vtype))
    return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  return MB_OK;
}

}  // namespace

// Segment ids (ids != null) or the composite sort keys of a 4-byte value
// column (comp != null) for `n` items over canonical offsets.
int seg_ids_fill(mb_executor* ex, const uint32_t* offsets, uint64_t nseg, uint64_t n,
                 uint32_t* ids, const mb_src* values, int enc, int desc, int ieee,
                 uint64_t* comp) {
  if (n == 0) return MB_OK;
  const uint64_t tiles = (n + kIdTile - 1) / kIdTile;
  Scratch lb;
  MB_TRY(lb.alloc(ex, (tiles + 1) * 4));
  MB_CUDA(cudaMemsetAsync(lb.ptr, 0xFF, (tiles + 1) * 4, ex->stream));
  const uint64_t blocks = std::min<uint64_t>((nseg + kThreads) / kThreads, 4096);
  seg_tile_bounds_kernel<<<(unsigned)std::max<uint64_t>(1, blocks), kThreads, 0, ex->stream>>>(
      offsets, nseg, kIdTile, tiles, lb.as<uint32_t>());
  MB_CUDA(cudaGetLastError());
  const Src v = values ? to_src(*values) : Src{};
  if (comp)
    seg_ids_kernel<true><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
        offsets, nseg, n, lb.as<uint32_t>(), nullptr, v, enc, desc, ieee, comp);
  else
    seg_ids_kernel<false><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
        offsets, nseg, n, lb.as<uint32_t>(), ids, v, 0, 0, 0, nullptr);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int seg_decode_u32(mb_executor* ex, const uint64_t* comp, uint64_t n, int enc, int desc,
                   uint32_t* out) {
  if (n == 0) return MB_OK;
  const unsigned g = (unsigned)std::min<uint64_t>((n + kThreads - 1) / kThreads, 148ull * 16);
  seg_decode_kernel<<<g, kThreads, 0, ex->stream>>>(comp, n, enc, desc, out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" {

int mb_segmentation_validate_offsets(mb_executor* ex, const uint32_t* offsets,
                                     uint64_t offset_count, uint32_t* value_count) {
  MB_TRY(check_exec(ex));
  if (offset_count == 0 || !offsets)
    return set_error(MB_ERR_INVALID_SEGMENTATION, "segmentation is not a valid ordered partition");
  MB_TRY(check_len_u32(offset_count - 1));
  Scratch bad;
  MB_TRY(bad.alloc(ex, 16));
  MB_CUDA(cudaMemsetAsync(bad.ptr, 0, 16, ex->stream));
  validate_offsets_kernel<<<grid_for_n(offset_count), 256, 0, ex->stream>>>(offsets, offset_count,
                                                                           bad.as<uint32_t>());
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaMemcpyAsync(bad.as<uint32_t>() + 1, offsets + offset_count - 1, 4,
                          cudaMemcpyDeviceToDevice, ex->stream));
  if (ex->capturing) return set_error(MB_ERR_LAUNCH, "validation cannot run inside graph capture");
  MB_CUDA(cudaMemcpyAsync(ex->host_pinned, bad.ptr, 8, cudaMemcpyDeviceToHost, ex->stream));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  if (ex->host_pinned[0] != 0)
    return set_error(MB_ERR_INVALID_SEGMENTATION, "segmentation is not a valid ordered partition");
  if (value_count) *value_count = ex->host_pinned[1];
  return MB_OK;
}

int mb_segmentation_from_lengths(mb_executor* ex, const mb_src* lengths, uint32_t* offsets,
                                 uint32_t* value_count) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, lengths, "lengths"));
  const uint64_t nseg = lengths->len;
  if (nseg >= 0xFFFFFFFFull)
    return set_error(MB_ERR_LENGTH_TOO_LARGE, "length does not fit in u32", nseg + 1);
  Scratch pre, stat;
  MB_TRY(stat.alloc(ex, 16));
  MB_CUDA(cudaMemsetAsync(stat.ptr, 0, 16, ex->stream));
  if (nseg > 0) {
    MB_TRY(pre.alloc(ex, nseg * 8));
    mb_src wide = *lengths;
    wide.vtype = MB_U64;  // lengths summed in u64 to detect overflow
    mb_col c{};
    c.data = pre.ptr;
    c.dtype = MB_U64;
    c.len = nseg;
    MB_TRY(mb_inclusive_scan(ex, &wide, MB_OP_ADD, c));
  }
  offsets_from_prefix_kernel<<<grid_for_n(nseg + 1), 256, 0, ex->stream>>>(
      pre.as<uint64_t>(), nseg, offsets, stat.as<uint32_t>());
  MB_CUDA(cudaGetLastError());
  if (ex->capturing) return set_error(MB_ERR_LAUNCH, "validation cannot run inside graph capture");
  MB_CUDA(cudaMemcpyAsync(ex->host_pinned, stat.ptr, 8, cudaMemcpyDeviceToHost, ex->stream));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  if (ex->host_pinned[0] != 0)
    return set_error(MB_ERR_LENGTH_TOO_LARGE, "length does not fit in u32", 0x100000000ull);
  if (value_count) *value_count = ex->host_pinned[1];
  return MB_OK;
}

int mb_segmentation_segment_ids(mb_executor* ex, const uint32_t* offsets, uint64_t segment_count,
                                uint32_t* ids, uint64_t value_count) {
  MB_TRY(check_exec(ex));
  if (value_count == 0) return MB_OK;
  return seg_ids_fill(ex, offsets, segment_count, value_count, ids, nullptr, 0, 0, 0, nullptr);
}

int mb_segmentation_lengths(mb_executor* ex, const uint32_t* offsets, uint64_t segment_count,
                            uint32_t* lengths) {
  MB_TRY(check_exec(ex));
  if (segment_count == 0) return MB_OK;
  lengths_kernel<<<grid_for_n(segment_count), 256, 0, ex->stream>>>(offsets, segment_count, lengths);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mb_segmentation_local_indices(mb_executor* ex, const uint32_t* offsets,
                                  uint64_t segment_count, uint32_t* local, uint64_t value_count) {
  MB_TRY(check_exec(ex));
  if (value_count == 0) return MB_OK;
  local_indices_kernel<<<grid_for_n(value_count), 256, 0, ex->stream>>>(offsets, segment_count,
                                                                       local, value_count);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mb_segmentation_from_segment_ids(mb_executor* ex, const mb_src* ids, uint64_t segment_count,
                                     uint32_t* offsets) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, ids, "segment ids"));
  if (segment_count >= 0xFFFFFFFFull)
    return set_error(MB_ERR_LENGTH_TOO_LARGE, "length does not fit in u32", segment_count + 1);
  if (compute_type(ids->vtype) != MB_U32 || dtype_size(ids->vtype) != 4)
    return set_error(MB_ERR_LAUNCH, "segment ids must be u32");
  const uint64_t n = ids->len;
  const Src s = to_src(*ids);
  if (n > 0) {
    Scratch bad;
    MB_TRY(bad.alloc(ex, 16));
    MB_CUDA(cudaMemsetAsync(bad.ptr, 0, 16, ex->stream));
    validate_ids_kernel<<<grid_for_n(n), 256, 0, ex->stream>>>(s, n, segment_count,
                                                             bad.as<uint32_t>());
    MB_CUDA(cudaGetLastError());
    uint32_t b = 0;
    MB_TRY(read_u32(ex, bad.as<uint32_t>(), &b));
    if (b) return set_error(MB_ERR_INVALID_SEGMENTATION, "segmentation is not a valid ordered partition");
  }
  offsets_from_ids_kernel<<<grid_for_n(segment_count + 1), 256, 0, ex->stream>>>(
      s, n, segment_count, offsets);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int mb_seg_inclusive_scan(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                          uint64_t segment_count, int op, mb_col out) {
  MB_TRY(check_values_out(ex, values, out, values ? values->len : 0));
  // MB_TUNE_SEG: 0 = tile-local scans plus carries (default), 1 = look-back
  const int mode = ex->tune[MB_TUNE_SEG] == 1 ? kScanIncl : kScanInclTiles;
  return seg_entry(ex, values, op, mode, nullptr, out.data, out.dtype, offsets, segment_count,
                   nullptr, nullptr, 0, nullptr);
}

int mb_seg_exclusive_scan(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                          uint64_t segment_count, int op, const void* init, mb_col out) {
  MB_TRY(check_values_out(ex, values, out, values ? values->len : 0));
  if (!init) return set_error(MB_ERR_LAUNCH, "exclusive scan needs an init value");
  const int mode = ex->tune[MB_TUNE_SEG] == 1 ? kScanExcl : kScanExclTiles;
  return seg_entry(ex, values, op, mode, init, out.data, out.dtype, offsets, segment_count,
                   nullptr, nullptr, 0, nullptr);
}

int mb_seg_reduce(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                  uint64_t segment_count, int op, const void* init, mb_col out) {
  MB_TRY(check_values_out(ex, values, out, segment_count));
  if (!init) return set_error(MB_ERR_LAUNCH, "reduce needs an init value");
  if (!op_commutative(op) && op != MB_OP_TAKE_RIGHT && op != MB_OP_TAKE_LEFT)
    return set_error(MB_ERR_LAUNCH, "operator not supported");
  if (values->len == 0) return segment_count ? mb_fill(ex, init, out) : MB_OK;
  // Tuning (MB_TUNE_SEG): 0 = tile-local folds plus the crossing-segment
  // pass (default), 1 = the segmented scan's look-back carried across tiles.
  const int mode = ex->tune[MB_TUNE_SEG] == 1 ? kReduce : kReduceTiles;
  return seg_entry(ex, values, op, mode, init, out.data, out.dtype, offsets, segment_count,
                   nullptr, nullptr, 0, nullptr);
}

int mb_inclusive_scan_by_key(mb_executor* ex, const mb_src* keys, int key_eq,
                             const mb_src* values, int op, mb_col out) {
  MB_TRY(check_values_out(ex, values, out, values ? values->len : 0));
  MB_TRY(check_src(ex, keys, "keys"));
  if (key_eq != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "by-key algorithms take EQUAL");
  if (keys->len != values->len)
    return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", keys->len, values->len);
  return seg_entry(ex, values, op, kScanIncl, nullptr, out.data, out.dtype, nullptr, 0, keys,
                   nullptr, 0, nullptr);
}

int mb_exclusive_scan_by_key(mb_executor* ex, const mb_src* keys, int key_eq,
                             const mb_src* values, int op, const void* init, mb_col out) {
  MB_TRY(check_values_out(ex, values, out, values ? values->len : 0));
  MB_TRY(check_src(ex, keys, "keys"));
  if (key_eq != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "by-key algorithms take EQUAL");
  if (keys->len != values->len)
    return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", keys->len, values->len);
  if (!init) return set_error(MB_ERR_LAUNCH, "exclusive scan needs an init value");
  return seg_entry(ex, values, op, kScanExcl, init, out.data, out.dtype, nullptr, 0, keys,
                   nullptr, 0, nullptr);
}

int mb_reduce_by_key(mb_executor* ex, const mb_src* keys, int key_eq, const mb_src* values,
                     int nvals, const int* ops, const uint64_t* inits, mb_col out_keys,
                     const mb_col* out_values, uint32_t* count_dev, uint32_t* count_host) {
  return mb_reduce_by_key_segmented(ex, keys, key_eq, values, nvals, ops, inits, nullptr, 0,
                                    out_keys, out_values, count_dev, count_host);
}

int mb_reduce_by_key_segmented(mb_executor* ex, const mb_src* keys, int key_eq,
                               const mb_src* values, int nvals, const int* ops,
                               const uint64_t* inits, const uint32_t* offsets,
                               uint64_t segment_count, mb_col out_keys, const mb_col* out_values,
                               uint32_t* count_dev, uint32_t* count_host) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, keys, "keys"));
  MB_TRY(check_col(ex, out_keys, "key output"));
  if (key_eq != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "by-key algorithms take EQUAL");
  if (nvals < 1 || nvals > 12) return set_error(MB_ERR_LAUNCH, "values take 1 to 12 columns");
  const uint64_t n = keys->len;
  if (dtype_size(out_keys.dtype) != dtype_size(keys->vtype))
    return set_error(MB_ERR_LAUNCH, "key output element type differs");
  for (int c = 0; c < nvals; ++c) {
    if (values[c].len != n)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n, values[c].len);
    MB_TRY(check_values_out(ex, &values[c], out_values[c], 0));
  }
  Scratch cnt;
  if (!count_dev) {
    MB_TRY(cnt.alloc(ex, 16));
    count_dev = cnt.as<uint32_t>();
  }
  if (n == 0) {
    MB_CUDA(cudaMemsetAsync(count_dev, 0, 4, ex->stream));
  } else {
    // MB_TUNE_SEG: 0 = tile-local runs plus the crossing-run pass (default),
    // 1 = the segmented scan's look-back carried across tiles
    const int mode = ex->tune[MB_TUNE_SEG] == 1 ? kReduce : kReduceKeysTiles;
    Scratch bases;
    RunBases rb;
    // Shared when every column ends where the keys do (the heads pass reads
    // the column's device length).
    bool same_len = true;
    for (int c = 0; c < nvals; ++c)
      same_len = same_len && (!values[c].len_dev || values[c].len_dev == keys->len_dev);
    if (mode == kReduceKeysTiles && nvals > 1 && same_len) {
      const uint64_t min_tile = SegCfg<uint64_t>::TILE;  // 8-byte values: the smallest
      const uint64_t base_words = ((n + min_tile - 1) / min_tile + 1 + 63) / 64 * 64;
      MB_TRY(bases.alloc(ex, (base_words + n / 32 + 256) * 4));
      rb.ptr = bases.as<uint32_t>();
      rb.bits = rb.ptr + base_words;
    }
    // A constant integer column under ADD (a group-by's count) needs no
    // value pass once the run heads are known: its runs are init + c * length.
    auto counts_runs = [&](int c) {
      const mb_src& v = values[c];
      return rb.ptr && v.kind == MB_SRC_CONSTANT && v.map == MB_UN_IDENTITY &&
             v.dtype == v.vtype && ops[c] == MB_OP_ADD &&
             (v.dtype == MB_U32 || v.dtype == MB_I32 || v.dtype == MB_U64 || v.dtype == MB_I64);
    };
    int primary = 0;  // writes the keys and the run count
    while (primary < nvals && counts_runs(primary)) ++primary;
    if (primary == nvals) primary = 0;
    bool any_const = false;
    for (int k = 0; k < nvals; ++k) {
      const int c = k == 0 ? primary : (k <= primary ? k - 1 : k);
      if (c != primary && counts_runs(c)) {
        any_const = true;
        continue;
      }
      // The keys' device length (a count left by an earlier step) bounds
      // value views that carry none, such as a constant column.
      mb_src v = values[c];
      if (!v.len_dev) v.len_dev = keys->len_dev;
      MB_TRY(seg_entry(ex, &v, ops[c], mode, &inits[c], out_values[c].data,
                       out_values[c].dtype, offsets, segment_count, keys,
                       c == primary ? out_keys.data : nullptr,
                       (int)dtype_size(out_keys.dtype), c == primary ? count_dev : nullptr, &rb));
    }
    if (any_const) {
      const uint64_t tiles = (n + rb.tile - 1) / rb.tile;
      Scratch starts;
      MB_TRY(starts.alloc(ex, n * 4));
      seg_run_starts_kernel<<<(unsigned)tiles, kThreads, 0, ex->stream>>>(
          rb.bits, rb.ptr, rb.tile, n, keys->len_dev, starts.as<uint32_t>());
      MB_CUDA(cudaGetLastError());
      const unsigned g = (unsigned)std::min<uint64_t>((n + kThreads - 1) / kThreads, 148ull * 8);
      for (int c = 0; c < nvals; ++c) {
        if (c == primary || !counts_runs(c)) continue;
        const mb_src& v = values[c];
        if (dtype_size(v.dtype) == 4) {
          const uint32_t init = (uint32_t)inits[c], val = (uint32_t)v.a;
          seg_const_runs_kernel<uint32_t><<<g, kThreads, 0, ex->stream>>>(
              starts.as<uint32_t>(), rb.ptr, rb.tile, n, keys->len_dev, init, val,
              out_values[c].data, out_values[c].dtype);
        } else {
          seg_const_runs_kernel<uint64_t><<<g, kThreads, 0, ex->stream>>>(
              starts.as<uint32_t>(), rb.ptr, rb.tile, n, keys->len_dev, (uint64_t)inits[c],
              (uint64_t)v.a, out_values[c].data, out_values[c].dtype);
        }
        MB_CUDA(cudaGetLastError());
      }
    }
  }
  if (count_host) MB_TRY(read_u32(ex, count_dev, count_host));
  return MB_OK;
}

}  // extern "C"
