// scan.cu -- single-pass inclusive / exclusive scan with decoupled look-back.
//
// Replaces massively's reduce-then-scan recursion (massively/src/core/
// scan.rs:122-592, 990-1234: a 256-item block scan, a recursive scan of the
// block partials and an add-prefix pass that reads and rewrites the output,
// about 16 bytes of traffic per u32) with one pass that reads the input once
// and writes the output once (8 bytes per u32).
//
// Plain 16-byte-aligned columns (the streaming path): one CTA per 32 KB tile.
// Thread 0 fetches the whole tile into shared memory with one cp.async.bulk
// copy (TMA, completion on an mbarrier), so the bytes in flight do not cost
// registers and many tiles per SM can be loading while others wait in their
// look-back.  The tile is scanned in place in three phases:
//   1. per warp, row by row (a row = 32 lanes x one 16-byte vector): serial
//      scan of the vector, warp shuffle scan of the vector totals, carry from
//      the previous row; the warp-local inclusive values go back to shared
//      memory;
//   2. warp 0 folds the eight warp totals in order, publishes the tile
//      aggregate and runs the look-back (lookback.cuh), giving every warp its
//      prefix;
//   3. every value is combined with its warp prefix on the way out to global
//      memory (16-byte streaming stores).
// Lazy views and device-length inputs use a register-tiled kernel with the
// same arithmetic structure.  Operand order is preserved everywhere, so
// non-commutative operators (TAKE_LEFT) scan correctly; floating-point
// association is a fixed tree inside the tile plus the deterministic fold
// across tiles, so results are identical run to run.

#include <algorithm>
#include <mutex>

#include "bulk.cuh"
#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kLoads = 4;  // register-tiled kernel: vectors per thread
constexpr int kRows = 8;   // smem kernel: vector rows per warp

template <class T>
struct ScanCfg {
  static constexpr int VEC = 16 / sizeof(T);
  static constexpr int ITEMS = VEC * kLoads;
  static constexpr int WARP_ITEMS = 32 * ITEMS;
  static constexpr int TILE = kThreads * ITEMS;
};

template <class T, int R>
struct TileCfg {
  static constexpr int ROWS = R;
  static constexpr int VEC = 16 / sizeof(T);
  static constexpr int WARP_ITEMS = 32 * ROWS * VEC;
  static constexpr int TILE = kWarps * WARP_ITEMS;
  static constexpr int TILE_BYTES = TILE * (int)sizeof(T);
};

// One-tile-per-CTA kernel.  Floats take 64 KB tiles: their deterministic
// look-back folds one aggregate per tile in sequence, so fewer, larger tiles
// shorten that chain.
template <class T>
struct SmemCfg : TileCfg<T, std::is_floating_point<T>::value ? 2 * kRows : kRows> {};

// Alternative shape for the autotuner: 64 KB tiles for every type.
template <class T>
struct BigCfg : TileCfg<T, 2 * kRows> {};

template <class T>
struct ScanParams {
  int op;
  int exclusive;
  int out_dtype;
  T init;
  uint32_t* counter;
  DevErr err;
};

template <class T>
struct ScanShared {
  T warp_total[kWarps];
  T excl;
};

template <class T>
__device__ __forceinline__ void load_vec(const T* p, uint64_t elem, T (&dst)[16 / sizeof(T)]) {
  uint4 u = __ldcs(reinterpret_cast<const uint4*>(p + elem));
  memcpy(dst, &u, 16);
}
template <class T>
__device__ __forceinline__ void store_vec(T* p, uint64_t elem, const T (&src)[16 / sizeof(T)]) {
  uint4 u;
  memcpy(&u, src, 16);
  __stcs(reinterpret_cast<uint4*>(p + elem), u);
}

// Warp 0: folds the warp totals, publishes the tile, runs the look-back and
// writes each warp's prefix (pre[w], has[w]).
template <class T, int OP, bool PACKED>
__device__ __forceinline__ void tile_prefixes(uint64_t tile, const ScanParams<T>& p,
                                              const TileState<T, PACKED>& st, const T* wtot,
                                              T* pre, bool* has) {
  constexpr bool DET = std::is_floating_point<T>::value;
  const Op<T, OP> op{p.op};
  const int lane = threadIdx.x & 31;
  T agg = wtot[0];
#pragma unroll
  for (int w = 1; w < kWarps; ++w) agg = op(agg, wtot[w]);
  T excl = agg;
  if (tile == 0) {
    if (lane == 0) st.publish(0, kFlagIncl, agg);
  } else {
    if (lane == 0) st.publish(tile, kFlagAgg, agg);
    // Floats: the fold-forward look-back (lookback.cuh); its per-tile
    // inclusive prefixes keep the look-back short for these 32 KB tiles.
    excl = lookback_exclusive<T, Op<T, OP>, DET>(st, tile, op, p.err, agg);
    if (lane == 0) st.publish(tile, kFlagIncl, op(excl, agg));
  }
  if (lane == 0) {
    bool h = tile > 0;
    T acc = excl;
    for (int w = 0; w < kWarps; ++w) {
      pre[w] = acc;
      has[w] = h;
      acc = h ? op(acc, wtot[w]) : wtot[w];
      h = true;
    }
  }
}

// Phase 1 of one tile held in `buf`: warp-local inclusive scan, row by row,
// in place; the warp totals go to s_wtot.  (No barrier inside.)
template <class T, int OP, class C>
__device__ __forceinline__ void smem_phase1(T* buf, const ScanParams<T>& p, T* s_wtot) {
  constexpr int VEC = C::VEC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Op<T, OP> op{p.op};
  T* wb = buf + warp * C::WARP_ITEMS;
  T carry = T(0);
#pragma unroll 2
  for (int j = 0; j < C::ROWS; ++j) {
    T v[VEC];
    uint4 u = *reinterpret_cast<const uint4*>(wb + (j * 32 + lane) * VEC);
    memcpy(v, &u, 16);
#pragma unroll
    for (int k = 1; k < VEC; ++k) v[k] = op(v[k - 1], v[k]);
    T g = v[VEC - 1];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T o = shfl_up(g, d);
      if (lane >= d) g = op(o, g);
    }
    const T rowtot = shfl_idx(g, 31);
    const T ge = shfl_up(g, 1);
    bool h = j > 0;
    T pj = carry;
    if (lane > 0) { pj = h ? op(pj, ge) : ge; h = true; }
    if (h) {
#pragma unroll
      for (int k = 0; k < VEC; ++k) v[k] = op(pj, v[k]);
    }
    memcpy(&u, v, 16);
    *reinterpret_cast<uint4*>(wb + (j * 32 + lane) * VEC) = u;
    carry = j > 0 ? op(carry, rowtot) : rowtot;
  }
  if (lane == 0) s_wtot[warp] = carry;
}

// Phase 3: every value combined with its warp prefix on the way out; `full`
// tiles store 16-byte vectors, the last, partial tile item by item.
template <class T, int OP, class C>
__device__ __forceinline__ void smem_phase3(const T* buf, uint64_t tile, uint64_t n, bool full,
                                            T* __restrict__ out, const ScanParams<T>& p,
                                            const T* s_pre, const bool* s_has) {
  constexpr int VEC = C::VEC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Op<T, OP> op{p.op};
  const T* wb = buf + warp * C::WARP_ITEMS;
  const T pre = s_pre[warp];
  const bool has = s_has[warp];
  const uint64_t wg = tile * (uint64_t)C::TILE + (uint64_t)warp * C::WARP_ITEMS;
#pragma unroll 2
  for (int j = 0; j < C::ROWS; ++j) {
    const int li = (j * 32 + lane) * VEC;  // warp-local index of item 0
    T v[VEC];
    uint4 u = *reinterpret_cast<const uint4*>(wb + li);
    memcpy(v, &u, 16);
    T o[VEC];
    if (p.exclusive) {
      // Inclusive value of the item before each item, then init op it.
      bool h0 = has;
      T prev0 = pre;
      if (li > 0) {
        prev0 = has ? op(pre, wb[li - 1]) : wb[li - 1];
        h0 = true;
      }
      o[0] = h0 ? op(p.init, prev0) : p.init;
#pragma unroll
      for (int k = 1; k < VEC; ++k) o[k] = op(p.init, has ? op(pre, v[k - 1]) : v[k - 1]);
    } else {
#pragma unroll
      for (int k = 0; k < VEC; ++k) o[k] = has ? op(pre, v[k]) : v[k];
    }
    if (full) {
      store_vec<T>(out, wg + li, o);
    } else {
#pragma unroll
      for (int k = 0; k < VEC; ++k)
        if (wg + li + k < n) out[wg + li + k] = o[k];
    }
  }
}

// Phases 1-3 of one tile, warp 0 running the look-back between them.
template <class T, int OP, bool PACKED, class C>
__device__ __forceinline__ void smem_tile(T* buf, uint64_t tile, uint64_t n, bool full,
                                          T* __restrict__ out, const ScanParams<T>& p,
                                          const TileState<T, PACKED>& st, T* s_wtot, T* s_pre,
                                          bool* s_has) {
  smem_phase1<T, OP, C>(buf, p, s_wtot);
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tile_prefixes<T, OP, PACKED>(tile, p, st, s_wtot, s_pre, s_has);
  __syncthreads();
  smem_phase3<T, OP, C>(buf, tile, n, full, out, p, s_pre, s_has);
}

template <class T, int OP, bool PACKED, class C>
__global__ void __launch_bounds__(kThreads)
    scan_smem_kernel(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                     ScanParams<T> p, TileState<T, PACKED> st) {
  extern __shared__ __align__(128) unsigned char scan_smem[];
  T* buf = reinterpret_cast<T*>(scan_smem);
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t s_tile;
  __shared__ T s_wtot[kWarps];
  __shared__ T s_pre[kWarps];
  __shared__ bool s_has[kWarps];

  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(p.counter, 1u);
    s_tile = t;
    mbar_init(&bar, 1);
    mbar_init_fence();
    if ((uint64_t)(t + 1) * C::TILE <= n) {
      mbar_arrive_expect_tx(&bar, C::TILE_BYTES);
      bulk_load(buf, in + (uint64_t)t * C::TILE, C::TILE_BYTES, &bar);
    }
  }
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t tile_base = tile * (uint64_t)C::TILE;
  if (tile_base >= n) return;
  const bool full = tile_base + C::TILE <= n;
  if (full) {
    if (!mbar_wait(&bar, 0)) raise_device_error(p.err, MB_DEV_ERR_LOOKBACK);
  } else {
    for (int i = threadIdx.x; i < C::TILE; i += kThreads)
      buf[i] = tile_base + i < n ? in[tile_base + i] : T(0);
    __syncthreads();
  }
  smem_tile<T, OP, PACKED, C>(buf, tile, n, full, out, p, st, s_wtot, s_pre, s_has);
}

// Barrier among the first `count` threads (ids 1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// The same tile scan with a ninth warp that runs the look-back while the
// bulk load lands and the eight compute warps scan their rows, so the
// look-back's L2 round trips leave the tile's critical path: by the time the
// tile's own aggregate is known its exclusive prefix usually is too.  The
// compute warps publish the aggregate after phase 1 and the inclusive prefix
// after joining the look-back warp.  (The look-back never needs the tile's
// own aggregate; the fold order is the same as warp 0's, so float results
// are unchanged.)
template <class T, int OP, bool PACKED, class C>
__global__ void __launch_bounds__(kThreads + 32)
    scan_smem_lb_kernel(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                        ScanParams<T> p, TileState<T, PACKED> st) {
  constexpr bool DET = std::is_floating_point<T>::value;
  extern __shared__ __align__(128) unsigned char scan_smem[];
  T* buf = reinterpret_cast<T*>(scan_smem);
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t s_tile;
  __shared__ T s_wtot[kWarps];
  __shared__ T s_pre[kWarps];
  __shared__ bool s_has[kWarps];
  __shared__ T s_excl;

  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(p.counter, 1u);
    s_tile = t;
    mbar_init(&bar, 1);
    mbar_init_fence();
    if ((uint64_t)(t + 1) * C::TILE <= n) {
      mbar_arrive_expect_tx(&bar, C::TILE_BYTES);
      bulk_load(buf, in + (uint64_t)t * C::TILE, C::TILE_BYTES, &bar);
    }
  }
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t tile_base = tile * (uint64_t)C::TILE;
  if (tile_base >= n) return;
  const bool full = tile_base + C::TILE <= n;
  const Op<T, OP> op{p.op};
  if (warp == kWarps) {
    // the look-back warp
    T excl = T(0);
    if (tile > 0) excl = lookback_exclusive<T, Op<T, OP>, DET>(st, tile, op, p.err, T(0));
    if ((threadIdx.x & 31) == 0) s_excl = excl;
  } else {
    if (full) {
      if (!mbar_wait(&bar, 0)) raise_device_error(p.err, MB_DEV_ERR_LOOKBACK);
    } else {
      for (int i = threadIdx.x; i < C::TILE; i += kThreads)
        buf[i] = tile_base + i < n ? in[tile_base + i] : T(0);
      named_sync(1, kThreads);
    }
    smem_phase1<T, OP, C>(buf, p, s_wtot);
    named_sync(1, kThreads);
    if (threadIdx.x == 0) {
      T agg = s_wtot[0];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) agg = op(agg, s_wtot[w]);
      st.publish(tile, tile == 0 ? kFlagIncl : kFlagAgg, agg);
    }
  }
  __syncthreads();  // s_excl and s_wtot are ready
  if (warp == kWarps) return;
  if (threadIdx.x == 0) {
    const T excl = s_excl;
    bool h = tile > 0;
    T acc = excl;
    T agg = s_wtot[0];
    for (int w = 0; w < kWarps; ++w) {
      s_pre[w] = acc;
      s_has[w] = h;
      acc = h ? op(acc, s_wtot[w]) : s_wtot[w];
      h = true;
      if (w > 0) agg = op(agg, s_wtot[w]);
    }
    if (tile > 0) st.publish(tile, kFlagIncl, op(excl, agg));
  }
  named_sync(1, kThreads);
  smem_phase3<T, OP, C>(buf, tile, n, full, out, p, s_pre, s_has);
}

// Register-tiled scan of one tile held in x (warp-striped vectors) into its
// final inclusive (or exclusive) values.  Called by all threads of the CTA.
template <class T, int OP, bool PACKED>
__device__ __forceinline__ void scan_tile(T (&x)[kLoads][16 / sizeof(T)], uint64_t tile,
                                          const ScanParams<T>& p,
                                          const TileState<T, PACKED>& st, ScanShared<T>& sh) {
  constexpr int VEC = 16 / sizeof(T);
  constexpr bool DET = std::is_floating_point<T>::value;
  const Op<T, OP> op{p.op};
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

#pragma unroll
  for (int j = 0; j < kLoads; ++j)
#pragma unroll
    for (int k = 1; k < VEC; ++k) x[j][k] = op(x[j][k - 1], x[j][k]);

  T ge[kLoads];
  T rowtot[kLoads];
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
  if (lane == 0) sh.warp_total[warp] = rp[kLoads - 1];
  __syncthreads();

  if (warp == 0) {
    T agg = sh.warp_total[0];
#pragma unroll
    for (int w = 1; w < kWarps; ++w) agg = op(agg, sh.warp_total[w]);
    if (tile == 0) {
      if (lane == 0) st.publish(0, kFlagIncl, agg);
    } else {
      if (lane == 0) st.publish(tile, kFlagAgg, agg);
      T excl = lookback_exclusive<T, Op<T, OP>, DET>(st, tile, op, p.err, agg);
      if (lane == 0) {
        st.publish(tile, kFlagIncl, op(excl, agg));
        sh.excl = excl;
      }
    }
  }
  __syncthreads();

  bool has_pre = tile > 0;
  T pre = has_pre ? sh.excl : T(0);
  for (int w = 0; w < warp; ++w) {
    T t = sh.warp_total[w];
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

  if (p.exclusive) {
#pragma unroll
    for (int j = 0; j < kLoads; ++j) {
      T up = shfl_up(y[j][VEC - 1], 1);
      T wrap = shfl_idx(j > 0 ? y[j - 1][VEC - 1] : y[0][VEC - 1], 31);
      bool h0;
      T prev0;
      if (lane > 0) { prev0 = up; h0 = true; }
      else if (j > 0) { prev0 = wrap; h0 = true; }
      else { prev0 = pre; h0 = has_pre; }
#pragma unroll
      for (int k = VEC - 1; k >= 1; --k) x[j][k] = op(p.init, y[j][k - 1]);
      x[j][0] = h0 ? op(p.init, prev0) : p.init;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
#pragma unroll
      for (int k = 0; k < VEC; ++k) x[j][k] = y[j][k];
  }
}

// One tile per CTA in registers: lazy views, device-length inputs, unaligned
// columns.
template <class T, int OP, bool PLAIN, bool PACKED>
__global__ void __launch_bounds__(kThreads)
    scan_kernel(Src in, void* out, uint64_t cap, ScanParams<T> p, TileState<T, PACKED> st) {
  using C = ScanCfg<T>;
  constexpr int VEC = C::VEC;
  __shared__ uint32_t s_tile;
  __shared__ ScanShared<T> sh;

  if (threadIdx.x == 0) s_tile = atomicAdd(p.counter, 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t n = in.len_dev ? min((uint64_t)*in.len_dev, cap) : cap;
  const uint64_t tile_base = tile * (uint64_t)C::TILE;
  if (tile_base >= n) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t warp_base = tile_base + (uint64_t)warp * C::WARP_ITEMS;
  const bool full = tile_base + C::TILE <= n;

  T x[kLoads][VEC];
  if (PLAIN && full) {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
      load_vec<T>((const T*)in.data, warp_base + (uint64_t)(j * 32 + lane) * VEC, x[j]);
  } else {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
#pragma unroll
      for (int k = 0; k < VEC; ++k) {
        const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
        if (i < n) {
          if constexpr (PLAIN) x[j][k] = ((const T*)in.data)[i];
          else x[j][k] = src_load<T>(in, i);
        } else {
          x[j][k] = T(0);
        }
      }
  }
  scan_tile<T, OP, PACKED>(x, tile, p, st, sh);
  if (PLAIN && full) {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
      store_vec<T>((T*)out, warp_base + (uint64_t)(j * 32 + lane) * VEC, x[j]);
  } else {
#pragma unroll
    for (int j = 0; j < kLoads; ++j)
#pragma unroll
      for (int k = 0; k < VEC; ++k) {
        const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
        if (i < n) {
          if constexpr (PLAIN) ((T*)out)[i] = x[j][k];
          else st_cast<T>(p.out_dtype, out, i, x[j][k]);
        }
      }
  }
}

template <class T>
int scan_run(mb_executor* ex, const mb_src& in, int op, bool exclusive, const void* init,
             const mb_col& out) {
  constexpr bool PACKED = sizeof(T) == 4;
  const uint64_t cap = in.len;
  if (cap == 0) return MB_OK;
  const bool plain = src_plain(in, DTypeOf<T>::value) && out.dtype == DTypeOf<T>::value &&
                     ((uintptr_t)in.data % 16 == 0) && ((uintptr_t)out.data % 16 == 0);
  const bool smem_path = plain && in.len_dev == nullptr;
  const int shape = smem_path ? std::max(0, ex->tune[MB_TUNE_SCAN]) : 0;
  // shapes: 0 = look-back warp, default tile; 1 = warp 0 runs the look-back,
  // default tile; 2 = look-back warp, 64 KB tiles
  const uint64_t tile_items = !smem_path ? ScanCfg<T>::TILE
                              : shape == 2 ? BigCfg<T>::TILE : SmemCfg<T>::TILE;
  const uint64_t tiles = (cap + tile_items - 1) / tile_items;
  Scratch scratch;
  const size_t state_bytes = TileState<T, PACKED>::bytes(tiles);
  MB_TRY(scratch.alloc(ex, 256 + state_bytes));
  MB_CUDA(cudaMemsetAsync(scratch.ptr, 0, 256 + state_bytes, ex->stream));
  ScanParams<T> p{};
  p.op = op;
  p.exclusive = exclusive ? 1 : 0;
  p.out_dtype = out.dtype;
  p.init = T(0);
  if (exclusive) memcpy(&p.init, init, sizeof(T));
  p.counter = scratch.as<uint32_t>();
  p.err = DevErr{ex->status_dev, scratch.as<uint32_t>() + 1};
  auto st = TileState<T, PACKED>::make(scratch.as<char>() + 256, tiles);
  const Src s = to_src(in);
  dim3 grid(grid_for(tiles)), block(kThreads);
  const size_t smem = shape == 2 ? BigCfg<T>::TILE_BYTES : SmemCfg<T>::TILE_BYTES;
#define MB_SCAN_SMEM(OPID, CFG)                                                             \
  do {                                                                                      \
    if (smem > 48 * 1024)                                                                   \
      MB_CUDA(cudaFuncSetAttribute(scan_smem_kernel<T, OPID, PACKED, CFG>,                  \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    scan_smem_kernel<T, OPID, PACKED, CFG><<<grid, block, smem, ex->stream>>>(              \
        (const T*)in.data, (T*)out.data, cap, p, st);                                       \
  } while (0)
#define MB_SCAN_LB(OPID, CFG)                                                               \
  do {                                                                                      \
    if (smem > 48 * 1024)                                                                   \
      MB_CUDA(cudaFuncSetAttribute(scan_smem_lb_kernel<T, OPID, PACKED, CFG>,               \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    scan_smem_lb_kernel<T, OPID, PACKED, CFG><<<grid, kThreads + 32, smem, ex->stream>>>(   \
        (const T*)in.data, (T*)out.data, cap, p, st);                                       \
  } while (0)
#define MB_SCAN_LAUNCH(OPID)                                                                    \
  do {                                                                                          \
    if (smem_path) {                                                                            \
      if (shape == 1)                                                                           \
        MB_SCAN_SMEM(OPID, SmemCfg<T>);                                                         \
      else if (shape == 2)                                                                      \
        MB_SCAN_LB(OPID, BigCfg<T>);                                                            \
      else                                                                                      \
        MB_SCAN_LB(OPID, SmemCfg<T>);                                                           \
    } else if (plain) {                                                                         \
      scan_kernel<T, OPID, true, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    } else {                                                                                    \
      scan_kernel<T, OPID, false, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    }                                                                                           \
  } while (0)
  TimedLaunch timed(ex, MB_KF_SCAN);
  switch (op) {
    case MB_OP_ADD: MB_SCAN_LAUNCH(MB_OP_ADD); break;
    case MB_OP_MIN: MB_SCAN_LAUNCH(MB_OP_MIN); break;
    case MB_OP_MAX: MB_SCAN_LAUNCH(MB_OP_MAX); break;
    default: MB_SCAN_LAUNCH(kOpDyn); break;
  }
#undef MB_SCAN_LAUNCH
#undef MB_SCAN_SMEM
#undef MB_SCAN_LB
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int scan_entry(mb_executor* ex, const mb_src* in, int op, bool exclusive, const void* init,
               const mb_col& out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, in, "input"));
  MB_TRY(check_col(ex, out, "output"));
  const int ct = compute_type(in->vtype);
  if (compute_type(out.dtype) != ct)
    return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  if (!op_valid_for(op, ct)) return set_error(MB_ERR_LAUNCH, "operator not defined for this type");
  if (out.len < in->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", in->len, out.len);
  if (exclusive && !init) return set_error(MB_ERR_LAUNCH, "exclusive scan needs an init value");
  // A narrow init is widened like the elements are.
  uint64_t init_wide = 0;
  if (exclusive) {
    int dt = in->vtype;
    uint64_t raw = 0;
    memcpy(&raw, init, dtype_size(dt));
    switch (dt) {
      case MB_I8: init_wide = (uint64_t)(int64_t)(int8_t)raw; break;
      case MB_I16: init_wide = (uint64_t)(int64_t)(int16_t)raw; break;
      default: init_wide = raw; break;
    }
  }
  MB_DISPATCH_CTYPE(ct, scan_run, ex, *in, op, exclusive, &init_wide, out);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

// ------------------------------------------------ allocation-free scan ----
//
// For callers that cannot allocate device memory during a call.  The
// look-back scratch (tile ticket, abort word, tile states) lives in this
// fixed array instead of the executor's pool.  The largest call it admits
// is 2^26 8-byte elements on the register-tiled path: 32,768 tiles, whose
// states take 655,616 bytes, plus two group-state arrays of 12,544 bytes
// and the 256-byte header, 680,960 bytes in all; the array is 1 MiB.  The
// code checks the exact size of every call against the array.
constexpr size_t kNoAllocBytes = 1u << 20;
constexpr uint64_t kNoAllocMax4 = 1ull << 27;  // 4-byte elements
constexpr uint64_t kNoAllocMax8 = 1ull << 26;  // 8-byte elements

static __device__ __align__(256) unsigned char g_scan_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the array on `device`, looked up once per device with
// that device current (host code may not use the symbol itself: on the host
// it names a host-side stand-in, not device memory).
int noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= kNoAllocMaxDevices)
    return set_error(MB_ERR_LAUNCH, "device ordinal out of range for the allocation-free scan");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[device]) {
    int prev = 0;
    MB_CUDA(cudaGetDevice(&prev));
    if (prev != device) MB_CUDA(cudaSetDevice(device));
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scan_noalloc_scratch);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(scan scratch)");
    g_noalloc_addr[device] = ptr;
  }
  *out = g_noalloc_addr[device];
  return MB_OK;
}

template <class T>
int scan_noalloc_run(mb_executor* ex, const mb_src& in, int op, const mb_col& out) {
  constexpr bool PACKED = sizeof(T) == 4;
  const uint64_t cap = in.len;
  if (cap == 0) return MB_OK;
  if (cap > (sizeof(T) == 4 ? kNoAllocMax4 : kNoAllocMax8))
    return set_error(MB_ERR_LENGTH_TOO_LARGE,
                     "allocation-free scan takes at most 2^27 4-byte or 2^26 8-byte elements", cap);
  const bool plain = src_plain(in, DTypeOf<T>::value) && out.dtype == DTypeOf<T>::value &&
                     ((uintptr_t)in.data % 16 == 0) && ((uintptr_t)out.data % 16 == 0);
  const bool smem_path = plain && in.len_dev == nullptr;
  const uint64_t tile_items = smem_path ? SmemCfg<T>::TILE : ScanCfg<T>::TILE;
  const uint64_t tiles = (cap + tile_items - 1) / tile_items;
  const size_t need = 256 + TileState<T, PACKED>::bytes(tiles);
  if (need > kNoAllocBytes)
    return set_error(MB_ERR_LENGTH_TOO_LARGE, "allocation-free scan: input too large", cap);
  void* scratch = nullptr;
  MB_TRY(noalloc_scratch(ex->device, &scratch));
  // The array keeps the previous call's contents: clear the ticket, the
  // abort word and the tile states this call uses.
  MB_CUDA(cudaMemsetAsync(scratch, 0, need, ex->stream));
  ScanParams<T> p{};
  p.op = op;
  p.exclusive = 0;
  p.out_dtype = out.dtype;
  p.init = T(0);
  p.counter = (uint32_t*)scratch;
  p.err = DevErr{ex->status_dev, (uint32_t*)scratch + 1};
  auto st = TileState<T, PACKED>::make((char*)scratch + 256, tiles);
  const Src s = to_src(in);
  dim3 grid(grid_for(tiles)), block(kThreads);
  const size_t smem = SmemCfg<T>::TILE_BYTES;
#define MB_SCAN_NOALLOC_LAUNCH(OPID)                                                            \
  do {                                                                                          \
    if (smem_path) {                                                                            \
      if (smem > 48 * 1024)                                                                     \
        MB_CUDA(cudaFuncSetAttribute(scan_smem_lb_kernel<T, OPID, PACKED, SmemCfg<T>>,          \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));  \
      scan_smem_lb_kernel<T, OPID, PACKED, SmemCfg<T>>                                          \
          <<<grid, kThreads + 32, smem, ex->stream>>>((const T*)in.data, (T*)out.data, cap, p,  \
                                                      st);                                      \
    } else if (plain) {                                                                         \
      scan_kernel<T, OPID, true, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    } else {                                                                                    \
      scan_kernel<T, OPID, false, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    }                                                                                           \
  } while (0)
  switch (op) {
    case MB_OP_ADD: MB_SCAN_NOALLOC_LAUNCH(MB_OP_ADD); break;
    case MB_OP_MIN: MB_SCAN_NOALLOC_LAUNCH(MB_OP_MIN); break;
    case MB_OP_MAX: MB_SCAN_NOALLOC_LAUNCH(MB_OP_MAX); break;
    default: MB_SCAN_NOALLOC_LAUNCH(kOpDyn); break;
  }
#undef MB_SCAN_NOALLOC_LAUNCH
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int scan_noalloc_entry(mb_executor* ex, const mb_src* in, int op, const mb_col& out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, in, "input"));
  MB_TRY(check_col(ex, out, "output"));
  const int ct = compute_type(in->vtype);
  if (compute_type(out.dtype) != ct)
    return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  if (!op_valid_for(op, ct)) return set_error(MB_ERR_LAUNCH, "operator not defined for this type");
  if (out.len < in->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", in->len, out.len);
  MB_DISPATCH_CTYPE(ct, scan_noalloc_run, ex, *in, op, out);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

}  // namespace
}  // namespace mb

extern "C" {

int mb_inclusive_scan(mb_executor* ex, const mb_src* in, int op, mb_col out) {
  return mb::scan_entry(ex, in, op, false, nullptr, out);
}

int mb_inclusive_scan_noalloc(mb_executor* ex, const mb_src* in, int op, mb_col out) {
  return mb::scan_noalloc_entry(ex, in, op, out);
}

int mb_exclusive_scan(mb_executor* ex, const mb_src* in, int op, const void* init, mb_col out) {
  return mb::scan_entry(ex, in, op, true, init, out);
}

}  // extern "C"
