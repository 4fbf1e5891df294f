// select.cu -- stable compaction: vector::copy_where, remove_where and
// partition in one pass over the data.
//
// Replaces massively's selection control (massively/src/core/selection.rs:
// 149-457: a three-kernel scan of the flags into positions, a kernel turning
// positions into compacted source indices, then a gather -- about five
// passes) with one kernel per call: each tile evaluates its flags (the
// stencil view, or a predicate fused onto the column being compacted so the
// column is read once), ranks kept rows with warp ballots (warp-striped
// items, so ranks follow input order), gets the kept-row count of all
// earlier tiles by decoupled look-back and writes every column's kept rows
// to consecutive output positions (on the bulk-copy path a ninth warp runs
// that look-back while the tile lands and the ballots are taken).  The count
// of kept rows stays on the
// device (massively's LogicalExtent::Device, massively/src/core/
// extent.rs:17-36).  partition writes rejected rows after the kept ones,
// both stable; its boundary comes from one reduction of the flags first.

#include <algorithm>

#include "bulk.cuh"
#include "common.cuh"
#include "lookback.cuh"

namespace mb {

int materialize(mb_executor* ex, const mb_src& in, void* dst);

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
constexpr int kMaxCols = 12;

enum SelMode : int { kCopy = 0, kRemove = 1, kPartition = 2 };

struct SelParams {
  int ncols;
  int mode;
  int fused;                  // stencil = predicate `fused_map` over column 0's data
  int fused_map;
  Src cols[kMaxCols];
  void* outs[kMaxCols];
  int esize[kMaxCols];
  Src stencil;
  uint32_t* count_dev;
  const uint32_t* boundary_dev;  // partition: number of kept rows
  uint32_t* counter;
  DevErr err;
};

__device__ __forceinline__ void st_raw(void* p, uint64_t i, int esize, uint64_t bits) {
  switch (esize) {
    case 1: ((uint8_t*)p)[i] = (uint8_t)bits; break;
    case 2: ((uint16_t*)p)[i] = (uint16_t)bits; break;
    case 4: ((uint32_t*)p)[i] = (uint32_t)bits; break;
    default: ((uint64_t*)p)[i] = bits; break;
  }
}

// NC > 0: NC plain 4-byte columns (all of them), flags fused on column 0 or
// a plain u32 stencil; every column's items are loaded before the look-back,
// so their latency overlaps it.  NC = 0: any columns and views, loaded after.
// Only NC = 1 (an unaligned column) and NC = 0 are launched: two or more
// preloaded columns cost more registers than the staged kernel below.
template <int NC>
__global__ void __launch_bounds__(kThreads) select_kernel(SelParams p, uint64_t cap,
                                                          TileState<uint32_t, true> st) {
  constexpr bool FAST = NC > 0;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_wcount[kWarps];
  __shared__ uint32_t s_excl;
  if (threadIdx.x == 0) s_tile = atomicAdd(p.counter, 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t n = src_len(p.cols[0]) < cap ? src_len(p.cols[0]) : cap;
  const uint64_t tile_base = tile * (uint64_t)kTile;
  if (tile_base >= n) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t warp_base = tile_base + (uint64_t)warp * 32 * kItems;
  const uint32_t invert = p.mode == kRemove ? 1u : 0u;

  uint32_t v[FAST ? NC : 1][FAST ? kItems : 1];
  unsigned ballot[kItems];
  uint32_t wcount = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
    const bool valid = i < n;
    uint32_t f = 0;
    if (valid) {
      if constexpr (FAST) {
#pragma unroll
        for (int c = 0; c < NC; ++c) v[c][k] = __ldcs((const uint32_t*)p.cols[c].data + i);
        if (p.fused) f = map_to<uint32_t>(p.fused_map, p.cols[0].dtype, v[0][k]) != 0;
        else f = __ldcs((const uint32_t*)p.stencil.data + i) != 0;
      } else {
        f = src_load<uint32_t>(p.stencil, i) != 0;
      }
      f ^= invert;
    }
    ballot[k] = __ballot_sync(kFull, valid && f);
    wcount += __popc(ballot[k]);
  }
  if (lane == 0) s_wcount[warp] = wcount;
  __syncthreads();
  if (warp == 0) {
    uint32_t c = lane < kWarps ? s_wcount[lane] : 0u;
    uint32_t agg = __reduce_add_sync(kFull, c);
    const Op<uint32_t, MB_OP_ADD> add{MB_OP_ADD};
    uint32_t excl = 0;
    if (tile == 0) {
      if (lane == 0) st.publish(0, kFlagIncl, agg);
    } else {
      if (lane == 0) st.publish(tile, kFlagAgg, agg);
      excl = lookback_exclusive<uint32_t, Op<uint32_t, MB_OP_ADD>, false>(st, tile, add,
                                                                           p.err, 0u);
      if (lane == 0) st.publish(tile, kFlagIncl, excl + agg);
    }
    if (lane == 0) {
      s_excl = excl;
      if (tile_base + kTile >= n && p.count_dev) *p.count_dev = excl + agg;
    }
  }
  __syncthreads();
  uint32_t before = s_excl;  // kept rows before this warp's chunk
  for (int w = 0; w < warp; ++w) before += s_wcount[w];
  const unsigned lt = (1u << lane) - 1u;
  const uint64_t boundary = p.mode == kPartition ? *p.boundary_dev : 0;

  // Per item: output position (or ~0 when the row is not written).
  uint32_t pos[kItems];
  uint32_t run = before;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
    const bool kept = (ballot[k] >> lane) & 1u;
    const uint32_t r = run + __popc(ballot[k] & lt);
    if (kept) pos[k] = r;
    else if (p.mode == kPartition && i < n) pos[k] = (uint32_t)(boundary + i - r);
    else pos[k] = 0xFFFFFFFFu;
    run += __popc(ballot[k]);
  }
  if constexpr (FAST) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      uint32_t* out = (uint32_t*)p.outs[c];
#pragma unroll
      for (int k = 0; k < kItems; ++k)
        if (pos[k] != 0xFFFFFFFFu) out[pos[k]] = v[c][k];
    }
  } else {
    for (int c = 0; c < p.ncols; ++c) {
#pragma unroll 4
      for (int k = 0; k < kItems; ++k) {
        if (pos[k] == 0xFFFFFFFFu) continue;
        const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
        st_raw(p.outs[c], pos[k], p.esize[c], src_load_bits(p.cols[c], i));
      }
    }
  }
}

// Fast path for plain 16-byte-aligned columns: one CTA per 32 KB tile of
// one or two 4-byte columns (plus their u32 stencil unless the predicate is
// fused on column 0).  Thread 0 fetches the tile(s) into shared memory with
// cp.async.bulk, so bytes in flight cost no registers; the CTA counts its
// kept rows from shared memory, runs the look-back, then re-evaluates the
// flags from shared memory and writes the kept rows.
constexpr int kSmemTile = 8192;  // 4-byte items per tile (32 KB)
constexpr int kSmemItems = kSmemTile / kThreads;  // 32 per thread, warp-striped

// PRED >= 0: the fused predicate fixed at compile time (IS_TRUE, IS_FALSE,
// IS_EVEN, IS_ODD on the 32 raw bits of a 4-byte integer column, where the
// sign does not matter); -1 evaluates the run-time map.
template <int PRED>
__device__ __forceinline__ uint32_t fused_flag(int map, int dtype, uint32_t x) {
  if constexpr (PRED == MB_UN_IS_TRUE) return x != 0;
  else if constexpr (PRED == MB_UN_IS_FALSE) return x == 0;
  else if constexpr (PRED == MB_UN_IS_EVEN) return (x & 1u) == 0;
  else if constexpr (PRED == MB_UN_IS_ODD) return (x & 1u) != 0;
  else return map_to<uint32_t>(map, dtype, x) != 0;
}

// Barrier among the first `count` threads (ids 1..15; 0 is __syncthreads).
__device__ __forceinline__ void sel_named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// NCOL (1 or 2) 4-byte data columns; the stencil tile follows them in
// shared memory unless the predicate is fused on column 0.
template <bool FUSED, int PRED, int NCOL>
__global__ void __launch_bounds__(kThreads + 32)
    select_smem_kernel(const uint32_t* __restrict__ in, const uint32_t* __restrict__ in1,
                       const uint32_t* __restrict__ stencil, uint32_t* __restrict__ out,
                       uint32_t* __restrict__ out1, uint64_t n, int fused_map, int in_dtype,
                       uint32_t invert, uint32_t* count_dev, uint32_t* counter, DevErr err,
                       TileState<uint32_t, true> st) {
  constexpr int kCols = NCOL + (FUSED ? 0 : 1);
  constexpr int kTileBytes = kSmemTile * 4;
  extern __shared__ __align__(128) unsigned char sel_smem[];
  uint32_t* buf = reinterpret_cast<uint32_t*>(sel_smem);  // [col][kSmemTile], stencil last
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_wcount[kWarps];
  __shared__ uint32_t s_excl;
  __shared__ uint32_t s_agg;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(counter, 1u);
    s_tile = t;
    mbar_init(&bar, 1);
    mbar_init_fence();
    if ((uint64_t)(t + 1) * kSmemTile <= n) {
      mbar_arrive_expect_tx(&bar, kCols * kTileBytes);
      bulk_load(buf, in + (uint64_t)t * kSmemTile, kTileBytes, &bar);
      if constexpr (NCOL == 2)
        bulk_load(buf + kSmemTile, in1 + (uint64_t)t * kSmemTile, kTileBytes, &bar);
      if constexpr (!FUSED)
        bulk_load(buf + NCOL * kSmemTile, stencil + (uint64_t)t * kSmemTile, kTileBytes, &bar);
    }
  }
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t tile_base = tile * (uint64_t)kSmemTile;
  if (tile_base >= n) return;
  const bool full = tile_base + kSmemTile <= n;
  // The ninth warp runs the look-back from the start, while the tile lands
  // and the compute warps take their ballots.
  uint32_t my_ballot = 0;
  if (warp == kWarps) {
    uint32_t excl = 0;
    if (tile > 0) {
      const Op<uint32_t, MB_OP_ADD> add{MB_OP_ADD};
      excl = lookback_exclusive<uint32_t, Op<uint32_t, MB_OP_ADD>, false>(st, tile, add, err, 0u);
    }
    if (lane == 0) s_excl = excl;
  } else {
    if (full) {
      if (!mbar_wait(&bar, 0)) raise_device_error(err, MB_DEV_ERR_LOOKBACK);
    } else {
      for (int i = threadIdx.x; i < kSmemTile; i += kThreads) {
        const bool ok = tile_base + i < n;
        buf[i] = ok ? in[tile_base + i] : 0u;
        if constexpr (NCOL == 2) buf[kSmemTile + i] = ok ? in1[tile_base + i] : 0u;
        if constexpr (!FUSED) buf[NCOL * kSmemTile + i] = ok ? stencil[tile_base + i] : 0u;
      }
      sel_named_sync(1, kThreads);
    }
    const uint32_t* wv = buf + warp * 32 * kSmemItems;
    const uint32_t* ws = wv + NCOL * kSmemTile;
    auto flag = [&](int k) -> bool {
      if (!full) {
        const uint64_t i = tile_base + (uint64_t)warp * 32 * kSmemItems + k * 32 + lane;
        if (i >= n) return false;
      }
      uint32_t f;
      if constexpr (FUSED) f = fused_flag<PRED>(fused_map, in_dtype, wv[k * 32 + lane]);
      else f = ws[k * 32 + lane] != 0;
      return (f ^ invert) != 0;
    };
    // Each round's ballot is kept by lane k (kSmemItems == 32 rounds), so the
    // write phase reuses it instead of evaluating the predicate again.
    static_assert(kSmemItems == 32, "one ballot per lane");
    uint32_t wcount = 0;
#pragma unroll 8
    for (int k = 0; k < kSmemItems; ++k) {
      const unsigned b = __ballot_sync(kFull, flag(k));
      if (lane == k) my_ballot = b;
      wcount += __popc(b);
    }
    if (lane == 0) s_wcount[warp] = wcount;
    sel_named_sync(1, kThreads);
    if (threadIdx.x == 0) {
      uint32_t agg = 0;
      for (int w = 0; w < kWarps; ++w) agg += s_wcount[w];
      s_agg = agg;
      st.publish(tile, tile == 0 ? kFlagIncl : kFlagAgg, agg);
    }
  }
  __syncthreads();  // s_excl, s_wcount and s_agg are ready
  if (warp == kWarps) return;
  if (threadIdx.x == 0) {
    const uint32_t excl = s_excl, agg = s_agg;
    if (tile > 0) st.publish(tile, kFlagIncl, excl + agg);
    if (tile_base + kSmemTile >= n && count_dev) *count_dev = excl + agg;
  }
  const uint32_t* wv = buf + warp * 32 * kSmemItems;
  uint32_t run = s_excl;
  for (int w = 0; w < warp; ++w) run += s_wcount[w];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll 8
  for (int k = 0; k < kSmemItems; ++k) {
    const unsigned b = __shfl_sync(kFull, my_ballot, k);
    if ((b >> lane) & 1u) {
      const uint32_t o = run + __popc(b & lt);
      out[o] = wv[k * 32 + lane];
      if constexpr (NCOL == 2) out1[o] = wv[kSmemTile + k * 32 + lane];
    }
    run += __popc(b);
  }
}
int select_entry(mb_executor* ex, const mb_src* in, int ncols, const mb_src* stencil,
                 const mb_col* out, uint32_t* count_dev, uint32_t* count_host, int mode,
                 uint32_t* boundary_dev) {
  MB_TRY(check_exec(ex));
  if (ncols < 1 || ncols > kMaxCols) return set_error(MB_ERR_LAUNCH, "1 to 12 columns");
  if (!in || !out) return set_error(MB_ERR_UNBOUND_COLUMN, "missing columns");
  const uint64_t n = in[0].len;
  for (int c = 0; c < ncols; ++c) {
    MB_TRY(check_src(ex, &in[c], "input"));
    MB_TRY(check_col(ex, out[c], "output"));
    if (in[c].len != n) return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n, in[c].len);
    if (out[c].len < n)
      return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out[c].len);
    if (dtype_size(out[c].dtype) != dtype_size(in[c].vtype))
      return set_error(MB_ERR_LAUNCH, "output element type differs from the input's");
  }
  MB_TRY(check_src(ex, stencil, "stencil"));
  if (stencil->len != n)
    return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n, stencil->len);
  Scratch cnt_tmp;
  if (!count_dev) {
    MB_TRY(cnt_tmp.alloc(ex, 16));
    count_dev = cnt_tmp.as<uint32_t>();
  }
  if (n == 0) {
    MB_CUDA(cudaMemsetAsync(count_dev, 0, 4, ex->stream));
  } else {
    SelParams p{};
    p.ncols = ncols;
    p.mode = mode;
    for (int c = 0; c < ncols; ++c) {
      p.cols[c] = to_src(in[c]);
      p.outs[c] = out[c].data;
      p.esize[c] = (int)dtype_size(in[c].vtype);
    }
    p.stencil = to_src(*stencil);
    p.count_dev = count_dev;
    p.boundary_dev = boundary_dev;
    // The predicate reads the same elements as column 0: evaluate it on the
    // loaded values (the column is read once).
    const bool same_data = stencil->kind == MB_SRC_COLUMN && in[0].kind == MB_SRC_COLUMN &&
                           stencil->data == in[0].data && stencil->dtype == in[0].dtype &&
                           in[0].map == MB_UN_IDENTITY;
    p.fused = same_data && stencil->map != MB_UN_IDENTITY;
    p.fused_map = stencil->map;
    // Every column plain, 4 bytes wide, without a device length; the flags
    // fused on column 0 or a plain u32 stencil.
    bool plain4 = ncols <= 2 &&
                  (p.fused || (src_plain(*stencil, MB_U32) && stencil->vtype == MB_U32 &&
                               stencil->dtype == MB_U32 && stencil->len_dev == nullptr));
    for (int c = 0; c < ncols && plain4; ++c)
      plain4 = src_plain(in[c], in[c].vtype) && dtype_size(in[c].vtype) == 4 &&
               in[c].len_dev == nullptr;
    const bool fast = ncols == 1 && plain4;
    const uint64_t tiles = (n + kTile - 1) / kTile;
    Scratch scratch;
    MB_TRY(scratch.alloc(ex, 256 + tiles * 8));
    MB_CUDA(cudaMemsetAsync(scratch.ptr, 0, 256 + tiles * 8, ex->stream));
    p.counter = scratch.as<uint32_t>();
    p.err = DevErr{ex->status_dev, scratch.as<uint32_t>() + 1};
    auto st = TileState<uint32_t, true>::make(scratch.as<char>() + 256, tiles);
    bool aligned = p.fused || (uintptr_t)stencil->data % 16 == 0;
    for (int c = 0; c < ncols; ++c) aligned = aligned && (uintptr_t)in[c].data % 16 == 0;
    TimedLaunch timed(ex, MB_KF_SELECT);
    if (plain4 && aligned && mode != kPartition) {
      // Tiles staged by TMA bulk copies: one per column and one for the stencil.
      static_assert(kSmemTile >= kTile, "the tile-state array is sized for kTile tiles");
      const int cols = ncols + (p.fused ? 0 : 1);
      const size_t smem = (size_t)cols * kSmemTile * 4;
      const uint64_t stiles = (n + kSmemTile - 1) / kSmemTile;
      const uint32_t* in1 = ncols == 2 ? (const uint32_t*)in[1].data : nullptr;
      uint32_t* out1 = ncols == 2 ? (uint32_t*)out[1].data : nullptr;
      auto launch = [&](auto kern) -> int {
        MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(unsigned)stiles, kThreads + 32, smem, ex->stream>>>(
            (const uint32_t*)in[0].data, in1, (const uint32_t*)stencil->data,
            (uint32_t*)out[0].data, out1, n, stencil->map, in[0].dtype,
            mode == kRemove ? 1u : 0u, count_dev, p.counter, p.err, st);
        MB_CUDA(cudaGetLastError());
        return MB_OK;
      };
      const bool int4 = in[0].dtype == MB_U32 || in[0].dtype == MB_I32;
      if (ncols == 2) {
        if (!p.fused) MB_TRY(launch(select_smem_kernel<false, -1, 2>));
        else MB_TRY(launch(select_smem_kernel<true, -1, 2>));
      } else if (!p.fused) MB_TRY(launch(select_smem_kernel<false, -1, 1>));
      else if (int4 && stencil->map == MB_UN_IS_EVEN)
        MB_TRY(launch(select_smem_kernel<true, MB_UN_IS_EVEN, 1>));
      else if (int4 && stencil->map == MB_UN_IS_ODD)
        MB_TRY(launch(select_smem_kernel<true, MB_UN_IS_ODD, 1>));
      else if (int4 && stencil->map == MB_UN_IS_TRUE)
        MB_TRY(launch(select_smem_kernel<true, MB_UN_IS_TRUE, 1>));
      else if (int4 && stencil->map == MB_UN_IS_FALSE)
        MB_TRY(launch(select_smem_kernel<true, MB_UN_IS_FALSE, 1>));
      else MB_TRY(launch(select_smem_kernel<true, -1, 1>));
    } else if (fast) {
      select_kernel<1><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(p, n, st);
    } else {
      select_kernel<0><<<(unsigned)tiles, kThreads, 0, ex->stream>>>(p, n, st);
    }
    MB_CUDA(cudaGetLastError());
  }
  if (count_host) MB_TRY(read_u32(ex, count_dev, count_host));
  return MB_OK;
}

}  // namespace
}  // namespace mb

namespace mb {
namespace {

// Run heads of adjacent-equal items: flags[i] = 1 when i == 0 or item i
// differs from item i-1 (floats compare as values, so NaN differs from
// itself and -0 equals +0, as massively's Equal does).
__global__ void __launch_bounds__(kThreads)
    run_head_flags_kernel(Src keys, uint64_t n, uint32_t* __restrict__ flags) {
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * kThreads) {
    uint32_t h = 1;
    if (i > 0) {
      const uint64_t a = src_load_bits(keys, i - 1), b = src_load_bits(keys, i);
      if (keys.vtype == MB_F32) h = __uint_as_float((uint32_t)a) != __uint_as_float((uint32_t)b);
      else if (keys.vtype == MB_F64)
        h = __longlong_as_double((long long)a) != __longlong_as_double((long long)b);
      else h = a != b;
    }
    flags[i] = h;
  }
}

// unique / unique_by_key: the first row of every run of equal keys, kept by
// the compaction kernel with the run-head flags as its stencil.
int unique_entry(mb_executor* ex, const mb_src* keys, const mb_src* values, int nvals, int equal,
                 const mb_col* out, uint32_t* count_dev, uint32_t* count_host) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, keys, "keys"));
  if (equal != MB_EQUAL) return set_error(MB_ERR_LAUNCH, "unique takes EQUAL");
  const uint64_t n = keys->len;
  MB_TRY(check_len_u32(n));
  Scratch flags;
  MB_TRY(flags.alloc(ex, std::max<uint64_t>(n, 1) * 4));
  if (n) {
    const uint64_t blocks = std::min<uint64_t>((n + kThreads - 1) / kThreads, 148ull * 16);
    run_head_flags_kernel<<<(unsigned)blocks, kThreads, 0, ex->stream>>>(to_src(*keys), n,
                                                                         flags.as<uint32_t>());
    MB_CUDA(cudaGetLastError());
  }
  mb_src st{};
  st.kind = MB_SRC_COLUMN;
  st.dtype = st.vtype = MB_U32;
  st.map = MB_UN_IDENTITY;
  st.data = flags.ptr;
  st.len = n;
  st.owner = keys->owner;
  st.len_dev = keys->len_dev;
  return select_entry(ex, values, nvals, &st, out, count_dev, count_host, kCopy, nullptr);
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_unique(mb_executor* ex, const mb_src* input, int equal, mb_col out, uint32_t* count_dev,
              uint32_t* count_host) {
  return unique_entry(ex, input, input, 1, equal, &out, count_dev, count_host);
}

int mb_unique_by_key(mb_executor* ex, const mb_src* keys, const mb_src* values, int nvals,
                     int equal, const mb_col* out_values, uint32_t* count_dev,
                     uint32_t* count_host) {
  if (values && keys && nvals >= 1)
    for (int c = 0; c < nvals; ++c)
      if (values[c].len != keys->len)
        return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", keys->len,
                         values[c].len);
  return unique_entry(ex, keys, values, nvals, equal, out_values, count_dev, count_host);
}

int mb_copy_where(mb_executor* ex, const mb_src* in, int ncols, const mb_src* stencil,
                  const mb_col* out, uint32_t* count_dev, uint32_t* count_host) {
  return select_entry(ex, in, ncols, stencil, out, count_dev, count_host, kCopy, nullptr);
}

int mb_remove_where(mb_executor* ex, const mb_src* in, int ncols, const mb_src* stencil,
                    const mb_col* out, uint32_t* count_dev, uint32_t* count_host) {
  return select_entry(ex, in, ncols, stencil, out, count_dev, count_host, kRemove, nullptr);
}

int mb_partition(mb_executor* ex, const mb_src* in, int ncols, int pred_col, int pred,
                 const mb_col* out, uint32_t* boundary_dev, uint32_t* boundary_host) {
  MB_TRY(check_exec(ex));
  if (!in || ncols < 1 || ncols > 12 || pred_col < 0 || pred_col >= ncols)
    return set_error(MB_ERR_LAUNCH, "partition: bad column selection");
  if (pred < MB_UN_IS_TRUE || pred > MB_UN_IS_POSITIVE || pred == MB_UN_NEGATE ||
      pred == MB_UN_BIT_NOT || pred == MB_UN_ABS)
    return set_error(MB_ERR_LAUNCH, "partition needs a predicate");
  // The stencil: the predicate over column pred_col, as a view.
  mb_src stencil = in[pred_col];
  if (stencil.map != MB_UN_IDENTITY || stencil.dtype != stencil.vtype) {
    return set_error(MB_ERR_LAUNCH, "partition predicate column must not be a mapped view");
  }
  stencil.map = pred;
  stencil.vtype = MB_U32;
  Scratch bnd;
  if (!boundary_dev) {
    MB_TRY(bnd.alloc(ex, 16));
    boundary_dev = bnd.as<uint32_t>();
  }
  const uint32_t zero = 0;
  MB_TRY(mb_reduce(ex, &stencil, MB_OP_ADD, &zero, boundary_dev, nullptr));
  MB_TRY(select_entry(ex, in, ncols, &stencil, out, nullptr, nullptr, kPartition, boundary_dev));
  if (boundary_host) MB_TRY(read_u32(ex, boundary_dev, boundary_host));
  return MB_OK;
}

}  // extern "C"
