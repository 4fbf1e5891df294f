// scan.cu -- single-pass inclusive / exclusive scan with decoupled look-back.
//
// Replaces massively's reduce-then-scan recursion (massively/src/core/
// scan.rs:122-592, 990-1234: a 256-item block scan, a recursive scan of the
// block partials and an add-prefix pass that reads and rewrites the output,
// about 16 bytes of traffic per u32) with one pass that reads the input once
// and writes the output once (8 bytes per u32).
//
// Tile = 256 threads x 4 vectors of 16 bytes (4096 u32 / 2048 u64, 16 KB).
// Each warp owns a contiguous chunk; lane l holds vectors j*32 + l for
// j = 0..3.  The scan runs serially over each vector, then as four warp
// shuffle scans (one per vector row) and a fixed-order fold over the eight
// warp totals.  Warp 0 publishes the tile aggregate and runs the look-back
// (lookback.cuh).  Operand order is preserved everywhere, so
// non-commutative operators (TAKE_LEFT) scan correctly.
//
// Plain aligned columns use the streaming kernel: persistent CTAs (a few per
// SM) take tiles in order from an atomic ticket and keep the next tiles'
// inputs in flight with cp.async.bulk copies into a 3-stage shared-memory
// ring, so HBM keeps streaming while a tile waits in its look-back.  Lazy
// views and device-length inputs use the one-tile-per-CTA kernel.
//
// Floating point: the association is a fixed tree inside the tile and the
// deterministic fold across tiles, so results are identical run to run.

#include "bulk.cuh"
#include "common.cuh"
#include "dispatch.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kLoads = 4;
constexpr int kStages = 3;

template <class T>
struct ScanCfg {
  static constexpr int VEC = 16 / sizeof(T);
  static constexpr int ITEMS = VEC * kLoads;
  static constexpr int WARP_ITEMS = 32 * ITEMS;
  static constexpr int TILE = kThreads * ITEMS;
  static constexpr int TILE_BYTES = TILE * (int)sizeof(T);
};

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

// Scans one tile held in x (warp-striped vectors) into its final inclusive
// (or exclusive) values.  Called by all threads of the CTA.
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

// One tile per CTA: lazy views, device-length inputs, unaligned columns.
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

// Persistent streaming kernel for plain 16-byte-aligned columns.
template <class T, int OP, bool PACKED>
__global__ void __launch_bounds__(kThreads)
    scan_stream_kernel(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                       uint64_t ntiles, ScanParams<T> p, TileState<T, PACKED> st) {
  using C = ScanCfg<T>;
  constexpr int VEC = C::VEC;
  extern __shared__ __align__(128) unsigned char scan_smem[];
  T* ring = reinterpret_cast<T*>(scan_smem);  // kStages tiles
  __shared__ __align__(8) uint64_t bar[kStages];
  __shared__ uint32_t s_tile[kStages];
  __shared__ ScanShared<T> sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Acquires the next tile for ring slot s and starts its copy (thread 0).
  auto issue = [&](int s) {
    const uint32_t t = atomicAdd(p.counter, 1u);
    s_tile[s] = t;
    if (t < ntiles && (uint64_t)(t + 1) * C::TILE <= n) {
      mbar_arrive_expect_tx(&bar[s], C::TILE_BYTES);
      bulk_load(ring + (size_t)s * C::TILE, in + (uint64_t)t * C::TILE, C::TILE_BYTES, &bar[s]);
    }
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bar[s], 1);
    mbar_init_fence();
    for (int s = 0; s < kStages; ++s) issue(s);
  }
  __syncthreads();
  uint32_t parity = 0;
  for (int it = 0;; ++it) {
    const int s = it % kStages;
    const uint64_t tile = s_tile[s];
    if (tile >= ntiles) break;
    const uint64_t tile_base = tile * (uint64_t)C::TILE;
    const bool full = tile_base + C::TILE <= n;
    const uint64_t warp_base = tile_base + (uint64_t)warp * C::WARP_ITEMS;
    T x[kLoads][VEC];
    if (full) {
      if (!mbar_wait(&bar[s], (parity >> s) & 1u)) raise_device_error(p.err, MB_DEV_ERR_LOOKBACK);
      parity ^= 1u << s;
      const T* tb = ring + (size_t)s * C::TILE + warp * C::WARP_ITEMS;
#pragma unroll
      for (int j = 0; j < kLoads; ++j) {
        uint4 u = *reinterpret_cast<const uint4*>(tb + (j * 32 + lane) * VEC);
        memcpy(x[j], &u, 16);
      }
    } else {
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
          x[j][k] = i < n ? in[i] : T(0);
        }
    }
    scan_tile<T, OP, PACKED>(x, tile, p, st, sh);
    if (full) {
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
        store_vec<T>(out, warp_base + (uint64_t)(j * 32 + lane) * VEC, x[j]);
    } else {
#pragma unroll
      for (int j = 0; j < kLoads; ++j)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          const uint64_t i = warp_base + (uint64_t)(j * 32 + lane) * VEC + k;
          if (i < n) out[i] = x[j][k];
        }
    }
    __syncthreads();  // ring slot s and `sh` are free again
    if (threadIdx.x == 0) {
      fence_proxy_async_smem();
      issue(s);
    }
  }
}

int stream_grid(const void* kernel, size_t smem, uint64_t ntiles, int device) {
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
  if (per_sm < 1) per_sm = 1;
  uint64_t g = (uint64_t)sms * per_sm;
  return (int)(g < ntiles ? g : ntiles);
}

template <class T>
int scan_run(mb_executor* ex, const mb_src& in, int op, bool exclusive, const void* init,
             const mb_col& out) {
  using C = ScanCfg<T>;
  constexpr bool PACKED = sizeof(T) == 4;
  const uint64_t cap = in.len;
  if (cap == 0) return MB_OK;
  const uint64_t tiles = (cap + C::TILE - 1) / C::TILE;
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
  const bool plain = src_plain(in, DTypeOf<T>::value) && out.dtype == DTypeOf<T>::value &&
                     ((uintptr_t)in.data % 16 == 0) && ((uintptr_t)out.data % 16 == 0);
  const bool stream = plain && in.len_dev == nullptr;
  const Src s = to_src(in);
  dim3 grid(grid_for(tiles)), block(kThreads);
  const size_t ring = (size_t)kStages * C::TILE_BYTES;
#define MB_SCAN_LAUNCH(OPID)                                                                    \
  do {                                                                                          \
    if (stream) {                                                                               \
      auto k = scan_stream_kernel<T, OPID, PACKED>;                                             \
      MB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring)); \
      const int g = stream_grid((const void*)k, ring, tiles, ex->device);                      \
      k<<<g, kThreads, ring, ex->stream>>>((const T*)in.data, (T*)out.data, cap, tiles, p, st); \
    } else if (plain) {                                                                         \
      scan_kernel<T, OPID, true, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    } else {                                                                                    \
      scan_kernel<T, OPID, false, PACKED><<<grid, block, 0, ex->stream>>>(s, out.data, cap, p, st); \
    }                                                                                           \
  } while (0)
  switch (op) {
    case MB_OP_ADD: MB_SCAN_LAUNCH(MB_OP_ADD); break;
    case MB_OP_MIN: MB_SCAN_LAUNCH(MB_OP_MIN); break;
    case MB_OP_MAX: MB_SCAN_LAUNCH(MB_OP_MAX); break;
    default: MB_SCAN_LAUNCH(kOpDyn); break;
  }
#undef MB_SCAN_LAUNCH
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

}  // namespace
}  // namespace mb

extern "C" {

int mb_inclusive_scan(mb_executor* ex, const mb_src* in, int op, mb_col out) {
  return mb::scan_entry(ex, in, op, false, nullptr, out);
}

int mb_exclusive_scan(mb_executor* ex, const mb_src* in, int op, const void* init, mb_col out) {
  return mb::scan_entry(ex, in, op, true, init, out);
}

}  // extern "C"
