// radix.cu -- onesweep LSD radix sort (keys, or keys + one value column).
//
// Replaces massively's block-local 4-bit radix passes (massively/src/core/
// radix.rs:120-546: per pass a block split of 256 items, a per-bucket
// histogram prefix, a one-thread bucket-offset kernel and a scatter of a
// permutation, then a final gather of the values; 8 passes for u32) with the
// onesweep scheme:
//
//   1. histogram:  one read of the keys builds the 256-bin histograms of
//                  every 8-bit digit at once;
//   2. plan:       one block scans them into global digit offsets, marks
//                  passes whose digit is the same for every key (skipped) and
//                  assigns the ping-pong buffers so the last active pass lands
//                  in the output -- on the device, so nothing synchronises and
//                  the whole sort can be captured in a CUDA graph;
//   3. onesweep:   per active digit, one kernel: every tile ranks its keys
//                  stably (warp match on the digit, per-warp counters bumped
//                  with shared-memory atomics), publishes its 256 digit
//                  counts, stages its keys in tile-sorted order in shared
//                  memory, obtains the counts of all earlier tiles by a
//                  per-digit decoupled look-back (overlapped with the value
//                  loads), and writes keys and values so consecutive threads
//                  store consecutive addresses of each digit run.
//
// Keys are ordered by massively's radix encodings (massively/src/core/
// radix.rs:46-89): unsigned as is, signed with the sign bit flipped, floats
// in total order (negative: all bits inverted; otherwise sign bit set).  The
// encoding only selects digits; keys move in their original bits.
//
// Byte model (8-bit digits): n*sk + 2*P*n*(sk+sv) for P digit passes.

#include <algorithm>

#include "bulk.cuh"
#include "common.cuh"
#include "lookback.cuh"

namespace mb {
namespace {

constexpr int kRadixBits = 8;
constexpr int kBins = 1 << kRadixBits;
constexpr int kHistThreads = 512;
constexpr int kHistUnroll = 4;  // 16-byte vectors per lane per chunk

// Look-back status word of one (tile, digit): the flag (none / aggregate /
// inclusive) in the top two bits, the digit's count below.  32-bit words
// hold counts below 2^30; a sort of 2^30 items or more uses 64-bit words, so
// every length up to 2^32 - 1 sorts.
template <class SW>
struct DigitStatus {
  static constexpr int kShift = 8 * (int)sizeof(SW) - 2;
  static constexpr SW kMask = ((SW)1 << kShift) - 1;

  __device__ __forceinline__ static SW load(const SW* p) {
    if constexpr (sizeof(SW) == 8) return ld_relaxed_u64(p);
    else return ld_relaxed_u32(p);
  }
  __device__ __forceinline__ static void store(SW* p, uint32_t flag, SW count) {
    const SW w = ((SW)flag << kShift) | (count & kMask);
    if constexpr (sizeof(SW) == 8) st_relaxed_u64(p, w);
    else st_relaxed_u32(p, w);
  }

  // Publishes digit d's count of `tile` (inclusive for tile 0).
  __device__ __forceinline__ static void publish(SW* status, uint64_t tile, int d, SW count) {
    store(status + tile * kBins + d, tile == 0 ? kFlagIncl : kFlagAgg, count);
  }

  // Decoupled look-back of digit d, eight predecessors per step, bounded:
  // the count of digit d in all tiles before `tile`; publishes this tile's
  // inclusive count.  After a wait that ran out it records the failure and
  // returns the partial sum (never more than the true count).
  __device__ __forceinline__ static SW lookback(SW* status, uint64_t tile, int d, SW tile_count,
                                                const DevErr& err) {
    SW excl = 0;
    if (tile == 0) return 0;
    constexpr int kBatch = 8;
    SpinGuard guard(err.abort);
    int64_t t = (int64_t)tile - 1;  // next predecessor to account for
    bool failed = false, done = false;
    while (!done) {
      SW w[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; ++j)
        w[j] = t - j >= 0 ? load(status + (uint64_t)(t - j) * kBins + d)
                          : ((SW)kFlagIncl << kShift);
      int used = 0;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (done || used < j) break;
        const uint32_t f = (uint32_t)(w[j] >> kShift);
        if (f == kFlagNone) break;
        excl += w[j] & kMask;
        ++used;
        if (f == kFlagIncl) done = true;
      }
      t -= used;
      if (!done && used < kBatch && guard.expired()) {
        failed = true;
        break;
      }
    }
    if (failed) raise_device_error(err, MB_DEV_ERR_LOOKBACK);
    store(status + tile * kBins + d, kFlagIncl, excl + tile_count);
    return excl;
  }
};

// Keys travel as their raw unsigned bits (K = uint32_t / uint64_t) and are
// never held in floating-point registers; ENC (enc_bits, common.cuh) selects
// massively's encoding of the element type they came from.
template <class K, int ENC>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
  return (uint32_t)((enc_bits<K, ENC>(k) >> shift) & (kBins - 1));
}

// Buffer plan of one sort, filled on the device by the plan kernel.
struct PassPlan {
  const void* in_k[8];
  void* out_k[8];
  const void* in_v[8];
  void* out_v[8];
  uint32_t active[8];
  uint32_t copy_only;
  uint32_t n;  // items sorted: the capacity, or the device length when one is given
  uint32_t pad_[2];
};

// ----------------------------------------------------------- histogram --

// All passes' digit counts in one read of the keys.  Each warp takes chunks
// of kHistUnroll x 32 16-byte vectors (all loads issued before any count),
// and counts into its own sub-histogram (COPIES per block, so warps of one
// block rarely contend on a bin).  Digit positions where every key of the
// chunk agrees (the high bytes of small keys, constant columns) are found
// with one OR-reduction per chunk and counted by one add, instead of 32-way
// conflicting atomics.  Keys that are not 16-byte aligned, and the tail after
// the last full chunk, go one key per thread.
template <class K, int ENC, int PASSES>
__global__ void __launch_bounds__(kHistThreads, 2)
    radix_histogram_kernel(const K* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ n_dev,
                           uint32_t* __restrict__ hist) {
  if (n_dev && *n_dev < n) n = *n_dev;
  constexpr int COPIES = 16 / PASSES;
  constexpr int KPV = 16 / (int)sizeof(K);      // keys per 16-byte vector
  constexpr int KPL = KPV * kHistUnroll;        // keys per lane per chunk
  constexpr uint64_t KPW = 32ull * KPL;         // keys per warp chunk
  __shared__ uint32_t sh[COPIES][PASSES][kBins];
  for (int i = threadIdx.x; i < COPIES * PASSES * kBins; i += kHistThreads)
    (&sh[0][0][0])[i] = 0;
  __syncthreads();
  uint32_t(*h)[kBins] = sh[(threadIdx.x >> 5) % COPIES];
  const uint32_t lane = lane_id();
  const uint64_t warps = (uint64_t)gridDim.x * (kHistThreads / 32);
  const uint64_t gw = (uint64_t)blockIdx.x * (kHistThreads / 32) + (threadIdx.x >> 5);
  const uint64_t chunks = ((uintptr_t)keys & 15) == 0 ? n / KPW : 0;
  for (uint64_t c = gw; c < chunks; c += warps) {
    const uint4* src = reinterpret_cast<const uint4*>(keys + c * KPW);
    uint4 v[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) v[u] = __ldcs(src + u * 32 + lane);
    K k[KPL];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) {
      const K* kv = reinterpret_cast<const K*>(&v[u]);
#pragma unroll
      for (int j = 0; j < KPV; ++j) k[u * KPV + j] = enc_bits<K, ENC>(kv[j]);
    }
    K any = 0, all = ~(K)0;
#pragma unroll
    for (int j = 0; j < KPL; ++j) {
      any |= k[j];
      all &= k[j];
    }
    const K ref = __shfl_sync(kFull, k[0], 0);
    const K diff = (any ^ all) | (k[0] ^ ref);
    K wdiff = (K)__reduce_or_sync(kFull, (uint32_t)diff);
    if constexpr (sizeof(K) == 8)
      wdiff |= (K)__reduce_or_sync(kFull, (uint32_t)((uint64_t)diff >> 32)) << 32;
#pragma unroll
    for (int p = 0; p < PASSES; ++p) {
      const int s = p * kRadixBits;
      if (((wdiff >> s) & (kBins - 1)) == 0) {  // warp-uniform
        if (lane == 0) atomicAdd(&h[p][(uint32_t)(ref >> s) & (kBins - 1)], (uint32_t)KPW);
      } else {
#pragma unroll
        for (int j = 0; j < KPL; ++j) atomicAdd(&h[p][(uint32_t)(k[j] >> s) & (kBins - 1)], 1u);
      }
    }
  }
  const uint64_t stride = (uint64_t)gridDim.x * kHistThreads;
  for (uint64_t i = chunks * KPW + (uint64_t)blockIdx.x * kHistThreads + threadIdx.x; i < n;
       i += stride) {
    const K u = enc_bits<K, ENC>(__ldcs(keys + i));
#pragma unroll
    for (int p = 0; p < PASSES; ++p)
      atomicAdd(&h[p][(uint32_t)(u >> (p * kRadixBits)) & (kBins - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < PASSES * kBins; i += kHistThreads) {
    uint32_t c = 0;
#pragma unroll
    for (int cp = 0; cp < COPIES; ++cp) c += (&sh[cp][0][0])[i];
    if (c) atomicAdd(hist + i, c);
  }
}

// The same counts with lane-private bins, for up to four passes (keys of up
// to 32 bits): bin b of pass p is counted at word (p * kBins + b) * 32 + lane,
// so the 32 atomics of one warp instruction always fall in 32 different
// banks and never on one address -- no bank conflicts, whatever the digits.
// 32 KB of counters per pass; one 1024-thread block per SM.
constexpr int kHistLaneThreads = 1024;

template <class K, int ENC, int PASSES>
__global__ void __launch_bounds__(kHistLaneThreads, 1)
    radix_histogram_lanes_kernel(const K* __restrict__ keys, uint64_t n,
                                 const uint32_t* __restrict__ n_dev, uint32_t* __restrict__ hist) {
  static_assert(PASSES <= 4, "lane-private bins for up to four passes");
  if (n_dev && *n_dev < n) n = *n_dev;
  constexpr int KPV = 16 / (int)sizeof(K);
  constexpr int KPL = KPV * kHistUnroll;
  constexpr uint64_t KPW = 32ull * KPL;
  extern __shared__ __align__(16) uint32_t lanes_sh[];  // [PASSES][kBins][32]
  for (int i = threadIdx.x; i < PASSES * kBins * 32; i += kHistLaneThreads) lanes_sh[i] = 0;
  __syncthreads();
  const uint32_t lane = lane_id();
  uint32_t* mine = lanes_sh + lane;
  const uint64_t warps = (uint64_t)gridDim.x * (kHistLaneThreads / 32);
  const uint64_t gw = (uint64_t)blockIdx.x * (kHistLaneThreads / 32) + (threadIdx.x >> 5);
  const uint64_t chunks = ((uintptr_t)keys & 15) == 0 ? n / KPW : 0;
  for (uint64_t c = gw; c < chunks; c += warps) {
    const uint4* src = reinterpret_cast<const uint4*>(keys + c * KPW);
    uint4 v[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) v[u] = __ldcs(src + u * 32 + lane);
    K k[KPL];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) {
      const K* kv = reinterpret_cast<const K*>(&v[u]);
#pragma unroll
      for (int j = 0; j < KPV; ++j) k[u * KPV + j] = enc_bits<K, ENC>(kv[j]);
    }
    K any = 0, all = ~(K)0;
#pragma unroll
    for (int j = 0; j < KPL; ++j) {
      any |= k[j];
      all &= k[j];
    }
    const K ref = __shfl_sync(kFull, k[0], 0);
    const K diff = (any ^ all) | (k[0] ^ ref);
    const K wdiff = (K)__reduce_or_sync(kFull, (uint32_t)diff);
#pragma unroll
    for (int p = 0; p < PASSES; ++p) {
      const int s = p * kRadixBits;
      if (((wdiff >> s) & (kBins - 1)) == 0) {  // warp-uniform
        if (lane == 0)
          atomicAdd(mine + (p * kBins + ((uint32_t)(ref >> s) & (kBins - 1))) * 32, (uint32_t)KPW);
      } else {
#pragma unroll
        for (int j = 0; j < KPL; ++j)
          atomicAdd(mine + (p * kBins + ((uint32_t)(k[j] >> s) & (kBins - 1))) * 32, 1u);
      }
    }
  }
  const uint64_t stride = (uint64_t)gridDim.x * kHistLaneThreads;
  for (uint64_t i = chunks * KPW + (uint64_t)blockIdx.x * kHistLaneThreads + threadIdx.x; i < n;
       i += stride) {
    const K u = enc_bits<K, ENC>(__ldcs(keys + i));
#pragma unroll
    for (int p = 0; p < PASSES; ++p)
      atomicAdd(mine + (p * kBins + ((uint32_t)(u >> (p * kRadixBits)) & (kBins - 1))) * 32, 1u);
  }
  __syncthreads();
  // fold the 32 lane copies of each bin (rotated start: no bank conflicts)
  for (int i = threadIdx.x; i < PASSES * kBins; i += kHistLaneThreads) {
    uint32_t c = 0;
#pragma unroll 8
    for (int l = 0; l < 32; ++l) c += lanes_sh[i * 32 + ((l + (int)lane) & 31)];
    if (c) atomicAdd(hist + i, c);
  }
}

// ---------------------------------------------------------------- plan --

// One block of 256 threads: exclusive digit offsets per pass (in place over
// `hist`), trivial-pass detection and the buffer assignment.
__global__ void __launch_bounds__(kBins)
    radix_plan_kernel(uint32_t* __restrict__ hist, int passes, uint64_t n,
                      const uint32_t* __restrict__ n_dev, PassPlan* plan, const void* in_k,
                      void* out_k, void* tmp_k, const void* in_v, void* out_v, void* tmp_v) {
  if (n_dev && *n_dev < n) n = *n_dev;
  if (threadIdx.x == 0) plan->n = (uint32_t)n;
  __shared__ uint32_t s_scan[kBins];
  __shared__ uint32_t s_trivial[8];
  const int d = threadIdx.x;
  for (int p = 0; p < passes; ++p) {
    const uint32_t c = hist[p * kBins + d];
    if (d == 0) s_trivial[p] = 0;
    __syncthreads();
    if ((uint64_t)c == n) s_trivial[p] = 1;
    s_scan[d] = c;
    __syncthreads();
    for (int off = 1; off < kBins; off <<= 1) {
      uint32_t v = d >= off ? s_scan[d - off] : 0;
      __syncthreads();
      s_scan[d] += v;
      __syncthreads();
    }
    hist[p * kBins + d] = s_scan[d] - c;  // exclusive offset
    __syncthreads();
  }
  if (d == 0) {
    int m = 0;
    for (int p = 0; p < passes; ++p) m += s_trivial[p] ? 0 : 1;
    plan->copy_only = (m == 0 && n > 0) ? 1u : 0u;
    int i = 0;  // index of the active pass among active passes
    const void* cur_k = in_k;
    const void* cur_v = in_v;
    for (int p = 0; p < passes; ++p) {
      if (s_trivial[p]) {
        plan->active[p] = 0;
        continue;
      }
      ++i;
      // The i-th active pass writes the output when (m - i) is even, else
      // the temporary, so the last active pass lands in the output.
      const bool to_out = ((m - i) % 2) == 0;
      void* nk = to_out ? out_k : tmp_k;
      void* nv = to_out ? out_v : tmp_v;
      plan->active[p] = 1;
      plan->in_k[p] = cur_k;
      plan->out_k[p] = nk;
      plan->in_v[p] = cur_v;
      plan->out_v[p] = nv;
      cur_k = nk;
      cur_v = nv;
    }
    for (int p = passes; p < 8; ++p) plan->active[p] = 0;
    if (plan->copy_only) {
      plan->in_k[0] = in_k;
      plan->out_k[0] = out_k;
      plan->in_v[0] = in_v;
      plan->out_v[0] = out_v;
    }
  }
}

// ------------------------------------------------------------ onesweep --

template <class K, class V, int THREADS, int ITEMS>
struct OnesweepSmem {
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  uint32_t warp_cnt[WARPS][kBins];  // per-warp digit counts, then exclusive prefixes
  uint32_t tile_start[kBins];       // exclusive prefix of the tile's digit counts
  uint32_t delta[kBins];            // global base - tile start, per digit
  uint32_t wsum[kBins / 32];        // digit-scan warp totals
  uint32_t tile_id;
  K keys[TILE];
  V vals[std::is_same<V, uint8_t>::value ? 1 : TILE];
};

// V = uint8_t means "keys only"; SW the look-back status word (DigitStatus).
template <class K, int ENC, class V, int THREADS, int ITEMS, class SW>
__global__ void __launch_bounds__(THREADS, (THREADS <= 256 ? 4 : 2))
    radix_onesweep_kernel(const PassPlan* __restrict__ plan, int pass, uint64_t n,
                          const uint32_t* __restrict__ digit_offsets, SW* __restrict__ status,
                          uint32_t* __restrict__ counter, DevErr err) {
  constexpr bool KEYS_ONLY = std::is_same<V, uint8_t>::value;
  using S = OnesweepSmem<K, V, THREADS, ITEMS>;
  if (plan->n < n) n = plan->n;  // device length
  constexpr int WARPS = S::WARPS;
  constexpr int TILE = S::TILE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;

  if (plan->copy_only) {
    // Every digit is constant: the stable order is the input order.
    if (pass != 0) return;
    const K* ik = (const K*)plan->in_k[0];
    K* ok = (K*)plan->out_k[0];
    const V* iv = (const V*)plan->in_v[0];
    V* ov = (V*)plan->out_v[0];
    for (uint64_t i = blockIdx.x * (uint64_t)THREADS + tid; i < n;
         i += (uint64_t)gridDim.x * THREADS) {
      ok[i] = ik[i];
      if constexpr (!KEYS_ONLY) ov[i] = iv[i];
    }
    return;
  }
  if (!plan->active[pass]) return;
  const K* __restrict__ in_k = (const K*)plan->in_k[pass];
  K* __restrict__ out_k = (K*)plan->out_k[pass];
  const V* __restrict__ in_v = (const V*)plan->in_v[pass];
  V* __restrict__ out_v = (V*)plan->out_v[pass];
  const int shift = pass * kRadixBits;

  if (tid == 0) sm.tile_id = atomicAdd(counter, 1u);
  for (int i = tid; i < WARPS * kBins; i += THREADS) (&sm.warp_cnt[0][0])[i] = 0;
  __syncthreads();
  const uint64_t tile = sm.tile_id;
  const uint64_t tile_base = tile * (uint64_t)TILE;
  const uint64_t warp_base = tile_base + (uint64_t)warp * 32 * ITEMS;

  // Warp-striped loads: item k of lane l is at warp_base + k*32 + l, so the
  // rounds below visit the keys in input order (stability).
  K key[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
    key[k] = i < n ? __ldcs(in_k + i) : K(0);
  }
  auto digit_k = [&](int k) -> uint32_t {
    const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
    return i < n ? digit_of<K, ENC>(key[k], shift) : (uint32_t)kBins;  // kBins: never counted
  };

  // Stable rank within the warp: peers with the same digit in a round are
  // ordered by lane; rounds are in input order.  The leader's atomic add on
  // the warp's digit counter returns the count of earlier rounds; a warp
  // issues its atomics in program order, so rounds apply in order.
  uint32_t rank[ITEMS];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t d = digit_k(k);
    const unsigned peers = __match_any_sync(kFull, d);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader && d < kBins) base = atomicAdd(&sm.warp_cnt[warp][d], (uint32_t)__popc(peers));
    rank[k] = __shfl_sync(kFull, base, leader) + __popc(peers & lt_mask);
  }
  __syncthreads();

  // Per digit (thread d): exclusive prefix over warps and the tile count,
  // published at once; then the tile-local exclusive scan over digits.
  uint32_t tile_count = 0;
  if (tid < kBins) {
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
      const uint32_t c = sm.warp_cnt[w][tid];
      sm.warp_cnt[w][tid] = tile_count;
      tile_count += c;
    }
    DigitStatus<SW>::publish(status, tile, tid, tile_count);
    uint32_t incl = tile_count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += o;
    }
    if (lane == 31) sm.wsum[warp] = incl;
    sm.tile_start[tid] = incl - tile_count;  // warp-local exclusive
  }
  __syncthreads();
  if (tid < kBins) {
    uint32_t add = 0;
    for (int w = 0; w < warp; ++w) add += sm.wsum[w];
    sm.tile_start[tid] += add;
  }
  __syncthreads();

  // Stage keys at their tile-sorted positions; keep the positions.
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t d = digit_k(k);
    if (d < kBins) {
      const uint32_t pos = sm.tile_start[d] + sm.warp_cnt[warp][d] + rank[k];
      rank[k] = pos;
      sm.keys[pos] = key[k];
    }
  }
  // Value loads go out before the look-back so their latency overlaps it.
  V val[KEYS_ONLY ? 1 : ITEMS];
  if constexpr (!KEYS_ONLY) {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
      val[k] = i < n ? __ldcs(in_v + i) : V(0);
    }
  }

  // Decoupled look-back, one digit per thread.
  if (tid < kBins) {
    const uint32_t excl = (uint32_t)DigitStatus<SW>::lookback(status, tile, tid, tile_count, err);
    sm.delta[tid] = digit_offsets[pass * kBins + tid] + excl - sm.tile_start[tid];
  }
  if constexpr (!KEYS_ONLY) {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint64_t i = warp_base + (uint64_t)k * 32 + lane;
      if (i < n) sm.vals[rank[k]] = val[k];
    }
  }
  __syncthreads();

  const uint64_t valid = n - tile_base < (uint64_t)TILE ? n - tile_base : (uint64_t)TILE;
  // Coalesced write-out: position i of the sorted tile goes to delta[d] + i.
#pragma unroll 4
  for (int i = tid; i < (int)valid; i += THREADS) {
    const K kk = sm.keys[i];
    const uint32_t d = digit_of<K, ENC>(kk, shift);
    const uint32_t o = sm.delta[d] + (uint32_t)i;
    if (o >= n) {  // only reachable after a failed look-back
      raise_device_error(err, MB_DEV_ERR_BOUNDS);
      continue;
    }
    __stcs(out_k + o, kk);
    if constexpr (!KEYS_ONLY) __stcs(out_v + o, sm.vals[i]);
  }
}

template <class K, class V, int THREADS, int ITEMS>
size_t onesweep_smem() {
  return sizeof(OnesweepSmem<K, V, THREADS, ITEMS>);
}

// ------------------------------------------------------- onesweep (TMA) --
//
// The same pass for 16-byte-aligned buffers: thread 0 fetches the tile's
// keys and values into shared memory with cp.async.bulk at CTA start (one
// DRAM round trip for both, no load instructions, no registers held while
// they are in flight); ranking reads the keys from shared memory, and the
// tile is permuted in place through registers.
//
// Ranking, per warp round of 32 keys: the lanes holding the same digit
// (peers) come from a per-warp table of 256 lane masks in shared memory --
// each lane ORs its bit into its digit's word and reads the word back --
// instead of eight ballots per key.  NT tables are used in turn: with one,
// a round needs three warp barriers (set, read, clear); with three, a
// round's words are cleared two rounds later, so one barrier per round
// suffices.  Then the lowest peer of each round adds the peer count to the
// warp's per-digit counter, in round order (one warp's atomics on one
// address apply in issue order, which keeps the ranks stable), and
// broadcasts the old count to its peers.

// NT = 0: peers come from ballots on the digit bits (no mask table).
template <class K, class V, int THREADS, int ITEMS, int NT>
struct OnesweepTmaSmem {
  static constexpr bool KEYS_ONLY = std::is_same<V, uint8_t>::value;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  K keys[TILE];                       // 16-byte aligned: bulk-copy target
  V vals[KEYS_ONLY ? 16 : TILE];
  // Slot kBins takes the empty items of a partial tile.  With NT = 0 the
  // one-word `mask` array is unused.
  uint32_t mask[NT <= 0 ? 1 : NT][NT <= 0 ? 1 : WARPS][NT <= 0 ? 1 : kBins + 1];
  uint32_t warp_cnt[WARPS][kBins + 1];
  uint32_t tile_start[kBins];
  uint32_t delta[kBins];
  uint32_t wsum[kBins / 32];
  uint32_t tile_id;
  uint32_t pad_;
  uint64_t bar;
};

template <class K, int ENC, class V, int THREADS, int ITEMS, int NT, bool P64, bool FULL, class SW>
__device__ __forceinline__ void onesweep_tile(OnesweepTmaSmem<K, V, THREADS, ITEMS, NT>& sm,
                                              const uint32_t tile, const uint32_t valid,
                                              const int pass, const uint32_t n,
                                              const uint32_t* __restrict__ digit_offsets,
                                              SW* __restrict__ status, const DevErr err,
                                              K* __restrict__ out_k, V* __restrict__ out_v) {
  using S = OnesweepTmaSmem<K, V, THREADS, ITEMS, NT>;
  constexpr bool KEYS_ONLY = S::KEYS_ONLY;
  constexpr int WARPS = S::WARPS;
  static_assert(S::TILE <= 65536, "tile positions must fit 16 bits");
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int shift = pass * kRadixBits;
  // Warp-striped items: item k of lane l is tile position
  // warp*32*ITEMS + k*32 + l, so the rounds follow input order.
  const uint32_t wl = (uint32_t)warp * 32 * ITEMS + lane;
  const uint32_t below_me = (1u << lane) - 1u;
  const uint32_t me = 1u << lane;

  uint32_t rd[ITEMS];  // digit << 16, then | rank
  if constexpr (NT <= 0) {
    // Peers from one ballot per digit bit: a lane's peers are the lanes
    // whose every bit agrees with its own.  No shared memory is touched for
    // them, so the ranking costs no bank conflicts (ALU work instead).  Bit 8
    // marks the empty items of a partial tile (digit kBins), which then form
    // a group of their own.  Per round the lowest peer (the leader) adds the
    // group's size to the warp's digit counter right away; the rounds'
    // atomics are issued in round order, which keeps the ranks stable.  Each
    // item keeps, packed in one register: digit (bits 20..28), leader lane
    // (15..19), peers below it (10..14) and, on the leader, the counter's
    // old value (0..9; a warp ranks at most 512 items).
    static_assert(32 * ITEMS <= 1024, "a warp's counter value must fit 10 bits");
    constexpr int NB = FULL ? kRadixBits : kRadixBits + 1;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint32_t li = wl + k * 32;
      const uint32_t d =
          (FULL || li < valid) ? digit_of<K, ENC>(sm.keys[li], shift) : (uint32_t)kBins;
      uint32_t eq = kFull;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(kFull, bit);
        eq &= bit ? bal : ~bal;
      }
      const uint32_t below = (uint32_t)__popc(eq & below_me);
      uint32_t base = 0;
      if (below == 0) base = atomicAdd(&sm.warp_cnt[warp][d], (uint32_t)__popc(eq));
      rd[k] = (d << 20) | ((uint32_t)(__ffs(eq) - 1) << 15) | (below << 10) | base;
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint32_t base = __shfl_sync(kFull, rd[k] & 0x3FFu, (rd[k] >> 15) & 31u);
      rd[k] = ((rd[k] >> 20) << 16) | (base + ((rd[k] >> 10) & 31u));
    }
  } else {
    uint32_t peers[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint32_t li = wl + k * 32;
      const uint32_t d =
          (FULL || li < valid) ? digit_of<K, ENC>(sm.keys[li], shift) : (uint32_t)kBins;
      rd[k] = d << 16;
      uint32_t* m = sm.mask[k % NT][warp];
      atomicOr(&m[d], me);
      __syncwarp();
      peers[k] = m[d];
      if constexpr (NT == 1) {
        __syncwarp();
        m[d] = 0;
        __syncwarp();
      } else {
        static_assert(NT >= 3, "a round's words are cleared two rounds before reuse");
        if (k > 0) sm.mask[(k - 1) % NT][warp][rd[k - 1] >> 16] = 0;
      }
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      uint32_t base = 0;
      if ((peers[k] & below_me) == 0)
        base = atomicAdd(&sm.warp_cnt[warp][rd[k] >> 16], (uint32_t)__popc(peers[k]));
      rd[k] |= base;
    }
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint32_t base = __shfl_sync(kFull, rd[k] & 0xFFFFu, __ffs(peers[k]) - 1);
      rd[k] = (rd[k] & 0xFFFF0000u) | (base + __popc(peers[k] & below_me));
    }
  }
  K key[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t li = wl + k * 32;
    key[k] = (FULL || li < valid) ? sm.keys[li] : K(0);
  }
  __syncthreads();  // counts final; every key of the tile is in registers

  // Per digit: the warps' counts to exclusive offsets, the tile's count
  // (published at once for the successors' look-back), and the tile-wide
  // exclusive offsets.
  uint32_t tile_count = 0;
  if (tid < kBins) {
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
      const uint32_t c = sm.warp_cnt[w][tid];
      sm.warp_cnt[w][tid] = tile_count;
      tile_count += c;
    }
    DigitStatus<SW>::publish(status, tile, tid, tile_count);
    uint32_t incl = tile_count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t o = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += o;
    }
    if (lane == 31) sm.wsum[warp] = incl;
    sm.tile_start[tid] = incl - tile_count;
  }
  __syncthreads();
  if (tid < kBins) {
    uint32_t start = sm.tile_start[tid];
    for (int w = 0; w < warp; ++w) start += sm.wsum[w];
    sm.tile_start[tid] = start;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) sm.warp_cnt[w][tid] += start;  // warp's first tile position
  }
  __syncthreads();

  // Keys to their tile-sorted positions (in place: all were read above).
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) rd[k] = (rd[k] & 0xFFFFu) + sm.warp_cnt[warp][rd[k] >> 16];
  // P64: 4-byte keys and values are staged as one 64-bit (value, key) word
  // per item over the keys + values area (one store and one load per item
  // instead of two each).
  static_assert(!P64 || (sizeof(K) == 4 && sizeof(V) == 4), "P64 stages 4-byte pairs");
  uint64_t* stage64 = reinterpret_cast<uint64_t*>(sm.keys);
  V val[KEYS_ONLY ? 1 : ITEMS];
  if constexpr (P64) {
    // Two tile positions (below 2^16) per register, to hold keys, values and
    // positions together in registers.
    static_assert(ITEMS % 2 == 0, "positions are packed in pairs");
    uint32_t pos2[ITEMS / 2];
#pragma unroll
    for (int k = 0; k < ITEMS; k += 2) pos2[k / 2] = rd[k] | (rd[k + 1] << 16);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
      const uint32_t li = wl + k * 32;
      val[k] = (FULL || li < valid) ? sm.vals[li] : V(0);
    }
    __syncthreads();  // every key and value of the tile is in registers
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (FULL || wl + k * 32 < valid)
        stage64[(pos2[k / 2] >> (16 * (k & 1))) & 0xFFFFu] =
            ((uint64_t)(uint32_t)val[k] << 32) | (uint32_t)key[k];
  } else {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (FULL || wl + k * 32 < valid) sm.keys[rd[k]] = key[k];
    if constexpr (!KEYS_ONLY) {
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        const uint32_t li = wl + k * 32;
        val[k] = (FULL || li < valid) ? sm.vals[li] : V(0);
      }
    }
  }

  // Decoupled look-back, one digit per thread.
  if (tid < kBins) {
    const uint32_t excl = (uint32_t)DigitStatus<SW>::lookback(status, tile, tid, tile_count, err);
    sm.delta[tid] = digit_offsets[pass * kBins + tid] + excl - sm.tile_start[tid];
  }
  if constexpr (!KEYS_ONLY && !P64) {
    __syncthreads();  // every original value is in registers
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (FULL || wl + k * 32 < valid) sm.vals[rd[k]] = val[k];
  }
  __syncthreads();

  // Write-out, fully unrolled so the shared-memory reads of all ITEMS
  // positions are in flight together.
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
    const uint32_t i = (uint32_t)r * THREADS + tid;
    if (!FULL && i >= valid) break;
    K kk;
    V vv{};
    if constexpr (P64) {
      const uint64_t kv = stage64[i];
      kk = (K)(uint32_t)kv;
      vv = (V)(uint32_t)(kv >> 32);
    } else {
      kk = sm.keys[i];
    }
    const uint32_t o = sm.delta[digit_of<K, ENC>(kk, shift)] + i;
    if (o >= n) {  // only reachable after a failed look-back
      raise_device_error(err, MB_DEV_ERR_BOUNDS);
      continue;
    }
    __stcs(out_k + o, kk);
    if constexpr (P64) __stcs(out_v + o, vv);
    else if constexpr (!KEYS_ONLY) __stcs(out_v + o, sm.vals[i]);
  }
}

// MINB: CTAs per SM the registers are budgeted for (0 = by tile shape);
// SW: the look-back status word (DigitStatus).
template <class K, int ENC, class V, int THREADS, int ITEMS, int NT, bool P64, int MINB, class SW>
__global__ void __launch_bounds__(THREADS, MINB > 0 ? MINB
                                          : NT <= 1 ? (THREADS >= 1024 ? 1 : THREADS >= 384 ? 2 : 4)
                                                    : 3)
    radix_onesweep_tma_kernel(const PassPlan* __restrict__ plan, int pass, uint32_t n,
                              const uint32_t* __restrict__ digit_offsets,
                              SW* __restrict__ status, uint32_t* __restrict__ counter,
                              DevErr err) {
  using S = OnesweepTmaSmem<K, V, THREADS, ITEMS, NT>;
  constexpr bool KEYS_ONLY = S::KEYS_ONLY;
  constexpr int WARPS = S::WARPS;
  constexpr int TILE = S::TILE;
  if (plan->n < n) n = plan->n;  // device length
  extern __shared__ __align__(128) unsigned char smem_tma[];
  S& sm = *reinterpret_cast<S*>(smem_tma);
  const int tid = threadIdx.x;

  if (plan->copy_only) {
    if (pass != 0) return;
    const K* ik = (const K*)plan->in_k[0];
    K* ok = (K*)plan->out_k[0];
    const V* iv = (const V*)plan->in_v[0];
    V* ov = (V*)plan->out_v[0];
    for (uint64_t i = blockIdx.x * (uint64_t)THREADS + tid; i < n;
         i += (uint64_t)gridDim.x * THREADS) {
      ok[i] = ik[i];
      if constexpr (!KEYS_ONLY) ov[i] = iv[i];
    }
    return;
  }
  if (!plan->active[pass]) return;
  const K* __restrict__ in_k = (const K*)plan->in_k[pass];
  const V* __restrict__ in_v = (const V*)plan->in_v[pass];

  if (tid == 0) {
    const uint32_t t = atomicAdd(counter, 1u);
    sm.tile_id = t;
    mbar_init(&sm.bar, 1);
    mbar_init_fence();
    if ((uint64_t)t * TILE + TILE <= n) {
      constexpr uint32_t kb = TILE * sizeof(K);
      constexpr uint32_t vb = KEYS_ONLY ? 0 : TILE * sizeof(V);
      mbar_arrive_expect_tx(&sm.bar, kb + vb);
      bulk_load(sm.keys, in_k + (uint64_t)t * TILE, kb, &sm.bar);
      if constexpr (!KEYS_ONLY) bulk_load(sm.vals, in_v + (uint64_t)t * TILE, vb, &sm.bar);
    }
  }
  if constexpr (NT <= 0) {
    for (int i = tid; i < WARPS * (kBins + 1); i += THREADS) (&sm.warp_cnt[0][0])[i] = 0;
  } else {
    for (int i = tid; i < (NT + 1) * WARPS * (kBins + 1); i += THREADS)
      (&sm.mask[0][0][0])[i] = 0;  // mask tables and warp_cnt (adjacent)
  }
  __syncthreads();
  const uint32_t tile = sm.tile_id;
  const uint32_t tile_base = tile * TILE;
  if (tile_base >= n) return;
  const uint32_t valid = n - tile_base < (uint32_t)TILE ? n - tile_base : (uint32_t)TILE;
  K* out_k = (K*)plan->out_k[pass];
  V* out_v = (V*)plan->out_v[pass];
  if (valid == TILE) {
    if (!mbar_wait(&sm.bar, 0)) raise_device_error(err, MB_DEV_ERR_LOOKBACK);
    onesweep_tile<K, ENC, V, THREADS, ITEMS, NT, P64, true, SW>(sm, tile, valid, pass, n,
                                                               digit_offsets, status, err, out_k,
                                                               out_v);
  } else {
    for (uint32_t i = tid; i < valid; i += THREADS) {
      sm.keys[i] = in_k[tile_base + i];
      if constexpr (!KEYS_ONLY) sm.vals[i] = in_v[tile_base + i];
    }
    __syncthreads();
    onesweep_tile<K, ENC, V, THREADS, ITEMS, NT, P64, false, SW>(sm, tile, valid, pass, n,
                                                                digit_offsets, status, err, out_k,
                                                                out_v);
  }
}

// Tile configurations of the onesweep kernel (MB_TUNE_RADIX).
struct RadixCfg {
  int threads, items;
  const char* text;
};
constexpr RadixCfg kRadixCfgs[] = {
    {256, 16, "onesweep 256 threads x 16 keys, one peer-mask table (three warp barriers per round)"},
    {256, 16, "onesweep 256 threads x 16 keys, three peer-mask tables (one warp barrier per round)"},
    {512, 16, "onesweep 512 threads x 16 keys (8192-key tiles), one peer-mask table"},
    {256, 12, "onesweep 256 threads x 12 keys (3072-key tiles), three peer-mask tables"},
    {1024, 16, "onesweep 1024 threads x 16 keys (16384-key tiles), one peer-mask table"},
    {384, 16, "onesweep 384 threads x 16 keys (6144-key tiles), one peer-mask table"},
    {512, 16, "onesweep 512 threads x 16 keys, 4-byte pairs staged as one 64-bit word"},
    {512, 12, "onesweep 512 threads x 12 keys (6144-key tiles), 64-bit pair staging"},
    {384, 16, "onesweep 384 threads x 16 keys (6144-key tiles), 64-bit pair staging"},
    {384, 16, "onesweep 384 threads x 16 keys, 64-bit pair staging, ballot peers, 3 CTAs/SM"},
};
constexpr int kRadixDefault = 0;    // 64-bit keys or values
constexpr int kRadixDefault32 = 6;  // 32-bit keys, values of at most 32 bits

// SW: the look-back status word, 32-bit below 2^30 items, else 64-bit.
template <class K, int ENC, class V, int THREADS, int ITEMS, int NT = 1, bool P64 = false,
          int MINB = 0, class SW = uint32_t>
int onesweep_sort_cfg(mb_executor* ex, const K* in_k, const V* in_v, K* out_k, V* out_v,
                      uint64_t n, const uint32_t* n_dev) {
  constexpr int PASSES = (int)sizeof(K);
  constexpr int TILE = THREADS * ITEMS;
  constexpr bool KEYS_ONLY = std::is_same<V, uint8_t>::value;
  const uint64_t tiles = (n + TILE - 1) / TILE;
  if (n > 0xFFFFFFFFull)
    return set_error(MB_ERR_LENGTH_TOO_LARGE, "radix sort length does not fit in u32", n);
  if (n >= (uint64_t)DigitStatus<SW>::kMask)
    return set_error(MB_ERR_LAUNCH, "radix sort: status words too narrow for this length", n);
  // Scratch: [plan][hist P*256][counters + abort word][status P*tiles*256]
  // [tmp keys][tmp values][keys output when none is given]
  const size_t plan_b = ((sizeof(PassPlan) + 255) / 256) * 256;
  const size_t hist_b = (size_t)PASSES * kBins * 4;
  const size_t cnt_b = 256;
  const size_t status_b = (size_t)PASSES * tiles * kBins * sizeof(SW);
  const size_t zero_b = plan_b + hist_b + cnt_b + status_b;
  const size_t tk_b = ((n * sizeof(K) + 255) / 256) * 256;
  const size_t tv_b = KEYS_ONLY ? 0 : ((n * sizeof(V) + 255) / 256) * 256;
  Scratch scratch;
  MB_TRY(scratch.alloc(ex, zero_b + tk_b + tv_b + (out_k ? 0 : tk_b)));
  char* base = scratch.as<char>();
  PassPlan* plan = (PassPlan*)base;
  uint32_t* hist = (uint32_t*)(base + plan_b);
  uint32_t* counters = (uint32_t*)(base + plan_b + hist_b);
  SW* status = (SW*)(base + plan_b + hist_b + cnt_b);
  K* tmp_k = (K*)(base + zero_b);
  V* tmp_v = KEYS_ONLY ? nullptr : (V*)(base + zero_b + tk_b);
  K* final_k = out_k ? out_k : (K*)(base + zero_b + tk_b + tv_b);
  MB_CUDA(cudaMemsetAsync(base, 0, zero_b, ex->stream));

  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  // Each block counts at least one chunk per warp (16 keys per thread); at
  // most two blocks per SM stay resident.
  const uint64_t hist_blocks = std::min<uint64_t>((n + kHistThreads * 16 - 1) / (kHistThreads * 16),
                                                  (uint64_t)sms * 2);
  {
    TimedLaunch timed(ex, MB_KF_RADIX_HISTOGRAM);
    if constexpr (PASSES <= 4) {
      // lane-private bins: one block per SM
      const size_t hsmem = (size_t)PASSES * kBins * 32 * sizeof(uint32_t);
      const uint64_t lane_blocks = std::min<uint64_t>(
          (n + kHistLaneThreads * 16 - 1) / (kHistLaneThreads * 16), (uint64_t)sms);
      MB_CUDA(cudaFuncSetAttribute(radix_histogram_lanes_kernel<K, ENC, PASSES>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
      radix_histogram_lanes_kernel<K, ENC, PASSES>
          <<<(unsigned)std::max<uint64_t>(1, lane_blocks), kHistLaneThreads, hsmem, ex->stream>>>(
              in_k, n, n_dev, hist);
    } else {
      radix_histogram_kernel<K, ENC, PASSES><<<(unsigned)std::max<uint64_t>(1, hist_blocks),
                                               kHistThreads, 0, ex->stream>>>(in_k, n, n_dev,
                                                                              hist);
    }
  }
  MB_CUDA(cudaGetLastError());
  radix_plan_kernel<<<1, kBins, 0, ex->stream>>>(hist, PASSES, n, n_dev, plan, in_k, final_k,
                                                 tmp_k, in_v, out_v, tmp_v);
  MB_CUDA(cudaGetLastError());
  const DevErr err{ex->status_dev, counters + 32};
  const bool aligned = (uintptr_t)in_k % 16 == 0 && (uintptr_t)final_k % 16 == 0 &&
                       (KEYS_ONLY || ((uintptr_t)in_v % 16 == 0 && (uintptr_t)out_v % 16 == 0));
  if (aligned) {
    const size_t smem = sizeof(OnesweepTmaSmem<K, V, THREADS, ITEMS, NT>);
    auto kern = radix_onesweep_tma_kernel<K, ENC, V, THREADS, ITEMS, NT,
                                          P64 && sizeof(K) == 4 && sizeof(V) == 4, MINB, SW>;
    MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int p = 0; p < PASSES; ++p) {
      {
        TimedLaunch timed(ex, MB_KF_RADIX_ONESWEEP);
        kern<<<(unsigned)tiles, THREADS, smem, ex->stream>>>(
            plan, p, (uint32_t)n, hist, status + (size_t)p * tiles * kBins, counters + p, err);
      }
      MB_CUDA(cudaGetLastError());
    }
    return MB_OK;
  }
  const size_t smem = onesweep_smem<K, V, THREADS, ITEMS>();
  auto kern = radix_onesweep_kernel<K, ENC, V, THREADS, ITEMS, SW>;
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int p = 0; p < PASSES; ++p) {
    {
      TimedLaunch timed(ex, MB_KF_RADIX_ONESWEEP);
      kern<<<(unsigned)tiles, THREADS, smem, ex->stream>>>(
          plan, p, n, hist, status + (size_t)p * tiles * kBins, counters + p, err);
    }
    MB_CUDA(cudaGetLastError());
  }
  return MB_OK;
}

template <class K, int ENC, class V>
int onesweep_sort(mb_executor* ex, const K* in_k, const V* in_v, K* out_k, V* out_v, uint64_t n,
                  const uint32_t* n_dev) {
  if (n == 0) return MB_OK;
  if (n >= (1ull << 30)) {
    // 2^30 items or more: 64-bit look-back status words, default shapes.
    if constexpr (sizeof(K) == 4 && sizeof(V) <= 4)
      return onesweep_sort_cfg<K, ENC, V, 512, 16, 1, true, 0, uint64_t>(ex, in_k, in_v, out_k,
                                                                         out_v, n, n_dev);
    else
      return onesweep_sort_cfg<K, ENC, V, 256, 16, 1, false, 0, uint64_t>(ex, in_k, in_v, out_k,
                                                                          out_v, n, n_dev);
  }
  int cfg = ex->tune[MB_TUNE_RADIX];
  if (cfg < 0) cfg = (sizeof(K) == 4 && sizeof(V) <= 4) ? kRadixDefault32 : kRadixDefault;
  switch (cfg) {
    case 1: return onesweep_sort_cfg<K, ENC, V, 256, 16, 3>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 2: return onesweep_sort_cfg<K, ENC, V, 512, 16, 1>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 3: return onesweep_sort_cfg<K, ENC, V, 256, 12, 3>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 4: return onesweep_sort_cfg<K, ENC, V, 1024, 16, 1>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 5: return onesweep_sort_cfg<K, ENC, V, 384, 16, 1>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 6:
      return onesweep_sort_cfg<K, ENC, V, 512, 16, 1, true>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 7:
      return onesweep_sort_cfg<K, ENC, V, 512, 12, 1, true>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 8:
      return onesweep_sort_cfg<K, ENC, V, 384, 16, 1, true>(ex, in_k, in_v, out_k, out_v, n, n_dev);
    case 9:
      return onesweep_sort_cfg<K, ENC, V, 384, 16, 0, true, 3>(ex, in_k, in_v, out_k, out_v, n,
                                                               n_dev);
    default: return onesweep_sort_cfg<K, ENC, V, 256, 16, 1>(ex, in_k, in_v, out_k, out_v, n, n_dev);
  }
}

// Dispatch on the value width (0 = keys only, 4, 8).  K is the unsigned
// integer type of the key's width, ENC its element type's encoding.
template <class K, int ENC>
int sort_keys_vals(mb_executor* ex, const void* ik, const void* iv, void* ok, void* ov,
                   size_t vsize, uint64_t n, const uint32_t* n_dev) {
  switch (vsize) {
    case 0: return onesweep_sort<K, ENC, uint8_t>(ex, (const K*)ik, nullptr, (K*)ok, nullptr, n, n_dev);
    case 4: return onesweep_sort<K, ENC, uint32_t>(ex, (const K*)ik, (const uint32_t*)iv, (K*)ok,
                                                   (uint32_t*)ov, n, n_dev);
    case 8: return onesweep_sort<K, ENC, uint64_t>(ex, (const K*)ik, (const uint64_t*)iv, (K*)ok,
                                                   (uint64_t*)ov, n, n_dev);
    default: return set_error(MB_ERR_LAUNCH, "radix values must be 4 or 8 bytes wide");
  }
}

// ---------------------------------------------------- bounded-wait check --
//
// Runs the library's own bounded waits against a condition that never comes,
// so a test can see them end: kind 0, the onesweep digit look-back of tiles
// 1..blocks, whose tile 0 never publishes (the look-back of tile 1 gives up
// after the spin limit and sets the launch's abort word; the later tiles
// then stop waiting as well); kind 1, an mbarrier wait for bulk-copy bytes
// that no copy delivers.  Each records MB_DEV_ERR_LOOKBACK and returns; no
// copy is ever in flight.
__global__ void __launch_bounds__(kBins) bounded_wait_check_kernel(int kind, uint32_t* status,
                                                                   DevErr err) {
  if (kind == 0) {
    const uint64_t tile = blockIdx.x + 1;
    DigitStatus<uint32_t>::publish(status, tile, threadIdx.x, 1u);
    DigitStatus<uint32_t>::lookback(status, tile, threadIdx.x, 1u, err);
  } else {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      mbar_init_fence();
      mbar_arrive_expect_tx(&bar, 16);  // 16 bytes that never arrive
      if (!mbar_wait(&bar, 0)) raise_device_error(err, MB_DEV_ERR_LOOKBACK);
    }
  }
}

}  // namespace

int bounded_wait_check(mb_executor* ex, int kind) {
  MB_TRY(check_exec(ex));
  if (kind != 0 && kind != 1) return set_error(MB_ERR_LAUNCH, "unknown bounded-wait check");
  constexpr int kBlocks = 4;
  Scratch scratch;
  const size_t status_b = (size_t)(kBlocks + 1) * kBins * 4;
  MB_TRY(scratch.alloc(ex, 256 + status_b));
  MB_CUDA(cudaMemsetAsync(scratch.ptr, 0, 256 + status_b, ex->stream));
  const DevErr err{ex->status_dev, scratch.as<uint32_t>()};
  bounded_wait_check_kernel<<<kind == 0 ? kBlocks : 1, kBins, 0, ex->stream>>>(
      kind, (uint32_t*)(scratch.as<char>() + 256), err);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

// Radix sort of plain device columns: keys of type `kdt` (32- or 64-bit
// elements), values of `vsize` bytes (0 = none).  out_k may be null.  With
// `n_dev`, only the first min(*n_dev, n) items are sorted (a count left on
// the device by an earlier step; no host synchronisation).
int radix_sort_plain(mb_executor* ex, int kdt, const void* ik, const void* iv, void* ok, void* ov,
                     size_t vsize, uint64_t n, const uint32_t* n_dev) {
  switch (kdt) {
    case MB_U32: return sort_keys_vals<uint32_t, kEncUnsigned>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    case MB_I32: return sort_keys_vals<uint32_t, kEncSigned>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    case MB_F32: return sort_keys_vals<uint32_t, kEncFloat>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    case MB_U64: return sort_keys_vals<uint64_t, kEncUnsigned>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    case MB_I64: return sort_keys_vals<uint64_t, kEncSigned>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    case MB_F64: return sort_keys_vals<uint64_t, kEncFloat>(ex, ik, iv, ok, ov, vsize, n, n_dev);
    default: return set_error(MB_ERR_LAUNCH, "radix keys must be 32- or 64-bit elements");
  }
}

int radix_tune_count() { return (int)(sizeof(kRadixCfgs) / sizeof(kRadixCfgs[0])); }
const char* radix_tune_text(int c) {
  return (c >= 0 && c < radix_tune_count()) ? kRadixCfgs[c].text : nullptr;
}

}  // namespace mb

extern "C" int mb_check_bounded_waits(mb_executor* ex, int kind) {
  return mb::bounded_wait_check(ex, kind);
}
