// segsort.cu -- ForEachSegment(Sort) of 4-byte values, sorted where they lie.
//
// massively sorts every segment with two global comparison sorts and three
// permutation applications (massively/src/seg/mod.rs:379-425).  Here each
// item is read once and written once, and the sorting happens in shared
// memory:
//
//   * The items are cut into ranges of kSsRange positions; a segment belongs
//     to the range that holds its start.  A classification kernel finds every
//     range's first segment (O(segments + ranges), no searches) and lists the
//     segments longer than a tile.
//   * One CTA per range sorts the range's segments no longer than kSsRange as
//     one pack -- fewer than kSsTile items, since the last of them starts
//     inside the range -- by (segment within the pack, encoded value) with a
//     stable LSD radix sort of 8-bit digits in shared memory.  A digit that
//     is the same for every item of the pack is skipped, so a pack of one
//     segment takes four passes and a pack of up to 256 segments five.  A
//     longer segment can only be the range's last one (it reaches past the
//     range); it is sorted next by the same CTA when it fits a tile.
//   * Segments longer than a tile go to the first CTAs of the same grid, one
//     segment per CTA: per non-constant digit, a counting pass over the
//     segment in tile-sized chunks, each chunk ranked in shared memory and
//     written to its digit's place in the segment (through global scratch
//     between passes).  A segment longer than kSsLongLimit (one CTA would
//     take too long) sends the whole call to the global radix sort of
//     (segment id, value) keys instead.
//
// Ranking inside a pass (ss_pass) is the onesweep kernel's (radix.cu): per
// warp round of 32 keys the lanes with the same digit come from a table of
// lane masks in shared memory, the lowest of them adds their count to the
// warp's digit counter, and the warps' counters are scanned into positions.
// Warps take consecutive runs of positions and rounds follow position order,
// so every pass is stable.
//
// Values are encoded as unsigned keys in the comparator's order (radix.rs:
// 46-89; complemented for GREATER).  Under `<` / `>` on floats -0 and +0 tie,
// so the encoding is not one to one there: the original bits ride along as a
// payload (PAY) and are what is written.  Otherwise the sorted keys decode
// back to the values.

#include <algorithm>

#include "common.cuh"
#include "lookback.cuh"

namespace mb {

namespace {

constexpr int kSsThreads = 256;
constexpr int kSsWarps = kSsThreads / 32;
constexpr int kSsItems = 16;
constexpr int kSsTile = kSsThreads * kSsItems;  // 4096 items
constexpr int kSsRange = kSsTile / 2;           // 2048 start positions per range
constexpr int kSsBins = 256;
constexpr int kSsNT = 3;                        // lane-mask tables used in turn
constexpr uint32_t kSsLongLimit = 1u << 17;     // longest segment one CTA sorts
constexpr uint32_t kSsLongCtas = 2 * 148;
static_assert(kSsThreads == kSsBins, "one thread per digit in the digit scans");

template <bool PAY>
struct SsSmem {
  uint64_t keys[kSsTile];  // (segment within the pack << 32) | encoded value
  uint32_t pay[PAY ? kSsTile : 1];
  uint32_t mask[kSsNT][kSsWarps][kSsBins];
  uint32_t warp_cnt[kSsWarps][kSsBins];
  uint32_t dstart[kSsBins];  // a pass: the digit's first position in the tile
  uint32_t dcount[kSsBins];  // a pass: the digit's count in the tile
  uint32_t gstart[kSsBins];  // long segments: the digit's next position in the segment
  uint32_t hist[4][kSsBins];
  uint32_t heads[kSsTile / 32];  // segment starts in the pack, one bit per item
  uint32_t hpre[kSsTile / 32];   // starts in the words before
  uint32_t wsum[kSsWarps];
  uint32_t red[kSsWarps][4];
  uint32_t flag[4];
};

template <int ENC>
__device__ __forceinline__ uint32_t ss_encode(uint32_t raw, int desc, int ieee) {
  if constexpr (ENC == kEncFloat) {
    if (ieee && (raw & 0x7FFFFFFFu) == 0) raw = 0;  // -0 == +0 under `<`
  }
  const uint32_t u = enc_bits<uint32_t, ENC>(raw);
  return desc ? ~u : u;
}

template <int ENC>
__device__ __forceinline__ uint32_t ss_decode(uint32_t u, int desc) {
  if (desc) u = ~u;
  if constexpr (ENC == kEncFloat) return (u & 0x80000000u) ? (u ^ 0x80000000u) : ~u;
  else if constexpr (ENC == kEncSigned) return u ^ 0x80000000u;
  else return u;
}

template <bool PLAIN>
__device__ __forceinline__ uint32_t ss_load(const Src& in, uint64_t i) {
  if constexpr (PLAIN) return __ldcs((const uint32_t*)in.data + i);
  else return (uint32_t)src_load_bits(in, i);
}

// Exclusive scan of one value per thread (kSsThreads of them) in thread
// order.  Uses sm.wsum, which every caller leaves alone until its next block
// barrier (so no barrier is needed after the reads here).
template <bool PAY>
__device__ __forceinline__ uint32_t ss_block_excl(SsSmem<PAY>& sm, uint32_t v) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) sm.wsum[warp] = incl;
  __syncthreads();
  uint32_t ex = incl - v;
  for (int w = 0; w < warp; ++w) ex += sm.wsum[w];
  return ex;
}

// One stable counting pass over the `valid` keys of sm.keys (and their
// payloads) on the 8-bit digit at `shift`.  Afterwards sm.keys[0, valid)
// holds them grouped by that digit in their previous order, and sm.dstart /
// sm.dcount give each digit's first position and count.  The mask tables
// are zero on entry and on exit.
//
// The keys are spread over all warps (warp w ranks the next `per` rounds of
// 32 positions), so a half-full tile keeps every warp busy.  A lane's peers
// (the lanes whose key has the same digit) come from a per-warp table of lane
// masks: each lane ORs its bit into its digit's word and reads the word back.
// Three tables are used in turn, so a round's words are cleared two rounds
// before their reuse.  The lowest peer adds the group's size to the warp's
// digit counter and its old value comes back through a shuffle before the
// next round's atomics: the ranks are stable.
template <bool PAY>
__device__ __forceinline__ void ss_pass(SsSmem<PAY>& sm, uint32_t valid, int shift) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t per = (valid + kSsThreads - 1) / kSsThreads;  // rounds per warp
  const uint32_t wbase = (uint32_t)warp * 32 * per;
  const int rounds = valid > wbase ? (int)min(per, (valid - wbase + 31) / 32) : 0;
  const uint32_t me = 1u << lane, below = me - 1u;
  for (int d = lane; d < kSsBins; d += 32) sm.warp_cnt[warp][d] = 0;
  __syncwarp();

  uint64_t key[kSsItems];
  uint32_t pay[PAY ? kSsItems : 1];
  uint32_t rd[kSsItems];  // digit << 16 | rank among the warp's keys of that digit
#pragma unroll
  for (int k = 0; k < kSsItems; ++k) {
    if (k < rounds) {
      const uint32_t li = wbase + k * 32 + lane;
      const bool ok = li < valid;  // only a warp's last round can be partial
      key[k] = ok ? sm.keys[li] : 0ull;
      if constexpr (PAY) pay[k] = ok ? sm.pay[li] : 0u;
      const uint32_t d = (uint32_t)(key[k] >> shift) & 0xFFu;
      uint32_t* m = sm.mask[k % kSsNT][warp];
      if (ok) atomicOr(&m[d], me);
      __syncwarp();
      const uint32_t peers = ok ? m[d] : 0u;
      // Round k - 1 was full; every lane has read its word by now.
      if (k > 0) sm.mask[(k - 1) % kSsNT][warp][rd[k - 1] >> 16] = 0;
      if (k == rounds - 1) {
        __syncwarp();
        if (ok) m[d] = 0;
      }
      uint32_t base = 0;
      if (peers != 0 && (peers & below) == 0)
        base = atomicAdd(&sm.warp_cnt[warp][d], (uint32_t)__popc(peers));
      base = __shfl_sync(kFull, base, peers ? __ffs(peers) - 1 : lane);
      rd[k] = (d << 16) | (base + __popc(peers & below));
    }
  }
  __syncthreads();  // every warp's counts are final; every key is in registers

  // Per digit (one per thread): the warps' counts to exclusive offsets, the
  // tile's count, and the tile-wide start.
  {
    const int d = tid;
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSsWarps; ++w) {
      const uint32_t c = sm.warp_cnt[w][d];
      sm.warp_cnt[w][d] = total;
      total += c;
    }
    const uint32_t start = ss_block_excl(sm, total);
    sm.dcount[d] = total;
    sm.dstart[d] = start;
#pragma unroll
    for (int w = 0; w < kSsWarps; ++w) sm.warp_cnt[w][d] += start;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSsItems; ++k) {
    if (k < rounds && wbase + k * 32 + lane < valid) {
      const uint32_t pos = sm.warp_cnt[warp][rd[k] >> 16] + (rd[k] & 0xFFFFu);
      sm.keys[pos] = key[k];
      if constexpr (PAY) sm.pay[pos] = pay[k];
    }
  }
  __syncthreads();
}

// After passes that left out the value bits `low` (the lowest varying
// digits), the keys are in order of (segment, value without `low`), equal
// ones in input order.  Sorts each run of keys equal there by the whole
// value: runs already in order are left as they are, runs of at most
// kSsFixRun keys that are not get a stable insertion sort by one thread.
// Returns false, with the keys in an unknown order, when a longer run is out
// of order (the caller then sorts the pack again with every digit).  Uses
// sm.hist for the run bitmap and the mask tables for run starts and flags,
// and leaves the mask tables zero.
constexpr uint32_t kSsFixRun = 32;

template <bool PAY>
__device__ bool ss_fix_runs(SsSmem<PAY>& sm, uint32_t len, uint32_t low) {
  const int tid = threadIdx.x;
  const uint64_t hmask = ~(uint64_t)low;
  uint32_t* rheads = sm.hist[0];  // kSsTile / 32 words: run starts
  uint32_t* rpre = sm.hist[1];    // runs before each word
  uint16_t* rstart = reinterpret_cast<uint16_t*>(&sm.mask[0][0][0]);  // kSsTile + 1 entries
  uint32_t* rflag = &sm.mask[2][0][0];  // kSsTile bits: the run is out of order
  static_assert(2 * sizeof(sm.mask[0]) >= (kSsTile + 1) * sizeof(uint16_t),
                "run starts fit the first two mask tables");
  if (tid < kSsTile / 32) {
    rheads[tid] = 0;
    rflag[tid] = 0;
  }
  if (tid == 0) sm.flag[0] = 0;
  __syncthreads();
  bool any = false;  // a key below the one before it in the same run
  for (uint32_t b = 0; b < len; b += kSsThreads) {  // a warp's 32 positions form one word
    const uint32_t p = b + tid;
    bool head = false;
    if (p < len) {
      const uint64_t k = sm.keys[p];
      const uint64_t q = p ? sm.keys[p - 1] : 0ull;
      head = p == 0 || ((q ^ k) & hmask) != 0;
      any |= !head && (uint32_t)q > (uint32_t)k;
    }
    const uint32_t word = __ballot_sync(kFull, head);
    if ((tid & 31) == 0) rheads[p >> 5] = word;
  }
  if (__syncthreads_or(any) == 0) return true;  // no run out of order
  {
    const uint32_t c = tid < kSsTile / 32 ? (uint32_t)__popc(rheads[tid]) : 0u;
    const uint32_t ex = ss_block_excl(sm, c);
    if (tid < kSsTile / 32) rpre[tid] = ex;
  }
  __syncthreads();
  const uint32_t runs = rpre[kSsTile / 32 - 1] + (uint32_t)__popc(rheads[kSsTile / 32 - 1]);
  for (uint32_t p = tid; p < len; p += kSsThreads) {
    const uint32_t w = p >> 5;
    const bool head = (rheads[w] >> (p & 31)) & 1u;
    const uint32_t r =
        rpre[w] + (uint32_t)__popc(rheads[w] & (0xFFFFFFFFu >> (31 - (p & 31)))) - 1u;
    if (head) rstart[r] = (uint16_t)p;
    else if ((uint32_t)sm.keys[p - 1] > (uint32_t)sm.keys[p])
      atomicOr(&rflag[r >> 5], 1u << (r & 31));
  }
  if (tid == 0) rstart[runs] = (uint16_t)len;
  __syncthreads();
  for (uint32_t r = tid; r < runs; r += kSsThreads) {
    if (!((rflag[r >> 5] >> (r & 31)) & 1u)) continue;
    const uint32_t a = rstart[r], b = rstart[r + 1];
    if (b - a > kSsFixRun) {
      sm.flag[0] = 1;
      continue;
    }
    for (uint32_t i = a + 1; i < b; ++i) {  // stable: only strictly greater keys move
      const uint64_t k = sm.keys[i];
      uint32_t pv = 0;
      if constexpr (PAY) pv = sm.pay[i];
      uint32_t j = i;
      while (j > a && (uint32_t)sm.keys[j - 1] > (uint32_t)k) {
        sm.keys[j] = sm.keys[j - 1];
        if constexpr (PAY) sm.pay[j] = sm.pay[j - 1];
        --j;
      }
      sm.keys[j] = k;
      if constexpr (PAY) sm.pay[j] = pv;
    }
  }
  __syncthreads();
  const bool ok = sm.flag[0] == 0;
  // Back to zero: the words that held run starts and flags.
  uint32_t* m0 = &sm.mask[0][0][0];
  for (int i = tid; i < (kSsTile + 2) / 2; i += kSsThreads) m0[i] = 0;
  if (tid < kSsTile / 32) rflag[tid] = 0;
  __syncthreads();
  return ok;
}

// Sorts the pack of segments [s_begin, s_end) (items [start, start + len),
// len < kSsTile, start = offsets[s_begin]) into out.
template <int ENC, bool PAY, bool PLAIN>
__device__ __forceinline__ void ss_pack(SsSmem<PAY>& sm, const Src& in, const uint32_t* __restrict__ off,
                        uint64_t s_begin, uint64_t s_end, uint32_t start, uint32_t len, int desc,
                        int ieee, uint32_t* __restrict__ out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (len == 0) return;
  if (len == 1) {  // nothing to order
    if (tid == 0) out[start] = ss_load<PLAIN>(in, start);
    return;
  }
  uint32_t raw[kSsItems];
#pragma unroll
  for (int k = 0; k < kSsItems; ++k) {
    const uint32_t p = (uint32_t)k * kSsThreads + tid;
    if (p < len) raw[k] = ss_load<PLAIN>(in, (uint64_t)start + p);
  }
  // Segment starts -> a bitmap over the pack's items, then per word the
  // starts before it.
  if (tid < kSsTile / 32) sm.heads[tid] = 0;
  __syncthreads();
  for (uint64_t s = s_begin + tid; s < s_end; s += kSsThreads) {
    const uint32_t pos = off[s] - start;
    if (pos < len) atomicOr(&sm.heads[pos >> 5], 1u << (pos & 31));
  }
  __syncthreads();
  {
    const uint32_t c = tid < kSsTile / 32 ? (uint32_t)__popc(sm.heads[tid]) : 0u;
    const uint32_t ex = ss_block_excl(sm, c);
    if (tid < kSsTile / 32) sm.hpre[tid] = ex;
  }
  __syncthreads();
  uint32_t or_lo = 0, and_lo = ~0u, or_hi = 0, and_hi = ~0u;
#pragma unroll
  for (int k = 0; k < kSsItems; ++k) {
    const uint32_t p = (uint32_t)k * kSsThreads + tid;
    if (p < len) {
      const uint32_t w = p >> 5;
      const uint32_t seg =
          sm.hpre[w] + (uint32_t)__popc(sm.heads[w] & (0xFFFFFFFFu >> (31 - (p & 31)))) - 1u;
      const uint32_t u = ss_encode<ENC>(raw[k], desc, ieee);
      sm.keys[p] = ((uint64_t)seg << 32) | u;
      if constexpr (PAY) sm.pay[p] = raw[k];
      or_lo |= u;
      and_lo &= u;
      or_hi |= seg;
      and_hi &= seg;
    }
  }
  or_lo = __reduce_or_sync(kFull, or_lo);
  and_lo = __reduce_and_sync(kFull, and_lo);
  or_hi = __reduce_or_sync(kFull, or_hi);
  and_hi = __reduce_and_sync(kFull, and_hi);
  if (lane == 0) {
    sm.red[warp][0] = or_lo;
    sm.red[warp][1] = and_lo;
    sm.red[warp][2] = or_hi;
    sm.red[warp][3] = and_hi;
  }
  __syncthreads();
  uint32_t var_lo = 0, var_hi = 0;
  {
    uint32_t a = 0, b = ~0u, c = 0, e = ~0u;
#pragma unroll
    for (int w = 0; w < kSsWarps; ++w) {
      a |= sm.red[w][0];
      b &= sm.red[w][1];
      c |= sm.red[w][2];
      e &= sm.red[w][3];
    }
    var_lo = a ^ b;  // bits that differ between some two items
    var_hi = c ^ e;
  }
  // The lowest of four varying value digits is left out of the passes
  // (`low`): a pack's keys rarely agree on segment and the value's top three
  // digits, and ss_fix_runs orders the few that do.  (Leaving out two digits
  // saved a pass but made runs common enough that their fix-up cost more.)
  uint32_t low = 0;
  {
    int m = 0, c = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) m += ((var_lo >> (8 * j)) & 0xFFu) != 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (((var_lo >> (8 * j)) & 0xFFu) && ++c == m - 3)
        low = j == 3 ? ~0u : ((1u << (8 * j + 8)) - 1u);
  }
  auto passes = [&](uint32_t vlo) {
    for (int shift = 0; shift < 64; shift += 8) {
      const uint32_t v = shift < 32 ? (vlo >> shift) : (var_hi >> (shift - 32));
      if (v & 0xFFu) ss_pass(sm, len, shift);
    }
  };
  passes(var_lo & ~low);
  if (low && !ss_fix_runs(sm, len, low)) {
    // A long run out of order: build the keys again and take every digit.
    for (uint32_t p = tid; p < len; p += kSsThreads) {
      const uint32_t r = ss_load<PLAIN>(in, (uint64_t)start + p);
      const uint32_t w = p >> 5;
      const uint32_t seg =
          sm.hpre[w] + (uint32_t)__popc(sm.heads[w] & (0xFFFFFFFFu >> (31 - (p & 31)))) - 1u;
      sm.keys[p] = ((uint64_t)seg << 32) | ss_encode<ENC>(r, desc, ieee);
      if constexpr (PAY) sm.pay[p] = r;
    }
    __syncthreads();
    passes(var_lo);
  }
  for (uint32_t p = tid; p < len; p += kSsThreads) {
    uint32_t v;
    if constexpr (PAY) v = sm.pay[p];
    else v = ss_decode<ENC>((uint32_t)sm.keys[p], desc);
    out[(uint64_t)start + p] = v;
  }
  __syncthreads();  // shared memory is reused by the next pack
}

// Sorts one segment longer than a tile: per non-constant digit a counting
// pass through global memory, tile-sized chunks ranked in shared memory.
// Scratch (indexed like the input): kx0 for keys (and `out` between passes);
// with PAY keys in kx0 / kx1 and payloads in px / out.
template <int ENC, bool PAY, bool PLAIN>
__device__ void ss_long(SsSmem<PAY>& sm, const Src& in, uint32_t start, uint32_t len, int desc,
                        int ieee, uint32_t* __restrict__ out, uint32_t* __restrict__ kx0,
                        uint32_t* __restrict__ kx1, uint32_t* __restrict__ px) {
  const int tid = threadIdx.x;
  for (int i = tid; i < 4 * kSsBins; i += kSsThreads) (&sm.hist[0][0])[i] = 0;
  if (tid < 4) sm.flag[tid] = 0;
  __syncthreads();
  for (uint32_t p = tid; p < len; p += kSsThreads) {
    const uint32_t u = ss_encode<ENC>(ss_load<PLAIN>(in, (uint64_t)start + p), desc, ieee);
#pragma unroll
    for (int j = 0; j < 4; ++j) atomicAdd(&sm.hist[j][(u >> (8 * j)) & 0xFFu], 1u);
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (sm.hist[j][tid] == len) sm.flag[j] = 1;  // digit j is the same everywhere
  __syncthreads();
  int passes[4];
  int np = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (!sm.flag[j]) passes[np++] = j;
  if (np == 0) {  // every key equal: the segment is its own order
    for (uint32_t p = tid; p < len; p += kSsThreads)
      out[(uint64_t)start + p] = ss_load<PLAIN>(in, (uint64_t)start + p);
    __syncthreads();
    return;
  }
  for (int q = 0; q < np; ++q) {
    const int j = passes[q];
    const int shift = 8 * j;
    const bool last = q == np - 1;
    const uint32_t* ksrc = nullptr;
    const uint32_t* psrc = nullptr;
    uint32_t* kdst;
    uint32_t* pdst = nullptr;
    if constexpr (PAY) {
      kdst = (q & 1) ? kx1 : kx0;
      pdst = ((np - 1 - q) & 1) ? px : out;
      if (q > 0) {
        ksrc = ((q - 1) & 1) ? kx1 : kx0;
        psrc = ((np - q) & 1) ? px : out;
      }
    } else {
      kdst = ((np - 1 - q) & 1) ? kx0 : out;
      if (q > 0) ksrc = ((np - q) & 1) ? kx0 : out;
    }
    sm.gstart[tid] = ss_block_excl(sm, sm.hist[j][tid]);
    __syncthreads();
    for (uint32_t c0 = 0; c0 < len; c0 += kSsTile) {
      const uint32_t valid = min((uint32_t)kSsTile, len - c0);
      const uint64_t g0 = (uint64_t)start + c0;
      for (uint32_t p = tid; p < valid; p += kSsThreads) {
        if (q == 0) {
          const uint32_t r = ss_load<PLAIN>(in, g0 + p);
          sm.keys[p] = ss_encode<ENC>(r, desc, ieee);
          if constexpr (PAY) sm.pay[p] = r;
        } else {
          sm.keys[p] = ksrc[g0 + p];
          if constexpr (PAY) sm.pay[p] = psrc[g0 + p];
        }
      }
      __syncthreads();
      ss_pass(sm, valid, shift);
      for (uint32_t i = tid; i < valid; i += kSsThreads) {
        const uint32_t u = (uint32_t)sm.keys[i];
        const uint32_t d = (u >> shift) & 0xFFu;
        const uint64_t o = (uint64_t)start + sm.gstart[d] + (i - sm.dstart[d]);
        if (last) {
          if constexpr (PAY) out[o] = sm.pay[i];
          else out[o] = ss_decode<ENC>(u, desc);
        } else {
          kdst[o] = u;
          if constexpr (PAY) pdst[o] = sm.pay[i];
        }
      }
      __syncthreads();
      sm.gstart[tid] += sm.dcount[tid];
      __syncthreads();
    }
  }
}

// Per segment s: ranges whose first segment is s (ranges r with
// offsets[s - 1] < r * kSsRange <= offsets[s]); s == nseg closes the list.
// Lists segments longer than a tile and takes the largest length.
__global__ void __launch_bounds__(256)
    ss_classify_kernel(const uint32_t* __restrict__ off, uint64_t nseg, uint32_t nranges,
                       uint32_t* __restrict__ first, uint32_t* __restrict__ stats,
                       uint32_t* __restrict__ long_list, uint64_t long_cap) {
  __shared__ uint32_t s_max[8];
  uint32_t mx = 0;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= nseg;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t o = off[s];
    const uint64_t r_lo = s == 0 ? 0 : (uint64_t)off[s - 1] / kSsRange + 1;
    const uint64_t r_hi = min((uint64_t)(o / kSsRange), (uint64_t)nranges - 1);
    for (uint64_t r = r_lo; r <= r_hi; ++r) first[r] = (uint32_t)s;
    if (s == nseg) {
      first[nranges] = (uint32_t)nseg;
    } else {
      const uint32_t len = off[s + 1] - o;
      mx = max(mx, len);
      if (len > (uint32_t)kSsTile) {
        const uint32_t i = atomicAdd(&stats[0], 1u);
        if (i < long_cap) long_list[i] = (uint32_t)s;  // always, for valid offsets
      }
    }
  }
  mx = __reduce_max_sync(kFull, mx);
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) mx = max(mx, s_max[w]);
    mx = max(mx, s_max[0]);
    if (mx) atomicMax(&stats[1], mx);
  }
}

// The first long_ctas CTAs sort the long segments (stats[0] of them, listed
// in long_list); CTA long_ctas + r sorts range r.
template <int ENC, bool PAY, bool PLAIN>
__global__ void __launch_bounds__(kSsThreads, PAY ? 2 : 3)
    ss_kernel(Src in, uint32_t n, const uint32_t* __restrict__ off, uint64_t nseg,
              const uint32_t* __restrict__ first, const uint32_t* __restrict__ stats,
              const uint32_t* __restrict__ long_list, uint32_t long_cap, uint32_t long_ctas,
              int desc, int ieee, uint32_t* __restrict__ out, uint32_t* __restrict__ kx0,
              uint32_t* __restrict__ kx1, uint32_t* __restrict__ px, DevErr err) {
  extern __shared__ __align__(16) unsigned char ss_raw[];
  SsSmem<PAY>& sm = *reinterpret_cast<SsSmem<PAY>*>(ss_raw);
  for (int i = threadIdx.x; i < kSsNT * kSsWarps * kSsBins; i += kSsThreads)
    (&sm.mask[0][0][0])[i] = 0;
  __syncthreads();
  // Offsets that are not a segmentation (decreasing, or past n) could make
  // a pack longer than the tile or a segment reach past the column: such a
  // CTA records a bounds error and sorts nothing.
  if (blockIdx.x < long_ctas) {
    const uint32_t count = min(stats[0], long_cap);
    for (uint32_t i = blockIdx.x; i < count; i += long_ctas) {
      const uint32_t s = long_list[i];
      const uint32_t a = off[s], b = off[s + 1];
      if (b < a || b > n) {
        if (threadIdx.x == 0) raise_device_error(err, MB_DEV_ERR_BOUNDS);
        continue;
      }
      ss_long<ENC, PAY, PLAIN>(sm, in, a, b - a, desc, ieee, out, kx0, kx1, px);
    }
    return;
  }
  const uint32_t r = blockIdx.x - long_ctas;
  const uint32_t sa = first[r], sb = first[r + 1];
  if (sa >= sb) return;  // no segment starts in this range
  const uint32_t last = sb - 1;
  const uint32_t lstart = off[last], lend = off[last + 1];
  const uint32_t llen = lend - lstart;
  const bool big = llen > (uint32_t)kSsRange;  // only the last one can be
  const uint32_t pend = big ? last : sb;
  const uint32_t ps = off[sa], pe = off[pend];
  if (pe < ps || pe - ps >= (uint32_t)kSsTile || pe > n || lend < lstart || lend > n) {
    if (threadIdx.x == 0) raise_device_error(err, MB_DEV_ERR_BOUNDS);
    return;
  }
  ss_pack<ENC, PAY, PLAIN>(sm, in, off, sa, pend, ps, pe - ps, desc, ieee, out);
  if (big && llen <= (uint32_t)kSsTile)
    ss_pack<ENC, PAY, PLAIN>(sm, in, off, last, last + 1, lstart, llen, desc, ieee, out);
}

template <int ENC, bool PAY, bool PLAIN>
int ss_launch(mb_executor* ex, const Src& in, uint32_t n, const uint32_t* off, uint64_t nseg,
              const uint32_t* first, uint32_t nranges, const uint32_t* stats,
              const uint32_t* long_list, uint32_t long_cap, uint32_t long_ctas, int desc,
              int ieee, uint32_t* out, uint32_t* kx0, uint32_t* kx1, uint32_t* px, DevErr err) {
  auto kern = ss_kernel<ENC, PAY, PLAIN>;
  const size_t smem = sizeof(SsSmem<PAY>);
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<long_ctas + nranges, kSsThreads, smem, ex->stream>>>(
      in, n, off, nseg, first, stats, long_list, long_cap, long_ctas, desc, ieee, out, kx0, kx1,
      px, err);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

}  // namespace

// Sorts every segment of a 4-byte column (u32 / i32 / f32, enc 0 / 1 / 2).
// Leaves *done false, having written nothing to `out`, when a segment is
// longer than kSsLongLimit (the caller then takes the global radix path).
int seg_sort_sized(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                   uint64_t nseg, int enc, int desc, int ieee, uint32_t* out, bool* done) {
  *done = false;
  const uint64_t n = values->len;
  if (n == 0 || n > 0xFFFFFFFFull || nseg == 0) return MB_OK;
  const uint32_t nranges = (uint32_t)((n + kSsRange - 1) / kSsRange);
  const uint64_t long_cap = n / (kSsTile + 1) + 1;
  const size_t first_b = ((uint64_t)(nranges + 1) * 4 + 255) / 256 * 256;
  Scratch meta;
  MB_TRY(meta.alloc(ex, 256 + first_b + long_cap * 4));
  uint32_t* stats = meta.as<uint32_t>();
  uint32_t* first = (uint32_t*)(meta.as<char>() + 256);
  uint32_t* long_list = (uint32_t*)(meta.as<char>() + 256 + first_b);
  MB_CUDA(cudaMemsetAsync(stats, 0, 16, ex->stream));
  const unsigned g = (unsigned)std::min<uint64_t>((nseg + 1 + 255) / 256, 148ull * 8);
  ss_classify_kernel<<<g, 256, 0, ex->stream>>>(offsets, nseg, nranges, first, stats, long_list,
                                                long_cap);
  MB_CUDA(cudaGetLastError());

  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturing = ex->capturing ||
                         (cudaStreamIsCapturing(ex->stream, &cs) == cudaSuccess &&
                          cs != cudaStreamCaptureStatusNone);
  uint32_t long_ctas = kSsLongCtas;
  if (!capturing) {
    // Two words to the host: how many long segments, and the longest.
    MB_CUDA(cudaMemcpyAsync(ex->host_pinned, stats, 8, cudaMemcpyDeviceToHost, ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
    const uint32_t count = ex->host_pinned[0], longest = ex->host_pinned[1];
    if (longest > kSsLongLimit) return MB_OK;  // the global path sorts this one
    long_ctas = std::min(count, kSsLongCtas);
  }
  Scratch kx;
  uint32_t *kx0 = nullptr, *kx1 = nullptr, *px = nullptr;
  if (long_ctas > 0) {
    MB_TRY(kx.alloc(ex, n * 4 * (ieee ? 3 : 1)));
    kx0 = kx.as<uint32_t>();
    if (ieee) {
      kx1 = kx0 + n;
      px = kx0 + 2 * n;
    }
  }
  const Src in = to_src(*values);
  const bool plain = src_plain(*values, values->vtype) && values->len_dev == nullptr;
  TimedLaunch timed(ex, MB_KF_SEG_SORT);
  const DevErr err{ex->status_dev, stats + 2};
#define MB_SS(ENC, PAY)                                                                        \
  (plain ? ss_launch<ENC, PAY, true>(ex, in, (uint32_t)n, offsets, nseg, first, nranges, stats, \
                                     long_list, (uint32_t)long_cap, long_ctas, desc, ieee, out,  \
                                     kx0, kx1, px, err)                                          \
         : ss_launch<ENC, PAY, false>(ex, in, (uint32_t)n, offsets, nseg, first, nranges, stats, \
                                      long_list, (uint32_t)long_cap, long_ctas, desc, ieee, out, \
                                      kx0, kx1, px, err))
  int rc;
  if (enc == kEncUnsigned) rc = MB_SS(kEncUnsigned, false);
  else if (enc == kEncSigned) rc = MB_SS(kEncSigned, false);
  else if (ieee) rc = MB_SS(kEncFloat, true);
  else rc = MB_SS(kEncFloat, false);
#undef MB_SS
  MB_TRY(rc);
  *done = true;
  return MB_OK;
}

}  // namespace mb
