// lookback.cuh -- tile status words and the warp-wide decoupled look-back
// used by every single-pass kernel (scan, compaction, segmented scan and
// reduce, by-key algorithms).
//
// A tile publishes its aggregate (flag 1) as soon as it has reduced its own
// items, then its inclusive prefix (flag 2) once it knows its exclusive
// prefix.  Its successors look back over a window of 32 predecessors.
//
// Two publication layouts:
//  * packed: 4-byte values, flag and value in one 64-bit word written with a
//    single relaxed store (one load per predecessor on the read side);
//  * split: flag word (release / acquire) + separate aggregate and inclusive
//    arrays, for wider values (8 and 16 bytes: 64-bit values, and the
//    (head count, value) pairs of the segmented kernels).
//
// Deterministic mode (floating point): the exclusive prefix of tile t is the
// left fold P(j) op A(j+1) op ... op A(t-1) starting from the nearest
// published inclusive prefix P(j).  Every P is itself such a fold, so the
// result equals the strictly sequential chain P(t-1) = P(t-2) op A(t-1) no
// matter how far back the look-back had to go -- bit-identical from run to
// run.  Integer operators are associative, so the default mode reduces the
// window with a warp tree instead.
//
// Every wait is bounded (SpinGuard): on expiry the tile records
// MB_DEV_ERR_LOOKBACK and continues with a fallback prefix so the launch
// ends; the host reports MB_ERR_LAUNCH at the next synchronisation.
#pragma once

#include "common.cuh"

namespace mb {

constexpr uint32_t kFlagNone = 0, kFlagAgg = 1, kFlagIncl = 2;
constexpr unsigned kFull = 0xFFFFFFFFu;

// Floating values are cast with the bit-reinterpreting intrinsics: they keep
// NaN bit patterns exactly.
template <class T>
__device__ __forceinline__ uint64_t to_bits64(T v) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte value");
  if constexpr (std::is_same<T, double>::value) {
    return (uint64_t)__double_as_longlong(v);
  } else if constexpr (std::is_same<T, float>::value) {
    return __float_as_uint(v);
  } else if constexpr (sizeof(T) == 4) {
    uint32_t b;
    memcpy(&b, &v, 4);
    return b;
  } else {
    uint64_t b;
    memcpy(&b, &v, 8);
    return b;
  }
}
template <class T>
__device__ __forceinline__ T from_bits64(uint64_t b) {
  T v;
  if constexpr (std::is_same<T, double>::value) {
    v = __longlong_as_double((long long)b);
  } else if constexpr (std::is_same<T, float>::value) {
    v = __uint_as_float((uint32_t)b);
  } else if constexpr (sizeof(T) == 4) {
    uint32_t w = (uint32_t)b;
    memcpy(&v, &w, 4);
  } else {
    memcpy(&v, &b, 8);
  }
  return v;
}

// Word-wise warp shuffles of any trivially copyable T (size multiple of 4).
template <class T>
__device__ __forceinline__ T shfl_idx(T v, int src) {
  static_assert(sizeof(T) % 4 == 0, "size must be a multiple of 4");
  uint32_t w[sizeof(T) / 4];
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); ++i) w[i] = __shfl_sync(kFull, w[i], src);
  memcpy(&v, w, sizeof(T));
  return v;
}
template <class T>
__device__ __forceinline__ T shfl_up(T v, int d) {
  uint32_t w[sizeof(T) / 4];
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); ++i) w[i] = __shfl_up_sync(kFull, w[i], d);
  memcpy(&v, w, sizeof(T));
  return v;
}
template <class T>
__device__ __forceinline__ T shfl_down(T v, int d) {
  uint32_t w[sizeof(T) / 4];
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); ++i) w[i] = __shfl_down_sync(kFull, w[i], d);
  memcpy(&v, w, sizeof(T));
  return v;
}

// Relaxed word-wise copies to / from global memory.
template <class T>
__device__ __forceinline__ void st_relaxed_any(T* dst, const T& v) {
  if constexpr (sizeof(T) % 8 == 0) {
    uint64_t w[sizeof(T) / 8];
    memcpy(w, &v, sizeof(T));
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 8); ++i) st_relaxed_u64((uint64_t*)dst + i, w[i]);
  } else {
    uint32_t w[sizeof(T) / 4];
    memcpy(w, &v, sizeof(T));
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); ++i) st_relaxed_u32((uint32_t*)dst + i, w[i]);
  }
}
template <class T>
__device__ __forceinline__ T ld_relaxed_any(const T* src) {
  T v;
  if constexpr (sizeof(T) % 8 == 0) {
    uint64_t w[sizeof(T) / 8];
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 8); ++i) w[i] = ld_relaxed_u64((const uint64_t*)src + i);
    memcpy(&v, w, sizeof(T));
  } else {
    uint32_t w[sizeof(T) / 4];
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); ++i) w[i] = ld_relaxed_u32((const uint32_t*)src + i);
    memcpy(&v, w, sizeof(T));
  }
  return v;
}

// How a value shares one 64-bit status word with its 2-bit flag (the packed
// layout).  4-byte values take the low word and the flag the high word;
// other types may specialise this (the segmented kernels pack a 30-bit head
// count beside a 4-byte value).
template <class T>
struct StatePack {
  static constexpr bool kPackable = sizeof(T) == 4;
  __device__ __forceinline__ static uint64_t pack(uint32_t flag, const T& v) {
    return ((uint64_t)flag << 32) | to_bits64(v);
  }
  __device__ __forceinline__ static uint32_t unpack(uint64_t w, T& v) {
    v = from_bits64<T>(w & 0xFFFFFFFFull);
    return (uint32_t)(w >> 32);
  }
};

// One value per slot, each with a "set" flag: the per-group states of the
// grouped deterministic look-back.  Same two layouts as the tile states.
template <class T, bool PACKED>
struct Slots {
  uint64_t* words;
  uint32_t* flags;
  T* vals;

  static size_t bytes(uint64_t n) { return PACKED ? n * 8 : ((n * sizeof(T) + 63) / 64) * 64 + n * 4; }
  static Slots make(void* base, uint64_t n) {
    Slots s{};
    if constexpr (PACKED) {
      s.words = (uint64_t*)base;
    } else {
      s.vals = (T*)base;
      s.flags = (uint32_t*)((char*)base + ((n * sizeof(T) + 63) / 64) * 64);
    }
    return s;
  }
  __device__ __forceinline__ void publish(uint64_t i, const T& v) const {
    if constexpr (PACKED) {
      st_relaxed_u64(words + i, StatePack<T>::pack(kFlagIncl, v));
    } else {
      st_relaxed_any(vals + i, v);
      st_release_u32(flags + i, 1u);
    }
  }
  __device__ __forceinline__ bool peek(uint64_t i, T& v) const {
    if constexpr (PACKED) {
      return StatePack<T>::unpack(ld_relaxed_u64(words + i), v) != kFlagNone;
    } else {
      if (ld_acquire_u32(flags + i) == 0) return false;
      v = ld_relaxed_any(vals + i);
      return true;
    }
  }
};

// Status storage of one launch.  `words` (packed) or `flags`/`agg`/`incl`,
// plus the group states of the deterministic look-back (groups of 32
// tiles: each group's aggregate and its inclusive prefix).
template <class T, bool PACKED>
struct TileState {
  uint64_t* words;
  uint32_t* flags;
  T* agg;
  T* incl;
  Slots<T, PACKED> gagg, gincl;

  static uint64_t groups(uint64_t tiles) { return tiles / 32 + 1; }
  static size_t main_bytes(uint64_t tiles) {
    const size_t b = PACKED ? tiles * 8 : tiles * (4 + 2 * sizeof(T)) + 64;
    return (b + 255) / 256 * 256;
  }
  static size_t slots_bytes(uint64_t tiles) {
    return (Slots<T, PACKED>::bytes(groups(tiles)) + 255) / 256 * 256;
  }
  static size_t bytes(uint64_t tiles) { return main_bytes(tiles) + 2 * slots_bytes(tiles); }
  static TileState make(void* base, uint64_t tiles) {
    TileState s{};
    if constexpr (PACKED) {
      s.words = (uint64_t*)base;
    } else {
      char* p = (char*)base;
      s.agg = (T*)p;
      s.incl = (T*)(p + tiles * sizeof(T));
      s.flags = (uint32_t*)(p + 2 * tiles * sizeof(T));
    }
    char* g = (char*)base + main_bytes(tiles);
    s.gagg = Slots<T, PACKED>::make(g, groups(tiles));
    s.gincl = Slots<T, PACKED>::make(g + slots_bytes(tiles), groups(tiles));
    return s;
  }
  __device__ __forceinline__ void publish(uint64_t t, uint32_t flag, T v) const {
    if constexpr (PACKED) {
      static_assert(StatePack<T>::kPackable, "value does not pack beside its flag");
      st_relaxed_u64(words + t, StatePack<T>::pack(flag, v));
    } else {
      st_relaxed_any((flag == kFlagAgg ? agg : incl) + t, v);
      st_release_u32(flags + t, flag);
    }
  }
  // Reads flag and the value it guards (aggregate for 1, inclusive for 2).
  __device__ __forceinline__ uint32_t peek(uint64_t t, T& v) const {
    if constexpr (PACKED) {
      return StatePack<T>::unpack(ld_relaxed_u64(words + t), v);
    } else {
      uint32_t f = ld_acquire_u32(flags + t);
      if (f != kFlagNone) v = ld_relaxed_any((f == kFlagAgg ? agg : incl) + t);
      return f;
    }
  }
};

// Waits (bounded) until every valid lane's predecessor has published.
// Returns false on expiry.
template <class T, class State>
__device__ __forceinline__ bool wait_window(const State& st, int64_t p, bool valid, uint32_t& f,
                                            T& v, SpinGuard& guard) {
  while (true) {
    f = valid ? st.peek((uint64_t)p, v) : kFlagIncl;
    if (!__any_sync(kFull, f == kFlagNone)) return true;
    bool exp = guard.expired();
    if (__any_sync(kFull, exp)) return false;
  }
}

// Exclusive prefix of `tile` (tile >= 1) under `op`; executed by one full
// warp, result valid in every lane.  On a wait that expires, records the
// error and returns `fallback`.
template <class T, class OpT, bool DET, class State>
__device__ T lookback_exclusive(const State& st, uint64_t tile, const OpT& op,
                                DevErr err, T fallback) {
  const int lane = (int)lane_id();
  SpinGuard guard(err.abort);
  if constexpr (!DET) {
    bool have = false;
    T acc = fallback;
    int64_t base = (int64_t)tile - 1;
    while (true) {
      const int64_t p = base - lane;
      const bool valid = p >= 0;
      uint32_t f;
      T v = fallback;
      if (!wait_window<T>(st, p, valid, f, v, guard)) {
        raise_device_error(err, MB_DEV_ERR_LOOKBACK);
        return fallback;
      }
      const uint32_t incl_mask = __ballot_sync(kFull, valid && f == kFlagIncl);
      const int stop = incl_mask ? __ffs(incl_mask) - 1 : 31;
      bool has = valid && lane <= stop;
      T x = v;
      // Ordered tree: the higher lane holds the earlier tile (left operand).
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        T y = shfl_down(x, off);
        bool yh = __shfl_down_sync(kFull, has, off);
        if (lane + off < 32 && yh) {
          x = has ? op(y, x) : y;
          has = true;
        }
      }
      T win = shfl_idx(x, 0);
      bool win_has = __shfl_sync(kFull, has, 0);
      if (win_has) {
        acc = have ? op(win, acc) : win;
        have = true;
      }
      if (incl_mask) return acc;
      base -= 32;
    }
  } else {
    // Phase 1: nearest predecessor j with an inclusive prefix; every tile
    // in (j, tile) has at least its aggregate published when found.
    int64_t base = (int64_t)tile - 1;
    int64_t j = 0;
    while (true) {
      const int64_t p = base - lane;
      const bool valid = p >= 0;
      uint32_t f;
      T v = fallback;
      if (!wait_window<T>(st, p, valid, f, v, guard)) {
        raise_device_error(err, MB_DEV_ERR_LOOKBACK);
        return fallback;
      }
      const uint32_t incl_mask = __ballot_sync(kFull, valid && f == kFlagIncl);
      if (incl_mask) {
        j = base - (__ffs(incl_mask) - 1);
        break;
      }
      base -= 32;
    }
    // Phase 2: fold forward from P(j); restart from any later inclusive
    // prefix that appeared meanwhile (it is the same chain value).
    T acc;
    {
      T v = fallback;
      st.peek((uint64_t)j, v);  // flag is 2: v = P(j)
      acc = shfl_idx(v, 0);
    }
    for (int64_t c = j + 1; c < (int64_t)tile; c += 32) {
      const int64_t q = c + lane;
      const bool valid = q < (int64_t)tile;
      T v = fallback;
      uint32_t f = valid ? st.peek((uint64_t)q, v) : kFlagNone;
      const int cnt = (int)min((int64_t)32, (int64_t)tile - c);
      for (int k = 0; k < cnt; ++k) {
        T vk = shfl_idx(v, k);
        uint32_t fk = __shfl_sync(kFull, f, k);
        acc = fk == kFlagIncl ? vk : op(acc, vk);
      }
    }
    return acc;
  }
}

// Deterministic exclusive prefix of `tile` (tile >= 1) for non-associative
// (floating-point) operators, executed by one full warp; `own` is the tile's
// aggregate, already published with kFlagAgg (in this mode tiles publish no
// inclusive prefix, except tile 0, whose inclusive prefix is its aggregate).
// Tiles form groups of 32; the prefix is a fixed association of the
// aggregates, whatever the timing:
//
//   H_g(k) = lane k of a warp inclusive scan (shuffle-up tree) over the
//            aggregates of group g's tiles 0..k,
//   A(g)   = H_g(31), published by the group's last tile,
//   G(g)   = G(g-1) op A(g), G(0) = A(0), published by whichever tile first
//            computes it (the same bits every time),
//   E(32g + r) = G(g-1) op H_g(r-1)   (either term absent at g = 0 / r = 0).
//
// A tile waits only for its own group's predecessors and folds serially one
// group aggregate per group back to the nearest published G, instead of one
// tile aggregate per tile back to the nearest inclusive tile.
template <class T, class OpT, class State>
__device__ T lookback_grouped(const State& st, uint64_t tile, const OpT& op, DevErr err,
                              T fallback, T own) {
  const int lane = (int)lane_id();
  SpinGuard guard(err.abort);
  const uint64_t g = tile >> 5;
  const int r = (int)(tile & 31);
  T hs = fallback;
  {
    const bool valid = lane < r;
    uint32_t f;
    T v = fallback;
    if (!wait_window<T>(st, (int64_t)(g << 5) + lane, valid, f, v, guard)) {
      raise_device_error(err, MB_DEV_ERR_LOOKBACK);
      return fallback;
    }
    if (lane == r) v = own;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T y = shfl_up(x, d);
      if (lane >= d) x = op(y, x);
    }
    if (r > 0) hs = shfl_idx(x, r - 1);
    if (r == 31) {
      const T a = shfl_idx(x, 31);
      if (lane == 0) {
        st.gagg.publish(g, a);
        if (g == 0) st.gincl.publish(0, a);
      }
    }
  }
  if (g == 0) return hs;
  // G(g-1): window by window back to the nearest group h with G(h); every
  // group after it has its aggregate (a group's A is published before any G
  // of it can be computed).
  int64_t base = (int64_t)g - 1;
  int64_t h = -1;
  T gh = fallback;
  while (true) {
    const int64_t q = base - lane;
    const bool valid = q >= 0;
    T va = fallback, vi = fallback;
    bool ha = false, hi = false;
    while (true) {
      if (valid) {  // both reads in flight together
        hi = st.gincl.peek((uint64_t)q, vi);
        ha = st.gagg.peek((uint64_t)q, va);
        ha = ha || hi;
      }
      if (!__any_sync(kFull, valid && !ha)) break;
      if (__any_sync(kFull, guard.expired())) {
        raise_device_error(err, MB_DEV_ERR_LOOKBACK);
        return fallback;
      }
    }
    const uint32_t m = __ballot_sync(kFull, valid && hi);
    if (!m) {
      if (base < 32) {
        // This window reaches group 0, whose G follows its A: read again.
        if (__any_sync(kFull, guard.expired())) {
          raise_device_error(err, MB_DEV_ERR_LOOKBACK);
          return fallback;
        }
        continue;
      }
      base -= 32;
      continue;
    }
    const int hl = __ffs(m) - 1;
    h = base - hl;
    gh = shfl_idx(vi, hl);
    if (base == (int64_t)g - 1) {
      // Found in the first window: the newer groups' aggregates are at hand.
      T acc = gh;
      for (int k = hl - 1; k >= 0; --k) acc = op(acc, shfl_idx(va, k));
      if (lane == 0 && hl > 0) st.gincl.publish(g - 1, acc);
      return r > 0 ? op(acc, hs) : acc;
    }
    break;
  }
  // Deeper: fold A(h+1) .. A(g-1) from fresh reads (all published).
  T acc = gh;
  for (int64_t c = h + 1; c < (int64_t)g; c += 32) {
    const int64_t q = c + lane;
    T va = fallback;
    if (q < (int64_t)g) st.gagg.peek((uint64_t)q, va);
    const int cnt = (int)min((int64_t)32, (int64_t)g - c);
    for (int k = 0; k < cnt; ++k) acc = op(acc, shfl_idx(va, k));
  }
  if (lane == 0) st.gincl.publish(g - 1, acc);
  return r > 0 ? op(acc, hs) : acc;
}

}  // namespace mb
