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

template <class T>
__device__ __forceinline__ uint64_t to_bits64(T v) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte value");
  if constexpr (sizeof(T) == 4) {
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
  if constexpr (sizeof(T) == 4) {
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

// Status storage of one launch.  `words` (packed) or `flags`/`agg`/`incl`.
template <class T, bool PACKED>
struct TileState {
  uint64_t* words;
  uint32_t* flags;
  T* agg;
  T* incl;

  static size_t bytes(uint64_t tiles) {
    return PACKED ? tiles * 8 : tiles * (4 + 2 * sizeof(T)) + 64;
  }
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
    return s;
  }
  __device__ __forceinline__ void publish(uint64_t t, uint32_t flag, T v) const {
    if constexpr (PACKED) {
      static_assert(sizeof(T) == 4, "packed layout holds 4-byte values");
      st_relaxed_u64(words + t, ((uint64_t)flag << 32) | to_bits64(v));
    } else {
      st_relaxed_any((flag == kFlagAgg ? agg : incl) + t, v);
      st_release_u32(flags + t, flag);
    }
  }
  // Reads flag and the value it guards (aggregate for 1, inclusive for 2).
  __device__ __forceinline__ uint32_t peek(uint64_t t, T& v) const {
    if constexpr (PACKED) {
      uint64_t w = ld_relaxed_u64(words + t);
      v = from_bits64<T>(w & 0xFFFFFFFFull);
      return (uint32_t)(w >> 32);
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

}  // namespace mb
