// oracle.cpp -- CPU oracle for the massively primitive path.  TEST
// INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg are the only callers; the product library never links it.
//
// A sequential C++17 restatement of massively's own CPU references,
// verification/oracle/src/vector.rs and verification/oracle/src/seg.rs, plus
// the semantic pins those files leave to the library sources:
//   * radix key encodings        massively/src/core/radix.rs:46-89
//   * empty segment -> init      massively/src/seg/mod.rs:728-729, 772-778
//   * PCG-hash input streams     massively/src/api/util/random.rs:12-22, 331-385
// Parity pin: tests/test_oracle_golden.py checks every function here against
// the known-answer vectors of massively's own tests (tests/golden/).
//
// Integer ADD / MUL wrap (two's complement), as the GPU kernels do; the Rust
// oracle panics on overflow in debug builds and its tests avoid overflow.
//
// Every entry point is `extern "C"`, dispatches on the mb_dtype / mb_op /
// mb_pred2 ids of include/massively_b200.h and works on host memory.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "../include/massively_b200.h"

namespace {

template <class T> struct Unsigned { using type = T; };
template <> struct Unsigned<int8_t> { using type = uint8_t; };
template <> struct Unsigned<int16_t> { using type = uint16_t; };
template <> struct Unsigned<int32_t> { using type = uint32_t; };
template <> struct Unsigned<int64_t> { using type = uint64_t; };
template <> struct Unsigned<float> { using type = uint32_t; };
template <> struct Unsigned<double> { using type = uint64_t; };

template <class T> constexpr bool kFloat = std::is_floating_point<T>::value;

// Binary operators of mb_op.  Wrapping integer arithmetic is done in the
// unsigned type of the same width.
template <class T> T apply_op(int op, T a, T b) {
  if constexpr (kFloat<T>) {
    switch (op) {
      case MB_OP_ADD: return a + b;
      case MB_OP_MUL: return a * b;
      case MB_OP_MIN: return b < a ? b : a;
      case MB_OP_MAX: return a < b ? b : a;
      case MB_OP_TAKE_LEFT: return a;
      case MB_OP_TAKE_RIGHT: return b;
      default: return a;
    }
  } else {
    using U = typename Unsigned<T>::type;
    U ua = (U)a, ub = (U)b;
    switch (op) {
      case MB_OP_ADD: return (T)(U)(ua + ub);
      case MB_OP_MUL: return (T)(U)(ua * ub);
      case MB_OP_MIN: return b < a ? b : a;
      case MB_OP_MAX: return a < b ? b : a;
      case MB_OP_BIT_AND: return (T)(U)(ua & ub);
      case MB_OP_BIT_OR: return (T)(U)(ua | ub);
      case MB_OP_BIT_XOR: return (T)(U)(ua ^ ub);
      case MB_OP_TAKE_LEFT: return a;
      case MB_OP_TAKE_RIGHT: return b;
      default: return a;
    }
  }
}

// Order-preserving radix encoding (massively/src/core/radix.rs:46-89).
template <class T> typename Unsigned<T>::type radix_encode(T v) {
  if constexpr (std::is_same<T, float>::value) {
    uint32_t raw; std::memcpy(&raw, &v, 4);
    return (raw & 0x80000000u) ? ~raw : (raw ^ 0x80000000u);
  } else if constexpr (std::is_same<T, double>::value) {
    uint64_t raw; std::memcpy(&raw, &v, 8);
    return (raw & 0x8000000000000000ull) ? ~raw : (raw ^ 0x8000000000000000ull);
  } else if constexpr (std::is_signed<T>::value) {
    using U = typename Unsigned<T>::type;
    return (U)((U)v ^ ((U)1 << (sizeof(T) * 8 - 1)));
  } else {
    return v;
  }
}
// Binary predicates of mb_pred2.
template <class T> bool apply_pred2(int p, T a, T b) {
  switch (p) {
    case MB_LESS: return a < b;
    case MB_GREATER: return b < a;
    case MB_TOTAL_LESS: return radix_encode<T>(a) < radix_encode<T>(b);
    case MB_EQUAL: return a == b;
    default: return false;
  }
}

// Unary predicates / maps of mb_unary that yield a flag.
template <class T> uint32_t apply_flag(int u, T x) {
  switch (u) {
    case MB_UN_IS_TRUE: return x != T(0);
    case MB_UN_IS_FALSE: return x == T(0);
    case MB_UN_IS_EVEN:
      if constexpr (kFloat<T>) return 0; else return ((uint64_t)x & 1u) == 0;
    case MB_UN_IS_ODD:
      if constexpr (kFloat<T>) return 0; else return ((uint64_t)x & 1u) != 0;
    case MB_UN_IS_NEGATIVE: return x < T(0);
    case MB_UN_IS_POSITIVE: return x > T(0);
    default: return x != T(0);
  }
}

// Rust's slice::sort_by with the Less-derived Ordering is a stable sort
// (verification/oracle/src/vector.rs:666-680); std::stable_sort with the
// same strict predicate yields the same permutation.
template <class T, class Get> void stable_sort_by(std::vector<size_t>& order, int less, Get get) {
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return apply_pred2<T>(less, get(x), get(y)); });
}

#define ORC_DISPATCH(dtype, FN, ...)                      \
  switch (dtype) {                                        \
    case MB_U8: return FN<uint8_t>(__VA_ARGS__);          \
    case MB_U16: return FN<uint16_t>(__VA_ARGS__);        \
    case MB_U32: return FN<uint32_t>(__VA_ARGS__);        \
    case MB_U64: return FN<uint64_t>(__VA_ARGS__);        \
    case MB_I8: return FN<int8_t>(__VA_ARGS__);           \
    case MB_I16: return FN<int16_t>(__VA_ARGS__);         \
    case MB_I32: return FN<int32_t>(__VA_ARGS__);         \
    case MB_I64: return FN<int64_t>(__VA_ARGS__);         \
    case MB_F32: return FN<float>(__VA_ARGS__);           \
    case MB_F64: return FN<double>(__VA_ARGS__);          \
    default: break;                                       \
  }

size_t dtype_size(int dt) {
  switch (dt) {
    case MB_U8: case MB_I8: return 1;
    case MB_U16: case MB_I16: return 2;
    case MB_U32: case MB_I32: case MB_F32: return 4;
    default: return 8;
  }
}

// ----------------------------------------------------------- vector.rs ----

// reduce: verification/oracle/src/vector.rs:33-42
template <class T> int reduce_t(const void* in, uint64_t n, int op, const void* init, void* out) {
  const T* x = (const T*)in;
  T acc; std::memcpy(&acc, init, sizeof(T));
  for (uint64_t i = 0; i < n; ++i) acc = apply_op<T>(op, acc, x[i]);
  std::memcpy(out, &acc, sizeof(T));
  return 0;
}

// inclusive_scan: vector.rs:44-59
template <class T> int inclusive_scan_t(const void* in, uint64_t n, int op, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  for (uint64_t i = 0; i < n; ++i) y[i] = i == 0 ? x[0] : apply_op<T>(op, y[i - 1], x[i]);
  return 0;
}

// exclusive_scan: vector.rs:61-74
template <class T> int exclusive_scan_t(const void* in, uint64_t n, int op, const void* init, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  T acc; std::memcpy(&acc, init, sizeof(T));
  for (uint64_t i = 0; i < n; ++i) { T v = x[i]; y[i] = acc; acc = apply_op<T>(op, acc, v); }
  return 0;
}

// copy_where / remove_where: vector.rs:255-271.  Rows of `width` bytes.
uint64_t compact_rows(const void* in, uint64_t n, uint64_t width, const uint32_t* stencil,
                      bool keep_set, void* out) {
  const uint8_t* x = (const uint8_t*)in; uint8_t* y = (uint8_t*)out;
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i)
    if ((stencil[i] != 0) == keep_set) { std::memcpy(y + k * width, x + i * width, width); ++k; }
  return k;
}

// partition: vector.rs:216-233 (matching, then failing; both stable)
template <class T> int64_t partition_t(const void* in, uint64_t n, int pred, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) if (apply_flag<T>(pred, x[i])) y[k++] = x[i];
  uint64_t b = k;
  for (uint64_t i = 0; i < n; ++i) if (!apply_flag<T>(pred, x[i])) y[k++] = x[i];
  return (int64_t)b;
}

// stable comparator sort: vector.rs:483-491 and 666-680.  Returns the
// permutation (source index per output position).
template <class T> int sort_perm_t(const void* keys, uint64_t n, int less, uint32_t* perm) {
  const T* k = (const T*)keys;
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  stable_sort_by<T>(order, less, [&](size_t i) { return k[i]; });
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)order[i];
  return 0;
}

// reduce_by_key: vector.rs:144-174.  A run continues while KeyEq(head, k[i]).
template <class K, class V>
int64_t reduce_by_key_kv(const K* k, const V* v, uint64_t n, int key_eq, int op, V init,
                         K* ok, V* ov) {
  uint64_t i = 0, r = 0;
  while (i < n) {
    K key = k[i];
    V acc = init;
    while (i < n && (i == 0 || apply_pred2<K>(key_eq, key, k[i]))) {
      acc = apply_op<V>(op, acc, v[i]);
      ++i;
      if (i < n && !apply_pred2<K>(key_eq, key, k[i])) break;
    }
    ok[r] = key; ov[r] = acc; ++r;
  }
  return (int64_t)r;
}

// Run heads of reduce_by_key (1 where a new run starts).  Used for the
// multi-column form: per-column reductions share the key runs.
template <class K> int run_heads_t(const void* keys, uint64_t n, int key_eq, uint8_t* heads) {
  const K* k = (const K*)keys;
  uint64_t head = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (i == 0 || !apply_pred2<K>(key_eq, k[head], k[i])) { heads[i] = 1; head = i; }
    else heads[i] = 0;
  }
  return 0;
}

// Per-run reduction of one value column given the run heads.
template <class V> int64_t runs_reduce_t(const void* vals, uint64_t n, const uint8_t* heads,
                                         int op, const void* init, void* out) {
  const V* v = (const V*)vals; V* o = (V*)out;
  V i0; std::memcpy(&i0, init, sizeof(V));
  int64_t r = -1;
  V acc = i0;
  for (uint64_t i = 0; i < n; ++i) {
    if (heads[i]) { if (r >= 0) o[r] = acc; ++r; acc = i0; }
    acc = apply_op<V>(op, acc, v[i]);
  }
  if (r >= 0) o[r] = acc;
  return r + 1;
}

// inclusive_scan_by_key / exclusive_scan_by_key: vector.rs:92-142 (adjacent
// key comparison).
template <class V> int scan_by_key_heads_t(const void* vals, uint64_t n, const uint8_t* heads,
                                           int op, int exclusive, const void* init, void* out) {
  const V* v = (const V*)vals; V* o = (V*)out;
  V i0{}; if (exclusive) std::memcpy(&i0, init, sizeof(V));
  V acc = i0;
  for (uint64_t i = 0; i < n; ++i) {
    if (exclusive) {
      if (heads[i]) acc = i0;
      o[i] = acc; acc = apply_op<V>(op, acc, v[i]);
    } else {
      acc = heads[i] ? v[i] : apply_op<V>(op, acc, v[i]);
      o[i] = acc;
    }
  }
  return 0;
}
template <class K> int adjacent_heads_t(const void* keys, uint64_t n, int key_eq, uint8_t* heads) {
  const K* k = (const K*)keys;
  for (uint64_t i = 0; i < n; ++i) heads[i] = (i == 0 || !apply_pred2<K>(key_eq, k[i - 1], k[i]));
  return 0;
}

// merge: vector.rs:493-513 (right taken only when strictly less).  Writes
// the source of every output element: left index i, or (1<<63) | right j.
template <class T> int merge_src_t(const void* l, uint64_t nl, const void* r, uint64_t nr,
                                   int less, uint64_t* src) {
  const T* a = (const T*)l; const T* b = (const T*)r;
  uint64_t i = 0, j = 0, k = 0;
  while (i < nl && j < nr) {
    if (apply_pred2<T>(less, b[j], a[i])) src[k++] = (1ull << 63) | j++;
    else src[k++] = i++;
  }
  while (i < nl) src[k++] = i++;
  while (j < nr) src[k++] = (1ull << 63) | j++;
  return 0;
}

// lower_bound / upper_bound: vector.rs:404-426 -- per value, the partition
// point of the sorted source: first index whose candidate is not less than
// the value (lower), or that the value is less than (upper).
template <class T> int bounds_t(const void* src, uint64_t n, const void* vals, uint64_t m,
                                int less, int upper, uint32_t* out) {
  const T* a = (const T*)src; const T* v = (const T*)vals;
  for (uint64_t q = 0; q < m; ++q) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      const bool in_prefix = upper ? !apply_pred2<T>(less, v[q], a[mid])
                                   : apply_pred2<T>(less, a[mid], v[q]);
      if (in_prefix) lo = mid + 1;
      else hi = mid;
    }
    out[q] = (uint32_t)lo;
  }
  return 0;
}

// set_union / set_intersection / set_difference: vector.rs:595-664.
// mode 0 union, 1 intersection, 2 difference.  Same source encoding.
template <class T> int64_t set_op_src_t(const void* l, uint64_t nl, const void* r, uint64_t nr,
                                        int less, int mode, uint64_t* src) {
  const T* a = (const T*)l; const T* b = (const T*)r;
  uint64_t i = 0, j = 0, k = 0;
  while (i < nl && j < nr) {
    if (apply_pred2<T>(less, a[i], b[j])) { if (mode != 1) src[k++] = i; ++i; }
    else if (apply_pred2<T>(less, b[j], a[i])) { if (mode == 0) src[k++] = (1ull << 63) | j; ++j; }
    else { if (mode != 2) src[k++] = i; ++i; ++j; }
  }
  if (mode != 1) while (i < nl) src[k++] = i++;
  if (mode == 0) while (j < nr) src[k++] = (1ull << 63) | j++;
  return (int64_t)k;
}

// unique: vector.rs:560-576
template <class T> int64_t unique_t(const void* in, uint64_t n, int eq, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (k == 0 || !apply_pred2<T>(eq, y[k - 1], x[i])) y[k++] = x[i];
  return (int64_t)k;
}

// -------------------------------------------------------------- seg.rs ----

// seg::inclusive_scan / exclusive_scan: verification/oracle/src/seg.rs:48-88
template <class T> int seg_scan_t(const void* in, const uint32_t* off, uint64_t nseg, int op,
                                  int exclusive, const void* init, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  T i0{}; if (exclusive) std::memcpy(&i0, init, sizeof(T));
  for (uint64_t s = 0; s < nseg; ++s) {
    T acc = i0;
    for (uint64_t i = off[s]; i < off[s + 1]; ++i) {
      if (exclusive) { y[i] = acc; acc = apply_op<T>(op, acc, x[i]); }
      else { acc = i == off[s] ? x[i] : apply_op<T>(op, acc, x[i]); y[i] = acc; }
    }
  }
  return 0;
}

// seg::reduce: seg.rs:155-169 (empty segment folds to init)
template <class T> int seg_reduce_t(const void* in, const uint32_t* off, uint64_t nseg, int op,
                                    const void* init, void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  T i0; std::memcpy(&i0, init, sizeof(T));
  for (uint64_t s = 0; s < nseg; ++s) {
    T acc = i0;
    for (uint64_t i = off[s]; i < off[s + 1]; ++i) acc = apply_op<T>(op, acc, x[i]);
    y[s] = acc;
  }
  return 0;
}

// seg::sort: seg.rs:18-39 (stable, per segment)
template <class T> int seg_sort_t(const void* in, const uint32_t* off, uint64_t nseg, int less,
                                  void* out) {
  const T* x = (const T*)in; T* y = (T*)out;
  for (uint64_t s = 0; s < nseg; ++s) {
    std::vector<T> seg(x + off[s], x + off[s + 1]);
    std::stable_sort(seg.begin(), seg.end(),
                     [&](const T& a, const T& b) { return apply_pred2<T>(less, a, b); });
    std::copy(seg.begin(), seg.end(), y + off[s]);
  }
  return 0;
}

// ------------------------------------------------------------ random ------

// massively/src/api/util/random.rs:12-16 (pcg_hash32_host)
inline uint32_t pcg_hash32(uint32_t input) {
  uint32_t state = input * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28) + 4)) ^ state) * 277803737u;
  return (word >> 22) ^ word;
}

// First-index searches and flags (vector.rs:176-218, 317-378), one entry
// for all of them; the result uses the C ABI's encoding: an index, MB_NONE
// for None, or a 0 / 1 flag.
//   0 find_if           vector.rs:212   position of the first passing item
//   1 is_partitioned    core/predicate.rs:111-127: no passing item after a
//                       failing one (flag)
//   2 adjacent_find     vector.rs:344   first i with eq(x[i], x[i+1])
//   3 is_sorted_until   vector.rs:367   first i >= 1 with less(x[i], x[i-1]),
//                                       else len
//   4 mismatch          vector.rs:330
//   5 equal             vector.rs:317   (flag)
//   6 lexicographical_compare  vector.rs:388 (flag)
//   7 find_first_of     vector.rs:354
template <class T> int64_t find_t(int kind, const void* av, uint64_t na, const void* bv,
                                  uint64_t nb, int op) {
  const T* a = (const T*)av; const T* b = (const T*)bv;
  const int64_t none = (int64_t)MB_NONE;
  switch (kind) {
    case 0:
      for (uint64_t i = 0; i < na; ++i) if (apply_flag<T>(op, a[i])) return (int64_t)i;
      return none;
    case 1: {
      uint64_t i = 0;
      while (i < na && apply_flag<T>(op, a[i])) ++i;
      while (i < na && !apply_flag<T>(op, a[i])) ++i;
      return i == na ? 1 : 0;
    }
    case 2:
      for (uint64_t i = 0; i + 1 < na; ++i) if (apply_pred2<T>(MB_EQUAL, a[i], a[i + 1])) return (int64_t)i;
      return none;
    case 3:
      for (uint64_t i = 1; i < na; ++i) if (apply_pred2<T>(op, a[i], a[i - 1])) return (int64_t)i;
      return (int64_t)na;
    case 4: {
      const uint64_t n = std::min(na, nb);
      for (uint64_t i = 0; i < n; ++i) if (!apply_pred2<T>(MB_EQUAL, a[i], b[i])) return (int64_t)i;
      return na != nb ? (int64_t)n : none;
    }
    case 5: {
      if (na != nb) return 0;
      for (uint64_t i = 0; i < na; ++i) if (!apply_pred2<T>(MB_EQUAL, a[i], b[i])) return 0;
      return 1;
    }
    case 6: {
      const uint64_t n = std::min(na, nb);
      for (uint64_t i = 0; i < n; ++i) {
        if (apply_pred2<T>(op, a[i], b[i])) return 1;
        if (apply_pred2<T>(op, b[i], a[i])) return 0;
      }
      return na < nb ? 1 : 0;
    }
    case 7:
      for (uint64_t i = 0; i < na; ++i)
        for (uint64_t k = 0; k < nb; ++k)
          if (apply_pred2<T>(MB_EQUAL, a[i], b[k])) return (int64_t)i;
      return none;
    default: return -1;
  }
}

// min_element / max_element / minmax_element: vector.rs:428-481, the
// sequential scans themselves (first minimum; first maximum; minmax moves its
// minimum on !less(x[min], x[i]) -- the last minimum -- and its maximum on
// less(x[max], x[i])).  out[0] (and out[1] for minmax) = index or MB_NONE.
template <class T> int arg_t(int kind, const void* in, uint64_t n, int less, uint32_t* out) {
  const T* x = (const T*)in;
  if (n == 0) {
    out[0] = MB_NONE;
    if (kind == 2) out[1] = MB_NONE;
    return 0;
  }
  uint64_t mn = 0, mx = 0;
  for (uint64_t i = 1; i < n; ++i) {
    switch (kind) {
      case 0: if (apply_pred2<T>(less, x[i], x[mn])) mn = i; break;
      case 1: if (apply_pred2<T>(less, x[mx], x[i])) mx = i; break;
      default:
        if (!apply_pred2<T>(less, x[mn], x[i])) mn = i;
        if (apply_pred2<T>(less, x[mx], x[i])) mx = i;
    }
  }
  out[0] = (uint32_t)(kind == 1 ? mx : mn);
  if (kind == 2) out[1] = (uint32_t)mx;
  return 0;
}

// scatter_reduce: massively/src/api/algorithm/scatter.rs:332-420 with
// core/scatter_reduce.rs:179.  Proposals are taken in input order (the
// stable index sort of the reference keeps it): for every destination d,
// acc = init op v_1 op ... op v_k, then out[d] = out[d] op acc.  Indices past
// the output are skipped.
template <class T> int scatter_reduce_t(const void* vals, const uint32_t* idx, uint64_t n,
                                        int op, const void* init, void* out, uint64_t nout) {
  const T* v = (const T*)vals; T* o = (T*)out;
  const T in = *(const T*)init;
  std::vector<T> acc(nout);
  std::vector<char> has(nout, 0);
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t d = idx[i];
    if (d >= nout) continue;
    acc[d] = has[d] ? apply_op<T>(op, acc[d], v[i]) : apply_op<T>(op, in, v[i]);
    has[d] = 1;
  }
  for (uint64_t d = 0; d < nout; ++d)
    if (has[d]) o[d] = apply_op<T>(op, o[d], acc[d]);
  return 0;
}

// Per-segment queries: verification/oracle/src/seg.rs:171-283, one u32 per
// segment (query ids of include/massively_b200.h MB_SEG_*).
template <class T> int seg_query_t(const void* in, const uint32_t* off, uint64_t nseg, int query,
                                   int op, uint32_t* out) {
  const T* x = (const T*)in;
  for (uint64_t s = 0; s < nseg; ++s) {
    const T* v = x + off[s];
    const uint64_t len = off[s + 1] - off[s];
    uint64_t r = 0;
    switch (query) {
      case MB_SEG_COUNT_IF:
        for (uint64_t i = 0; i < len; ++i) r += apply_flag<T>(op, v[i]) != 0;
        break;
      case MB_SEG_FIND_IF:
        r = len;
        for (uint64_t i = 0; i < len; ++i) if (apply_flag<T>(op, v[i])) { r = i; break; }
        break;
      case MB_SEG_ADJACENT_FIND:
        r = len;
        for (uint64_t i = 0; i + 1 < len; ++i) if (v[i] == v[i + 1]) { r = i; break; }
        break;
      case MB_SEG_IS_SORTED_UNTIL: case MB_SEG_IS_SORTED:
        r = len;
        for (uint64_t i = 1; i < len; ++i) if (apply_pred2<T>(op, v[i], v[i - 1])) { r = i; break; }
        if (query == MB_SEG_IS_SORTED) r = r == len;
        break;
      case MB_SEG_ALL_OF:
        r = 1;
        for (uint64_t i = 0; i < len; ++i) if (!apply_flag<T>(op, v[i])) { r = 0; break; }
        break;
      case MB_SEG_ANY_OF: case MB_SEG_NONE_OF:
        r = 0;
        for (uint64_t i = 0; i < len; ++i) if (apply_flag<T>(op, v[i])) { r = 1; break; }
        if (query == MB_SEG_NONE_OF) r = !r;
        break;
      default: return -1;
    }
    out[s] = (uint32_t)r;
  }
  return 0;
}

// Per-segment transforms: verification/oracle/src/seg.rs:41-46 (reverse),
// 90-107 (adjacent_difference), 109-129 (unique: compared with the last
// kept item), 131-146 (filter), 148-153 (take).  kind: 0 filter, 1 take,
// 2 unique, 3 reverse, 4 adjacent_difference.  Writes values to `out` and
// the new offsets (nseg + 1) to `new_off`; returns the value count.
template <class T> int64_t seg_transform_t(const void* in, const uint32_t* off, uint64_t nseg,
                                           int kind, int param, void* out, uint32_t* new_off) {
  const T* x = (const T*)in;
  T* o = (T*)out;
  uint64_t w = 0;
  new_off[0] = 0;
  for (uint64_t s = 0; s < nseg; ++s) {
    const T* v = x + off[s];
    const uint64_t len = off[s + 1] - off[s];
    const uint64_t start = w;
    for (uint64_t i = 0; i < len; ++i) {
      switch (kind) {
        case 0: if (apply_flag<T>(param, v[i])) o[w++] = v[i]; break;
        case 1: if (i < (uint64_t)param) o[w++] = v[i]; break;
        case 2: if (w == start || !(o[w - 1] == v[i])) o[w++] = v[i]; break;
        case 3: o[w++] = v[len - 1 - i]; break;
        default: o[w++] = i == 0 ? v[0] : apply_op<T>(param, v[i - 1], v[i]); break;
      }
    }
    new_off[s + 1] = (uint32_t)w;
  }
  return (int64_t)w;
}

}  // namespace

extern "C" {

uint32_t orc_pcg_hash32(uint32_t x) { return pcg_hash32(x); }

// random.rs:18-22
uint32_t orc_seed_key(uint64_t seed) {
  uint32_t lo = (uint32_t)seed, hi = (uint32_t)(seed >> 32);
  return pcg_hash32(lo ^ pcg_hash32(hi));
}

// uniform_u32: random.rs:352-356 and 376-385 (index = offset + i, u32 wrap)
void orc_uniform_u32(uint32_t mn, uint32_t mx, uint64_t seed, uint64_t offset, uint64_t n,
                     uint32_t* out) {
  uint32_t key = orc_seed_key(seed);
  uint32_t span = mx - mn;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t v = pcg_hash32((uint32_t)(offset + i) ^ key ^ 0u);
    out[i] = span == 0xffffffffu ? v : mn + v % (span + 1u);
  }
}

// uniform_u64: random.rs:343-348 and 387-396
void orc_uniform_u64(uint64_t mn, uint64_t mx, uint64_t seed, uint64_t offset, uint64_t n,
                     uint64_t* out) {
  uint32_t key = orc_seed_key(seed);
  uint64_t span = mx - mn;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t idx = (uint32_t)(offset + i);
    uint64_t lo = pcg_hash32(idx ^ key ^ 0u);
    uint64_t hi = pcg_hash32(idx ^ key ^ 0x9e3779b9u);
    uint64_t v = lo | (hi << 32);
    out[i] = span == ~0ull ? v : mn + v % (span + 1ull);
  }
}

// Host N(0,1) samples: Box-Muller in f64 on two PCG streams (open unit
// interval), rounded to f32.  The device normal_f32 of random.rs:398-405
// depends on device ln/cos and is not reproducible on a CPU, so workloads
// generate normals here once and upload the same bytes everywhere.
void orc_normal_f32(uint64_t seed, uint64_t offset, uint64_t n, float* out) {
  uint32_t key = orc_seed_key(seed);
  const double two_pi = 6.283185307179586476925286766559;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t idx = (uint32_t)(offset + i);
    double u1 = ((double)(pcg_hash32(idx ^ key) >> 8) + 0.5) * (1.0 / 16777216.0);
    double u2 = ((double)(pcg_hash32(idx ^ key ^ 0x9e3779b9u) >> 8) + 0.5) * (1.0 / 16777216.0);
    out[i] = (float)(std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2));
  }
}

int orc_reduce(int dt, const void* in, uint64_t n, int op, const void* init, void* out) {
  ORC_DISPATCH(dt, reduce_t, in, n, op, init, out);
  return -1;
}
int orc_inclusive_scan(int dt, const void* in, uint64_t n, int op, void* out) {
  ORC_DISPATCH(dt, inclusive_scan_t, in, n, op, out);
  return -1;
}
int orc_exclusive_scan(int dt, const void* in, uint64_t n, int op, const void* init, void* out) {
  ORC_DISPATCH(dt, exclusive_scan_t, in, n, op, init, out);
  return -1;
}
int64_t orc_copy_where(const void* in, uint64_t n, uint64_t width, const uint32_t* stencil,
                       void* out) {
  return (int64_t)compact_rows(in, n, width, stencil, true, out);
}
int64_t orc_remove_where(const void* in, uint64_t n, uint64_t width, const uint32_t* stencil,
                         void* out) {
  return (int64_t)compact_rows(in, n, width, stencil, false, out);
}
int64_t orc_partition(int dt, const void* in, uint64_t n, int pred, void* out) {
  ORC_DISPATCH(dt, partition_t, in, n, pred, out);
  return -1;
}
// gather / scatter: vector.rs:285-311 (rows of `width` bytes)
void orc_gather(const void* src, uint64_t width, const uint32_t* idx, const uint32_t* stencil,
                uint64_t n, void* out) {
  for (uint64_t i = 0; i < n; ++i)
    if (!stencil || stencil[i])
      std::memcpy((uint8_t*)out + i * width, (const uint8_t*)src + (uint64_t)idx[i] * width, width);
}
// replace_where (verification/oracle/src/vector.rs:277-283): out[i] = value
// where stencil[i] != 0.  transform_where (vector.rs:20-31) is the same loop
// over the operator's results: out[i] = src[i] where stencil[i] != 0, with
// `src` already holding op(input) (orc_masked_copy).
void orc_replace_where(const void* value, uint64_t width, const uint32_t* stencil, uint64_t n,
                       void* out) {
  for (uint64_t i = 0; i < n; ++i)
    if (stencil[i] != 0) std::memcpy((uint8_t*)out + i * width, value, width);
}
void orc_masked_copy(const void* src, uint64_t width, const uint32_t* stencil, uint64_t n,
                     void* out) {
  for (uint64_t i = 0; i < n; ++i)
    if (stencil[i] != 0)
      std::memcpy((uint8_t*)out + i * width, (const uint8_t*)src + i * width, width);
}
void orc_scatter(const void* src, uint64_t width, const uint32_t* idx, const uint32_t* stencil,
                 uint64_t n, void* out) {
  for (uint64_t i = 0; i < n; ++i)
    if (!stencil || stencil[i])
      std::memcpy((uint8_t*)out + (uint64_t)idx[i] * width, (const uint8_t*)src + i * width, width);
}
int orc_sort_perm(int dt, const void* keys, uint64_t n, int less, uint32_t* perm) {
  ORC_DISPATCH(dt, sort_perm_t, keys, n, less, perm);
  return -1;
}
// Radix order of up to three key columns, left column primary
// (massively/src/core/radix.rs:500-531): a stable sort under the
// lexicographic total order of the encoded keys.
int orc_radix_perm(int nkeys, const int* dts, const void* const* cols, uint64_t n, uint32_t* perm) {
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  auto enc = [&](int c, size_t i) -> uint64_t {
    const void* p = cols[c];
    switch (dts[c]) {
      case MB_U8: return radix_encode<uint8_t>(((const uint8_t*)p)[i]);
      case MB_U16: return radix_encode<uint16_t>(((const uint16_t*)p)[i]);
      case MB_U32: return radix_encode<uint32_t>(((const uint32_t*)p)[i]);
      case MB_U64: return radix_encode<uint64_t>(((const uint64_t*)p)[i]);
      case MB_I8: return radix_encode<int8_t>(((const int8_t*)p)[i]);
      case MB_I16: return radix_encode<int16_t>(((const int16_t*)p)[i]);
      case MB_I32: return radix_encode<int32_t>(((const int32_t*)p)[i]);
      case MB_I64: return radix_encode<int64_t>(((const int64_t*)p)[i]);
      case MB_F32: return radix_encode<float>(((const float*)p)[i]);
      case MB_F64: return radix_encode<double>(((const double*)p)[i]);
    }
    return 0;
  };
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    for (int c = 0; c < nkeys; ++c) {
      uint64_t a = enc(c, x), b = enc(c, y);
      if (a != b) return a < b;
    }
    return false;
  });
  for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)order[i];
  return 0;
}
// The same order for one key column at full benchmark sizes, on `threads`
// host threads.  A stable sort's result is unique: it is the sort by
// (encoded key, input index), which has no ties.  So the items are sorted as
// (encoded key, index) pairs -- in chunks, one per thread, then merged
// pairwise -- and the permutation equals orc_radix_perm's exactly.
int orc_radix_perm_par(int dt, const void* col, uint64_t n, int threads, uint32_t* perm) {
  if (n > 0xFFFFFFFFull) return -1;
  if (threads < 1) threads = 1;
  std::vector<std::pair<uint64_t, uint32_t>> v(n), w(n);
  auto enc = [&](uint64_t i) -> uint64_t {
    switch (dt) {
      case MB_U32: return radix_encode<uint32_t>(((const uint32_t*)col)[i]);
      case MB_U64: return radix_encode<uint64_t>(((const uint64_t*)col)[i]);
      case MB_I32: return radix_encode<int32_t>(((const int32_t*)col)[i]);
      case MB_I64: return radix_encode<int64_t>(((const int64_t*)col)[i]);
      case MB_F32: return radix_encode<float>(((const float*)col)[i]);
      case MB_F64: return radix_encode<double>(((const double*)col)[i]);
    }
    return 0;
  };
  if (dt != MB_U32 && dt != MB_U64 && dt != MB_I32 && dt != MB_I64 && dt != MB_F32 && dt != MB_F64)
    return -1;
  std::vector<uint64_t> bounds;
  for (int t = 0; t <= threads; ++t) bounds.push_back(n * (uint64_t)t / (uint64_t)threads);
  {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        for (uint64_t i = bounds[t]; i < bounds[t + 1]; ++i) v[i] = {enc(i), (uint32_t)i};
        std::sort(v.begin() + bounds[t], v.begin() + bounds[t + 1]);
      });
    for (auto& th : pool) th.join();
  }
  // pairwise merges of neighbouring sorted runs until one is left
  while (bounds.size() > 2) {
    std::vector<uint64_t> next;
    std::vector<std::thread> pool;
    for (size_t r = 0; r + 1 < bounds.size(); r += 2) {
      const uint64_t a = bounds[r], b = bounds[r + 1];
      const uint64_t c = r + 2 < bounds.size() ? bounds[r + 2] : b;
      next.push_back(a);
      pool.emplace_back([&, a, b, c] {
        std::merge(v.begin() + a, v.begin() + b, v.begin() + b, v.begin() + c, w.begin() + a);
      });
    }
    next.push_back(n);
    for (auto& th : pool) th.join();
    v.swap(w);
    bounds.swap(next);
  }
  for (uint64_t i = 0; i < n; ++i) perm[i] = v[i].second;
  return 0;
}
int orc_run_heads(int kdt, const void* keys, uint64_t n, int key_eq, uint8_t* heads) {
  ORC_DISPATCH(kdt, run_heads_t, keys, n, key_eq, heads);
  return -1;
}
int orc_adjacent_heads(int kdt, const void* keys, uint64_t n, int key_eq, uint8_t* heads) {
  ORC_DISPATCH(kdt, adjacent_heads_t, keys, n, key_eq, heads);
  return -1;
}
int64_t orc_runs_reduce(int vdt, const void* vals, uint64_t n, const uint8_t* heads, int op,
                        const void* init, void* out) {
  ORC_DISPATCH(vdt, runs_reduce_t, vals, n, heads, op, init, out);
  return -1;
}
// reduce_by_key for u32 keys and u32 values: the literal restatement of
// vector.rs:144-174 (kept beside the heads/runs split it is checked against).
int64_t orc_reduce_by_key_u32(const uint32_t* k, const uint32_t* v, uint64_t n, int op,
                              uint32_t init, uint32_t* ok, uint32_t* ov) {
  return reduce_by_key_kv<uint32_t, uint32_t>(k, v, n, MB_EQUAL, op, init, ok, ov);
}
int orc_scan_by_key(int vdt, const void* vals, uint64_t n, const uint8_t* heads, int op,
                    int exclusive, const void* init, void* out) {
  ORC_DISPATCH(vdt, scan_by_key_heads_t, vals, n, heads, op, exclusive, init, out);
  return -1;
}
int orc_merge_src(int dt, const void* l, uint64_t nl, const void* r, uint64_t nr, int less,
                  uint64_t* src) {
  ORC_DISPATCH(dt, merge_src_t, l, nl, r, nr, less, src);
  return -1;
}
int64_t orc_set_op_src(int dt, const void* l, uint64_t nl, const void* r, uint64_t nr, int less,
                       int mode, uint64_t* src) {
  ORC_DISPATCH(dt, set_op_src_t, l, nl, r, nr, less, mode, src);
  return -1;
}
int orc_bounds(int dt, const void* src, uint64_t n, const void* vals, uint64_t m, int less,
               int upper, uint32_t* out) {
  ORC_DISPATCH(dt, bounds_t, src, n, vals, m, less, upper, out);
  return -1;
}
int orc_scatter_reduce(int dt, const void* vals, const uint32_t* idx, uint64_t n, int op,
                       const void* init, void* out, uint64_t nout) {
  ORC_DISPATCH(dt, scatter_reduce_t, vals, idx, n, op, init, out, nout);
  return -1;
}
int orc_seg_query(int dt, const void* in, const uint32_t* off, uint64_t nseg, int query, int op,
                  uint32_t* out) {
  ORC_DISPATCH(dt, seg_query_t, in, off, nseg, query, op, out);
  return -1;
}
int64_t orc_seg_transform(int dt, const void* in, const uint32_t* off, uint64_t nseg, int kind,
                          int param, void* out, uint32_t* new_off) {
  ORC_DISPATCH(dt, seg_transform_t, in, off, nseg, kind, param, out, new_off);
  return -1;
}
int64_t orc_find(int kind, int dt, const void* a, uint64_t na, const void* b, uint64_t nb,
                 int op) {
  ORC_DISPATCH(dt, find_t, kind, a, na, b, nb, op);
  return -1;
}
int orc_arg(int kind, int dt, const void* in, uint64_t n, int less, uint32_t* out) {
  ORC_DISPATCH(dt, arg_t, kind, in, n, less, out);
  return -1;
}
int64_t orc_unique(int dt, const void* in, uint64_t n, int eq, void* out) {
  ORC_DISPATCH(dt, unique_t, in, n, eq, out);
  return -1;
}
int orc_seg_scan(int dt, const void* in, const uint32_t* off, uint64_t nseg, int op, int exclusive,
                 const void* init, void* out) {
  ORC_DISPATCH(dt, seg_scan_t, in, off, nseg, op, exclusive, init, out);
  return -1;
}
int orc_seg_reduce(int dt, const void* in, const uint32_t* off, uint64_t nseg, int op,
                   const void* init, void* out) {
  ORC_DISPATCH(dt, seg_reduce_t, in, off, nseg, op, init, out);
  return -1;
}
int orc_seg_sort(int dt, const void* in, const uint32_t* off, uint64_t nseg, int less, void* out) {
  ORC_DISPATCH(dt, seg_sort_t, in, off, nseg, less, out);
  return -1;
}
// Segmentation::from_offsets validation (massively/src/seg/segmentation.rs:
// 196-232): non-empty, starts at 0, non-decreasing.  Returns the value count
// or -1 when invalid.
int64_t orc_validate_offsets(const uint32_t* off, uint64_t count) {
  if (count == 0 || off[0] != 0) return -1;
  for (uint64_t i = 1; i < count; ++i) if (off[i] < off[i - 1]) return -1;
  return off[count - 1];
}

// Scale-test input generator of massively's oracle scale tests
// (verification/oracle/tests/vector_scale/common.rs:138-159).
void orc_scale_lcg(uint64_t n, uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i)
    out[i] = (uint32_t)(((uint64_t)i * 1103515245ull + 12345ull) % 1000003ull);
}
void orc_scale_other(uint64_t n, uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i)
    out[i] = (uint32_t)(((uint64_t)i * 1664525ull + 1013904223ull) % 1000003ull);
}

uint64_t orc_dtype_size(int dt) { return dtype_size(dt); }

}  // extern "C"
