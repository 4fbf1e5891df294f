// search.cu -- vectorised lower_bound / upper_bound over a sorted source.
//
// massively (massively/src/api/algorithm/search.rs:81-147, oracle
// verification/oracle/src/vector.rs:404-426) returns, for every value, the
// partition point of the sorted source: the first index whose element is not
// less than the value (lower_bound) or that the value is less than
// (upper_bound).  Here each query is one thread's binary search in two
// levels: first over kSamples evenly spaced source elements held in shared
// memory (gathered once per call by a small kernel into a contiguous
// scratch row, so every block loads them with coalesced reads), then over
// the one source interval between two samples that holds the answer, in
// global memory.  With 4096 samples a 2^24-element source leaves 12 of 24
// probes to global memory.
//
// A plain, 16-byte-aligned source of 4- or 8-byte elements takes a search by
// lines instead (search_lines_kernel): level j holds every B^j-th source
// element (B = 4: one 16-byte load of u32, two of u64), built once per call,
// the top level (up to 64 KB) in shared memory.  Below the top each level
// costs one line read and a count of the line's elements inside the prefix:
// a 4-ary search.  Each load of a warp touches 32 different lines, so what
// bounds the search is the number of load instructions per query: five for a
// 2^24-element u32 source, against twelve dependent 4-byte probes for the
// two-level binary search.  (128-byte lines -- two levels, sixteen loads --
// measured 5.2 ms against 3.7 ms for the binary search.)

#include <algorithm>

#include "common.cuh"
#include "dispatch.cuh"

namespace mb {
namespace {

constexpr int kThreads = 256;
constexpr int kSampleBytes = 16384;  // shared-memory sample row per block

template <class T>
constexpr int samples_of() {
  return kSampleBytes / (int)sizeof(T);
}

template <class T, int LESS>
__device__ __forceinline__ bool less_ct(T a, T b) {
  if constexpr (LESS == MB_GREATER) return b < a;
  else if constexpr (LESS == MB_TOTAL_LESS) return radix_enc<T>(a) < radix_enc<T>(b);
  else return a < b;
}

// Whether `candidate` lies in the prefix that the partition point of
// `value` closes.
template <class T, int LESS, bool UPPER>
__device__ __forceinline__ bool in_prefix(T candidate, T value) {
  if constexpr (UPPER) return !less_ct<T, LESS>(value, candidate);
  else return less_ct<T, LESS>(candidate, value);
}

template <class T, bool PLAIN>
__device__ __forceinline__ T load_at(const Src& s, uint64_t i) {
  if constexpr (PLAIN) return ((const T*)s.data)[i];
  else return src_load<T>(s, i);
}

// samples[k] = source[k * step] for every k with k * step < n.
template <class T, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    search_samples_kernel(Src source, uint64_t step, T* __restrict__ samples) {
  const uint64_t n = src_len(source);
  for (int k = blockIdx.x * kThreads + threadIdx.x; k < samples_of<T>(); k += gridDim.x * kThreads)
    if ((uint64_t)k * step < n) samples[k] = load_at<T, PLAIN>(source, (uint64_t)k * step);
}

template <class T, int LESS, bool UPPER, bool PLAIN>
__global__ void __launch_bounds__(kThreads)
    search_kernel(Src source, Src values, uint64_t step, const T* __restrict__ samples,
                  uint32_t* __restrict__ out) {
  constexpr int S = samples_of<T>();
  __shared__ T s_samp[S];
  const uint64_t n = src_len(source);
  const uint64_t m = src_len(values);
  const int ns = (int)min((uint64_t)S, n == 0 ? 0 : (n - 1) / step + 1);  // samples in use
  for (int k = threadIdx.x; k < ns; k += kThreads) s_samp[k] = samples[k];
  __syncthreads();
  for (uint64_t q = blockIdx.x * (uint64_t)kThreads + threadIdx.x; q < m;
       q += (uint64_t)gridDim.x * kThreads) {
    const T v = load_at<T, PLAIN>(values, q);
    // c = samples inside the prefix (they are sorted, so a prefix of them)
    int lo = 0, hi = ns;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (in_prefix<T, LESS, UPPER>(s_samp[mid], v)) lo = mid + 1;
      else hi = mid;
    }
    uint64_t ans;
    if (lo == 0) {
      ans = 0;  // the first element already closes the prefix (or n == 0)
    } else {
      // The answer lies in ((lo-1)*step, min(lo*step, n)]: the sample at
      // lo*step (if any) is outside the prefix.
      uint64_t a = (uint64_t)(lo - 1) * step + 1;
      uint64_t b = min((uint64_t)lo * step, n);
      while (a < b) {
        const uint64_t mid = (a + b) >> 1;
        if (in_prefix<T, LESS, UPPER>(load_at<T, PLAIN>(source, mid), v)) a = mid + 1;
        else b = mid;
      }
      ans = a;
    }
    out[q] = (uint32_t)ans;
  }
}

// ---------------------------------------------------------- by lines --

constexpr int kLineThreads = 512;
constexpr int kLineTopBytes = 65536;  // shared-memory top level
constexpr int kMaxLevels = 16;

template <class T>
constexpr int line_of() {
  return 4;
}
template <class T>
constexpr int line_bytes() {
  return line_of<T>() * (int)sizeof(T);
}
// Top-level entries: a complete binary tree of 2^h - 1 nodes fits the
// shared-memory row (index 0 unused).
template <class T>
constexpr int top_of() {
  return kLineTopBytes / (int)sizeof(T) - 1;
}

// Level j (1..levels) holds len[j] = ceil(n / B^j) elements at off[j] of the
// level scratch (off[j] a multiple of B, so every line is 16-byte aligned);
// level `levels` is the top, held in shared memory.  levels == 0: the source
// itself is the top.
struct LinePlan {
  int levels;
  uint64_t len[kMaxLevels + 1];
  uint64_t off[kMaxLevels + 1];
};

template <class T>
__global__ void __launch_bounds__(kThreads)
    search_levels_kernel(const T* __restrict__ src, LinePlan lp, T* __restrict__ lv) {
  constexpr int B = line_of<T>();
  for (uint64_t t = blockIdx.x * (uint64_t)kThreads + threadIdx.x; t < lp.len[1];
       t += (uint64_t)gridDim.x * kThreads) {
    const T v = src[t * B];
    lv[lp.off[1] + t] = v;
    uint64_t u = t;
    for (int j = 2; j <= lp.levels; ++j) {
      if (u % B) break;
      u /= B;
      lv[lp.off[j] + u] = v;
    }
  }
}

// How many of the B elements of one line (starting at element `first` of a
// level of `len` elements) are inside the prefix; elements past `len` are not.
template <class T, int LESS, bool UPPER>
__device__ __forceinline__ int line_count(const T* __restrict__ line, uint64_t first, uint64_t len,
                                          T v) {
  constexpr int B = line_of<T>();
  int c = 0;
  if (first + B <= len) {
    uint4 raw[line_bytes<T>() / 16];
#pragma unroll
    for (int i = 0; i < line_bytes<T>() / 16; ++i)
      raw[i] = __ldg(reinterpret_cast<const uint4*>(line) + i);
    T e[B];
    memcpy(e, raw, line_bytes<T>());
#pragma unroll
    for (int u = 0; u < B; ++u) c += in_prefix<T, LESS, UPPER>(e[u], v) ? 1 : 0;
  } else {
    for (uint64_t u = 0; first + u < len; ++u) c += in_prefix<T, LESS, UPPER>(line[u], v) ? 1 : 0;
  }
  return c;
}

template <class T, int LESS, bool UPPER, bool PLAIN_V>
__global__ void __launch_bounds__(kLineThreads)
    search_lines_kernel(const T* __restrict__ src, uint64_t n, Src values, LinePlan lp,
                        const T* __restrict__ lv, uint32_t* __restrict__ out) {
  constexpr int B = line_of<T>();
  extern __shared__ __align__(16) unsigned char sl_raw[];
  T* tree = reinterpret_cast<T*>(sl_raw);
  const int k = lp.levels;
  const T* topg = k ? lv + lp.off[k] : src;
  const int ns = (int)(k ? lp.len[k] : n);
  // The top level as a complete binary search tree in breadth-first order
  // (node i's children at 2i and 2i + 1): a search step of every lane of a
  // warp reads the same tree level, a run of consecutive words, where a
  // binary search over the sorted row has every lane's probe a multiple of a
  // power of two apart (one bank) for the first nine steps.  Nodes past the
  // last element repeat it, and the count is capped at ns.
  int h = 0;
  while ((1 << h) - 1 < ns) ++h;
  for (int i = 1 + threadIdx.x; i < (1 << h); i += kLineThreads) {
    const int l = 31 - __clz(i);
    const int r = (((i - (1 << l)) * 2 + 1) << (h - l - 1)) - 1;  // its rank in the row
    tree[i] = topg[min(r, ns - 1)];
  }
  __syncthreads();
  const uint64_t m = src_len(values);
  for (uint64_t q = blockIdx.x * (uint64_t)kLineThreads + threadIdx.x; q < m;
       q += (uint64_t)gridDim.x * kLineThreads) {
    T v;
    if constexpr (PLAIN_V) v = __ldcs((const T*)values.data + q);  // streamed past L2
    else v = load_at<T, PLAIN_V>(values, q);
    int i = 1;
    for (int l = 0; l < h; ++l) i = 2 * i + (in_prefix<T, LESS, UPPER>(tree[i], v) ? 1 : 0);
    const int lo = min(i - (1 << h), ns);  // top elements inside the prefix
    uint64_t ans = (uint64_t)lo;
    if (k > 0 && lo > 0) {
      // The prefix ends inside block lo - 1 of the top level; each level
      // below narrows it to one of the block's B sub-blocks.
      uint64_t t = (uint64_t)lo - 1;
      for (int j = k - 1; j >= 0; --j) {
        const uint64_t first = t * B;
        const T* base = j ? lv + lp.off[j] : src;
        const int c = line_count<T, LESS, UPPER>(base + first, first, j ? lp.len[j] : n, v);
        if (j) t = first + (uint64_t)c - 1;
        else ans = first + (uint64_t)c;
      }
    } else if (k > 0) {
      ans = 0;
    }
    __stcs(out + q, (uint32_t)ans);
  }
}

template <class T, int LESS, bool UPPER, bool PLAIN_V>
int search_lines_launch(mb_executor* ex, const mb_src& source, const mb_src& values,
                        uint32_t* out) {
  constexpr int B = line_of<T>();
  constexpr int S = top_of<T>();
  const uint64_t n = source.len, m = values.len;
  LinePlan lp{};
  uint64_t span = 1, total = 0;
  while ((n + span - 1) / span > (uint64_t)S) {
    span *= B;
    ++lp.levels;
    if (lp.levels > kMaxLevels) return set_error(MB_ERR_LAUNCH, "search levels");
    lp.len[lp.levels] = (n + span - 1) / span;
    lp.off[lp.levels] = total;
    total += (lp.len[lp.levels] + B - 1) / B * B;
  }
  Scratch levels;
  if (lp.levels > 0) {
    MB_TRY(levels.alloc(ex, total * sizeof(T)));
    const unsigned g = (unsigned)std::min<uint64_t>((lp.len[1] + kThreads - 1) / kThreads, 148ull * 16);
    search_levels_kernel<T><<<std::max(1u, g), kThreads, 0, ex->stream>>>(
        (const T*)source.data, lp, levels.as<T>());
    MB_CUDA(cudaGetLastError());
  }
  const int ns = (int)(lp.levels ? lp.len[lp.levels] : n);
  int h = 0;
  while ((1 << h) - 1 < ns) ++h;
  const size_t smem = (size_t)(1 << h) * sizeof(T);
  auto kern = search_lines_kernel<T, LESS, UPPER, PLAIN_V>;
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kLineTopBytes));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t blocks =
      std::min<uint64_t>((m + kLineThreads - 1) / kLineThreads, (uint64_t)sms * 3);
  kern<<<(unsigned)std::max<uint64_t>(1, blocks), kLineThreads, smem, ex->stream>>>(
      (const T*)source.data, n, to_src(values), lp, lp.levels ? levels.as<T>() : nullptr, out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T, int LESS, bool UPPER, bool PLAIN>
int search_launch(mb_executor* ex, const mb_src& source, const mb_src& values, uint32_t* out) {
  constexpr int S = samples_of<T>();
  const uint64_t n = source.len, m = values.len;
  const uint64_t step = std::max<uint64_t>(1, (n + S - 1) / S);
  Scratch samples;
  MB_TRY(samples.alloc(ex, (size_t)S * sizeof(T)));
  const Src s = to_src(source), v = to_src(values);
  search_samples_kernel<T, PLAIN><<<(S + kThreads - 1) / kThreads, kThreads, 0, ex->stream>>>(
      s, step, samples.as<T>());
  MB_CUDA(cudaGetLastError());
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t blocks = std::min<uint64_t>((m + kThreads - 1) / kThreads, (uint64_t)sms * 8);
  search_kernel<T, LESS, UPPER, PLAIN><<<(unsigned)std::max<uint64_t>(1, blocks), kThreads, 0,
                                         ex->stream>>>(s, v, step, samples.as<T>(), out);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

template <class T>
int search_run(mb_executor* ex, const mb_src& source, const mb_src& values, int less, bool upper,
               uint32_t* out) {
  const int ct = DTypeOf<T>::value;
  const bool plain = src_plain(source, ct) && src_plain(values, ct);
  // By lines: a plain, 16-byte-aligned source with no device length.
  const bool lines = src_plain(source, ct) && source.len_dev == nullptr &&
                     (uintptr_t)source.data % 16 == 0;
  const bool pv = src_plain(values, ct);
#define MB_SEARCH_LINES(L)                                                                  \
  do {                                                                                      \
    if (upper)                                                                              \
      return pv ? search_lines_launch<T, L, true, true>(ex, source, values, out)           \
                : search_lines_launch<T, L, true, false>(ex, source, values, out);         \
    return pv ? search_lines_launch<T, L, false, true>(ex, source, values, out)            \
              : search_lines_launch<T, L, false, false>(ex, source, values, out);          \
  } while (0)
  if (lines && ex->tune[MB_TUNE_SEARCH] != 1) {
    switch (less) {
      case MB_GREATER: MB_SEARCH_LINES(MB_GREATER);
      case MB_TOTAL_LESS: MB_SEARCH_LINES(MB_TOTAL_LESS);
      default: MB_SEARCH_LINES(MB_LESS);
    }
  }
#undef MB_SEARCH_LINES
#define MB_SEARCH(L)                                                                        \
  do {                                                                                      \
    if (upper)                                                                              \
      return plain ? search_launch<T, L, true, true>(ex, source, values, out)               \
                   : search_launch<T, L, true, false>(ex, source, values, out);             \
    return plain ? search_launch<T, L, false, true>(ex, source, values, out)                \
                 : search_launch<T, L, false, false>(ex, source, values, out);              \
  } while (0)
  switch (less) {
    case MB_GREATER: MB_SEARCH(MB_GREATER);
    case MB_TOTAL_LESS: MB_SEARCH(MB_TOTAL_LESS);
    default: MB_SEARCH(MB_LESS);
  }
#undef MB_SEARCH
}

int search_entry(mb_executor* ex, const mb_src* source, const mb_src* values, int less, mb_col out,
                 bool upper) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, source, "source"));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_col(ex, out, "output"));
  if (compute_type(source->vtype) != compute_type(values->vtype))
    return set_error(MB_ERR_LAUNCH, "source and values element types differ");
  if (less < MB_LESS || less > MB_TOTAL_LESS)
    return set_error(MB_ERR_LAUNCH, "search takes LESS, GREATER or TOTAL_LESS");
  if (out.dtype != MB_U32 && out.dtype != MB_I32)
    return set_error(MB_ERR_LAUNCH, "bounds are MIndex (u32)");
  MB_TRY(check_len_u32(source->len));
  if (out.len < values->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than the values", values->len,
                     out.len);
  if (values->len == 0) return MB_OK;
  MB_DISPATCH_CTYPE(compute_type(source->vtype), search_run, ex, *source, *values, less, upper,
                    (uint32_t*)out.data);
  return set_error(MB_ERR_LAUNCH, "unsupported element type");
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_lower_bound(mb_executor* ex, const mb_src* source, const mb_src* values, int less,
                   mb_col out) {
  return search_entry(ex, source, values, less, out, false);
}

int mb_upper_bound(mb_executor* ex, const mb_src* source, const mb_src* values, int less,
                   mb_col out) {
  return search_entry(ex, source, values, less, out, true);
}

}  // extern "C"
