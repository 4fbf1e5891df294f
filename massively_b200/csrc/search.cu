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
