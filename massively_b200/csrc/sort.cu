// sort.cu -- routing of vector::radix_sort_by_key / sort / sort_by_key onto
// the onesweep radix kernels (radix.cu).
//
// Direct path: one plain key column of 32- or 64-bit elements in massively's
// radix order and at most one plain 4- or 8-byte value column sort as
// (key, value) pairs in one onesweep pass set.
//
// Permutation path (everything else: up to three key columns, lazy keys,
// narrow element types, several value columns, IEEE `<` on floats, the
// descending comparator): LSD over the key columns, last column first -- an
// encode kernel writes the column's order-preserving unsigned key read
// through the current permutation, and a (key, permutation) pair sort
// refines the permutation; finally every value (and key) column is gathered
// once.  This mirrors massively's right-first column passes
// (massively/src/core/radix.rs:500-531) with 8-bit onesweep passes.
//
// Comparator sorts (massively/src/api/algorithm/ordering.rs:64-76,
// by_key.rs:226-270) with the built-in LESS / GREATER / TOTAL_LESS are
// stable sorts under an order-preserving encoding: for floats LESS treats
// -0 and +0 as equal (canonical zero), GREATER inverts the encoding.  Both
// give exactly the stable order of the comparator for every input without
// NaN (a NaN makes `<` no strict weak order, so the reference's result is
// unspecified there; this library orders NaNs by total order).

#include <algorithm>
#include <utility>
#include <vector>

#include "common.cuh"

namespace mb {

int radix_sort_plain(mb_executor* ex, int kdt, const void* ik, const void* iv, void* ok, void* ov,
                     size_t vsize, uint64_t n, const uint32_t* n_dev = nullptr);
int gather_raw(mb_executor* ex, const void* src, size_t esize, uint64_t nsrc,
               const uint32_t* idx, uint64_t n, void* dst, const uint32_t* n_dev = nullptr);
int materialize(mb_executor* ex, const mb_src& in, void* dst);
int seg_ids_fill(mb_executor* ex, const uint32_t* offsets, uint64_t nseg, uint64_t n,
                 uint32_t* ids, const mb_src* values, int enc, int desc, int ieee,
                 uint64_t* comp);
int seg_decode_u32(mb_executor* ex, const uint64_t* comp, uint64_t n, int enc, int desc,
                   uint32_t* out);
int seg_sort_sized(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                   uint64_t nseg, int enc, int desc, int ieee, uint32_t* out, bool* done);

namespace {

constexpr int kThreads = 256;

enum EncMode : int { kEncTotal = 0, kEncIeee = 1 };

unsigned grid_of(uint64_t n) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g > 148ull * 16) g = 148ull * 16;
  return (unsigned)(g ? g : 1);
}

// out[i] = order-preserving unsigned encoding of view element i
// (inverted for descending order).
// Keys are read as raw bits of their element type (narrow signed types
// sign-extended to 32 bits) and encoded as integers.
template <class U, int ENC>
__global__ void __launch_bounds__(kThreads)
    encode_keys_kernel(Src in, U* out, uint64_t n, int ieee, int desc) {
  constexpr U sign = (U)1 << (sizeof(U) * 8 - 1);
  const uint64_t lim = src_len(in) < n ? src_len(in) : n;  // the view's logical length
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < lim;
       i += (uint64_t)gridDim.x * kThreads) {
    U raw = (U)src_load_bits(in, i);
    if (in.vtype == MB_I8) raw = (U)(uint32_t)(int32_t)(int8_t)raw;
    if (in.vtype == MB_I16) raw = (U)(uint32_t)(int32_t)(int16_t)raw;
    if constexpr (ENC == kEncFloat) {
      if (ieee && (raw & ~sign) == 0) raw = 0;  // -0 == +0 under `<`
    }
    const U u = enc_bits<U, ENC>(raw);
    out[i] = desc ? (U)~u : u;
  }
}

__global__ void __launch_bounds__(kThreads) iota_kernel(uint32_t* out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)kThreads + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * kThreads)
    out[i] = (uint32_t)i;
}

// A column read as stored (no view, no map, no cast); it may carry a device
// length, which the sort honours.
bool is_plain_column(const mb_src& s) {
  return s.kind == MB_SRC_COLUMN && s.map == MB_UN_IDENTITY && s.dtype == s.vtype;
}
bool wide_key_type(int dt) {
  return dt == MB_U32 || dt == MB_I32 || dt == MB_F32 || dt == MB_U64 || dt == MB_I64 ||
         dt == MB_F64;
}

template <class U, int ENC>
int encode_run(mb_executor* ex, const Src& s, void* out, uint64_t n, int ieee, int desc) {
  encode_keys_kernel<U, ENC><<<grid_of(n), kThreads, 0, ex->stream>>>(s, (U*)out, n, ieee, desc);
  MB_CUDA(cudaGetLastError());
  return MB_OK;
}

int encode_keys(mb_executor* ex, const Src& s, int vtype, void* out, uint64_t n, int ieee,
                int desc) {
  switch (compute_type(vtype)) {
    case MB_U32: return encode_run<uint32_t, kEncUnsigned>(ex, s, out, n, ieee, desc);
    case MB_I32: return encode_run<uint32_t, kEncSigned>(ex, s, out, n, ieee, desc);
    case MB_F32: return encode_run<uint32_t, kEncFloat>(ex, s, out, n, ieee, desc);
    case MB_U64: return encode_run<uint64_t, kEncUnsigned>(ex, s, out, n, ieee, desc);
    case MB_I64: return encode_run<uint64_t, kEncSigned>(ex, s, out, n, ieee, desc);
    case MB_F64: return encode_run<uint64_t, kEncFloat>(ex, s, out, n, ieee, desc);
    default: return set_error(MB_ERR_LAUNCH, "unsupported key type");
  }
}

// The permutation path.  `modes[c]` / `descs[c]` per key column.
int permutation_sort(mb_executor* ex, const mb_src* keys, int nk, const int* ieee,
                     const int* desc, const mb_src* values, int nv, const mb_col* out_values,
                     const mb_col* out_keys, uint64_t n, const uint32_t* n_dev) {
  Scratch perm_a, perm_b, ukeys, mat;
  MB_TRY(perm_a.alloc(ex, n * 4));
  MB_TRY(perm_b.alloc(ex, n * 4));
  MB_TRY(ukeys.alloc(ex, n * 8));
  iota_kernel<<<grid_of(n), kThreads, 0, ex->stream>>>(perm_a.as<uint32_t>(), n);
  MB_CUDA(cudaGetLastError());
  uint32_t* cur = perm_a.as<uint32_t>();
  uint32_t* nxt = perm_b.as<uint32_t>();
  // Largest materialisation any non-plain key column needs.
  size_t mat_bytes = 0;
  for (int c = 0; c < nk; ++c)
    if (!is_plain_column(keys[c])) mat_bytes = std::max(mat_bytes, (size_t)n * dtype_size(keys[c].vtype));
  if (mat_bytes) MB_TRY(mat.alloc(ex, mat_bytes));
  for (int c = nk - 1; c >= 0; --c) {
    const void* col = keys[c].data;
    if (!is_plain_column(keys[c])) {
      MB_TRY(materialize(ex, keys[c], mat.ptr));
      col = mat.ptr;
    }
    // View of the key column through the current permutation.
    Src s{};
    s.kind = (c == nk - 1) ? MB_SRC_COLUMN : MB_SRC_PERMUTE;
    s.dtype = s.vtype = keys[c].vtype;
    s.map = MB_UN_IDENTITY;
    s.data = col;
    s.index = cur;
    s.len = n;
    s.len_dev = n_dev;
    MB_TRY(encode_keys(ex, s, keys[c].vtype, ukeys.ptr, n, ieee[c], desc[c]));
    const int udt = dtype_size(compute_type(keys[c].vtype)) == 8 ? MB_U64 : MB_U32;
    MB_TRY(radix_sort_plain(ex, udt, ukeys.ptr, cur, nullptr, nxt, 4, n, n_dev));
    std::swap(cur, nxt);
  }
  // Gather the outputs through the final permutation.
  for (int pass = 0; pass < 2; ++pass) {
    const mb_src* srcs = pass == 0 ? values : keys;
    const mb_col* outs = pass == 0 ? out_values : out_keys;
    const int cnt = pass == 0 ? nv : (out_keys ? nk : 0);
    for (int c = 0; c < cnt; ++c) {
      const mb_src& s = srcs[c];
      const void* col = s.data;
      Scratch tmp;
      if (!is_plain_column(s)) {
        MB_TRY(tmp.alloc(ex, n * dtype_size(s.vtype)));
        MB_TRY(materialize(ex, s, tmp.ptr));
        col = tmp.ptr;
      }
      MB_TRY(gather_raw(ex, col, dtype_size(s.vtype), n, cur, n, outs[c].data, n_dev));
    }
  }
  return MB_OK;
}

int validate_sort(mb_executor* ex, const mb_src* keys, int nk, const mb_src* values, int nv,
                  const mb_col* out_values, const mb_col* out_keys, uint64_t* n_out) {
  MB_TRY(check_exec(ex));
  if (nk < 1 || nk > 3) return set_error(MB_ERR_LAUNCH, "radix keys take 1 to 3 columns");
  if (nv < 0 || nv > 12) return set_error(MB_ERR_LAUNCH, "values take 0 to 12 columns");
  if (!keys) return set_error(MB_ERR_UNBOUND_COLUMN, "missing keys");
  const uint64_t n = keys[0].len;
  for (int c = 0; c < nk; ++c) {
    MB_TRY(check_src(ex, &keys[c], "keys"));
    if (keys[c].len != n) return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n, keys[c].len);
    if (dtype_size(keys[c].vtype) == 0) return set_error(MB_ERR_LAUNCH, "bad key type");
  }
  for (int c = 0; c < nv; ++c) {
    MB_TRY(check_src(ex, &values[c], "values"));
    if (values[c].len != n)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n, values[c].len);
    MB_TRY(check_col(ex, out_values[c], "output"));
    if (out_values[c].len < n)
      return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out_values[c].len);
    if (dtype_size(out_values[c].dtype) != dtype_size(values[c].vtype))
      return set_error(MB_ERR_LAUNCH, "value output element type differs");
  }
  if (out_keys) {
    for (int c = 0; c < nk; ++c) {
      MB_TRY(check_col(ex, out_keys[c], "key output"));
      if (out_keys[c].len < n)
        return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out_keys[c].len);
      if (dtype_size(out_keys[c].dtype) != dtype_size(keys[c].vtype))
        return set_error(MB_ERR_LAUNCH, "key output element type differs");
    }
  }
  *n_out = n;
  return MB_OK;
}

int sort_general(mb_executor* ex, const mb_src* keys, int nk, const int* ieee, const int* desc,
                 const mb_src* values, int nv, const mb_col* out_values, const mb_col* out_keys) {
  uint64_t n = 0;
  MB_TRY(validate_sort(ex, keys, nk, values, nv, out_values, out_keys, &n));
  if (n == 0 || (nv == 0 && !out_keys)) return MB_OK;
  bool natural = true;
  for (int c = 0; c < nk; ++c) natural = natural && !ieee[c] && !desc[c];
  const bool direct = nk == 1 && natural && is_plain_column(keys[0]) &&
                      wide_key_type(keys[0].vtype) &&
                      (nv == 0 || (nv == 1 && is_plain_column(values[0]) &&
                                   (dtype_size(values[0].vtype) == 4 ||
                                    dtype_size(values[0].vtype) == 8)));
  // A device length (a count left on the device by copy_where and the like)
  // bounds every kernel on the device; the host sizes by capacity.
  const uint32_t* n_dev = nullptr;
  for (int c = 0; c < nk && !n_dev; ++c) n_dev = keys[c].len_dev;
  for (int c = 0; c < nv && !n_dev; ++c) n_dev = values[c].len_dev;
  if (direct) {
    const size_t vs = nv ? dtype_size(values[0].vtype) : 0;
    return radix_sort_plain(ex, keys[0].vtype, keys[0].data, nv ? values[0].data : nullptr,
                            out_keys ? out_keys[0].data : nullptr,
                            nv ? out_values[0].data : nullptr, vs, n, n_dev);
  }
  return permutation_sort(ex, keys, nk, ieee, desc, values, nv, out_values, out_keys, n, n_dev);
}

void comparator_mode(int less, int vtype, int* ieee, int* desc) {
  *ieee = (less == MB_LESS || less == MB_GREATER) && dtype_is_float(vtype);
  *desc = less == MB_GREATER;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" {

int mb_radix_sort_by_key(mb_executor* ex, const mb_src* keys, int nkeys, const mb_src* values,
                         int nvals, const mb_col* out_values, const mb_col* out_keys) {
  int ieee[3] = {0, 0, 0}, desc[3] = {0, 0, 0};
  return sort_general(ex, keys, nkeys, ieee, desc, values, nvals, out_values, out_keys);
}

int mb_sort(mb_executor* ex, const mb_src* keys, int less, mb_col out) {
  MB_TRY(check_exec(ex));
  if (!keys) return set_error(MB_ERR_UNBOUND_COLUMN, "missing keys");
  if (less < MB_LESS || less > MB_TOTAL_LESS)
    return set_error(MB_ERR_LAUNCH, "sort takes LESS, GREATER or TOTAL_LESS");
  int ieee, desc;
  comparator_mode(less, keys->vtype, &ieee, &desc);
  return sort_general(ex, keys, 1, &ieee, &desc, nullptr, 0, nullptr, &out);
}

// ForEachSegment(Sort(less)) (massively/src/seg/mod.rs:379-425).  4-byte
// values are sorted where they lie, in shared memory (segsort.cu).  Other
// types, and 4-byte calls with a segment too long for one CTA, take a stable
// global radix sort of (segment id, value) pairs -- the segment id primary --
// in place of massively's two global comparison sorts and three permutation
// applications.  Segment ids need ceil(log2(segments)/8) digit passes;
// constant high digits are skipped by the onesweep plan.
int mb_seg_sort(mb_executor* ex, const mb_src* values, const uint32_t* offsets,
                uint64_t segment_count, int less, mb_col out) {
  MB_TRY(check_exec(ex));
  MB_TRY(check_src(ex, values, "values"));
  MB_TRY(check_col(ex, out, "output"));
  const uint64_t n = values->len;
  if (out.len < n) return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n, out.len);
  if (less < MB_LESS || less > MB_TOTAL_LESS)
    return set_error(MB_ERR_LAUNCH, "seg sort takes LESS, GREATER or TOTAL_LESS");
  if (n == 0) return MB_OK;
  const int vt = values->vtype;
  if (dtype_size(vt) == 4 && dtype_size(out.dtype) == 4 && (vt == MB_U32 || vt == MB_I32 ||
                                                            vt == MB_F32)) {
    // 4-byte values: one radix sort of 64-bit keys (segment id << 32 |
    // order-preserving bits of the value); the id's constant high digits
    // are skipped by the onesweep plan.  Where the encoding is a bijection
    // the sorted keys decode back to the values; under `<` / `>` on floats
    // (-0 and +0 tie) the original bits ride along as the sort's values.
    int ieee = 0, desc = 0;
    comparator_mode(less, vt, &ieee, &desc);
    const int enc = vt == MB_U32 ? 0 : vt == MB_I32 ? 1 : 2;
    bool done = false;
    MB_TRY(seg_sort_sized(ex, values, offsets, segment_count, enc, desc, ieee,
                          (uint32_t*)out.data, &done));
    if (done) return MB_OK;
    Scratch comp, sorted;
    MB_TRY(comp.alloc(ex, n * 8));
    MB_TRY(sorted.alloc(ex, n * 8));
    MB_TRY(seg_ids_fill(ex, offsets, segment_count, n, nullptr, values, enc, desc, ieee,
                        comp.as<uint64_t>()));
    if (!ieee) {
      MB_TRY(radix_sort_plain(ex, MB_U64, comp.ptr, nullptr, sorted.ptr, nullptr, 0, n));
      return seg_decode_u32(ex, sorted.as<uint64_t>(), n, enc, desc, (uint32_t*)out.data);
    }
    const void* raw = values->data;
    Scratch mat;
    if (!is_plain_column(*values)) {
      MB_TRY(mat.alloc(ex, n * 4));
      MB_TRY(materialize(ex, *values, mat.ptr));
      raw = mat.ptr;
    }
    return radix_sort_plain(ex, MB_U64, comp.ptr, raw, sorted.ptr, out.data, 4, n);
  }
  Scratch ids, ids_out;
  MB_TRY(ids.alloc(ex, n * 4));
  MB_TRY(ids_out.alloc(ex, n * 4));
  MB_TRY(mb_segmentation_segment_ids(ex, offsets, segment_count, ids.as<uint32_t>(), n));
  mb_src keys[2];
  keys[0] = mb_src{};
  keys[0].kind = MB_SRC_COLUMN;
  keys[0].dtype = keys[0].vtype = MB_U32;
  keys[0].map = MB_UN_IDENTITY;
  keys[0].data = ids.ptr;
  keys[0].len = n;
  keys[1] = *values;
  int ieee[2] = {0, 0}, desc[2] = {0, 0};
  comparator_mode(less, values->vtype, &ieee[1], &desc[1]);
  mb_col outs[2];
  outs[0] = mb_col{};
  outs[0].data = ids_out.ptr;
  outs[0].dtype = MB_U32;
  outs[0].len = n;
  outs[1] = out;
  return sort_general(ex, keys, 2, ieee, desc, nullptr, 0, nullptr, outs);
}

int mb_sort_by_key(mb_executor* ex, const mb_src* keys, int less, const mb_src* values, int nvals,
                   const mb_col* out_keys, const mb_col* out_values) {
  MB_TRY(check_exec(ex));
  if (!keys) return set_error(MB_ERR_UNBOUND_COLUMN, "missing keys");
  if (less < MB_LESS || less > MB_TOTAL_LESS)
    return set_error(MB_ERR_LAUNCH, "sort_by_key takes LESS, GREATER or TOTAL_LESS");
  int ieee, desc;
  comparator_mode(less, keys->vtype, &ieee, &desc);
  return sort_general(ex, keys, 1, &ieee, &desc, values, nvals, out_values, out_keys);
}

}  // extern "C"
