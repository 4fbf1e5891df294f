// user_ops.cu -- user-written operators, compiled at run time with NVRTC.
//
// massively's operators are user `#[cube]` trait impls (op::ReductionOp,
// op::UnaryOp: massively/src/core/op.rs:33-96, core/reduce.rs:63-66) that
// CubeCL monomorphises into the algorithm kernels.  The built-in ids of
// mb_op / mb_unary cover the common ones; this file takes the rest as CUDA C
// source: a `__device__` function over the element type `T` (binary
// operators) or `In` -> `Out` (maps), spliced into a small set of kernels
// (reduce, inclusive / exclusive scan, map) compiled for sm_100a by NVRTC
// and loaded with the CUDA library API.
//
// The kernels are plain and in-order:
//   reduce   each block folds a grid-strided share (the operator must be
//            associative and commutative, as massively requires,
//            core/reduce.rs:35-38), a second launch folds the block partials
//            in block order, then `init op total`;
//   scan     three launches -- per-tile scans of 2048 items (each thread
//            scans 8 consecutive items, then a block scan of the thread
//            totals, all in index order), one block scanning the tile totals,
//            and a pass applying each tile's prefix -- so the operator needs
//            to be associative only;
//   map      one item per thread, grid-strided.
// Inputs are plain device columns of the compiled element type.
//
// NVRTC is opened with dlopen on first use, so the library loads (and every
// built-in path works) where it is absent; a compile error is returned as
// MB_ERR_LAUNCH with NVRTC's log as the message.

#include <dlfcn.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace mb {
namespace {

// ------------------------------------------------------------------ NVRTC --

typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;

struct Nvrtc {
  bool ok = false;
  std::string why;
  nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*,
                          const char* const*) = nullptr;
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*) = nullptr;
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*) = nullptr;
  nvrtcResult_t (*log)(nvrtcProgram_t, char*) = nullptr;
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*) = nullptr;
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char*) = nullptr;
  nvrtcResult_t (*destroy)(nvrtcProgram_t*) = nullptr;
};

Nvrtc& nvrtc() {
  static Nvrtc n;
  static std::once_flag once;
  std::call_once(once, [] {
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    void* h = nullptr;
    for (const char* nm : names)
      if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
      n.why = "NVRTC (libnvrtc.so.12) could not be loaded";
      return;
    }
    auto sym = [&](const char* s) { return dlsym(h, s); };
    n.create = (decltype(n.create))sym("nvrtcCreateProgram");
    n.compile = (decltype(n.compile))sym("nvrtcCompileProgram");
    n.log_size = (decltype(n.log_size))sym("nvrtcGetProgramLogSize");
    n.log = (decltype(n.log))sym("nvrtcGetProgramLog");
    n.cubin_size = (decltype(n.cubin_size))sym("nvrtcGetCUBINSize");
    n.cubin = (decltype(n.cubin))sym("nvrtcGetCUBIN");
    n.destroy = (decltype(n.destroy))sym("nvrtcDestroyProgram");
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    if (!n.ok) n.why = "NVRTC is missing an entry point";
  });
  return n;
}

const char* ctype_name(int dt) {
  switch (dt) {
    case MB_U8: return "unsigned char";
    case MB_U16: return "unsigned short";
    case MB_U32: return "unsigned int";
    case MB_U64: return "unsigned long long";
    case MB_I8: return "signed char";
    case MB_I16: return "short";
    case MB_I32: return "int";
    case MB_I64: return "long long";
    case MB_F32: return "float";
    default: return "double";
  }
}

// The kernels the user's function is spliced into.  USER_OP(a, b) is the
// binary operator, USER_MAP(x) the map.
const char* kBinaryKernels = R"MBJ(
#define MBJ_TILE_ITEMS 8
#define MBJ_THREADS 256
extern "C" __global__ void mbj_reduce_partial(const T* in, unsigned long long n, T* part,
                                              unsigned* has) {
  __shared__ T s_v[MBJ_THREADS];
  __shared__ unsigned s_h[MBJ_THREADS];
  T acc;
  unsigned h = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)MBJ_THREADS + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * MBJ_THREADS) {
    acc = h ? USER_OP(acc, in[i]) : in[i];
    h = 1;
  }
  s_v[threadIdx.x] = acc;
  s_h[threadIdx.x] = h;
  __syncthreads();
  for (int d = MBJ_THREADS / 2; d > 0; d >>= 1) {
    if (threadIdx.x < d && s_h[threadIdx.x + d]) {
      s_v[threadIdx.x] = s_h[threadIdx.x] ? USER_OP(s_v[threadIdx.x], s_v[threadIdx.x + d])
                                          : s_v[threadIdx.x + d];
      s_h[threadIdx.x] = 1;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s_v[0];
    has[blockIdx.x] = s_h[0];
  }
}
extern "C" __global__ void mbj_reduce_final(const T* part, const unsigned* has, unsigned parts,
                                            const T* init, T* out) {
  if (threadIdx.x != 0) return;
  T acc = *init;
  for (unsigned b = 0; b < parts; ++b)
    if (has[b]) acc = USER_OP(acc, part[b]);
  *out = acc;
}
// Inclusive scan of each 2048-item tile into `out`; tile totals to `tot`.
extern "C" __global__ void mbj_scan_tiles(const T* in, T* out, unsigned long long n, T* tot) {
  __shared__ T s_t[MBJ_THREADS];
  const unsigned long long base =
      (unsigned long long)blockIdx.x * (MBJ_THREADS * MBJ_TILE_ITEMS) +
      (unsigned long long)threadIdx.x * MBJ_TILE_ITEMS;
  T v[MBJ_TILE_ITEMS];
  int cnt = 0;
  for (int k = 0; k < MBJ_TILE_ITEMS; ++k) {
    if (base + k < n) {
      v[k] = cnt ? USER_OP(v[k - 1], in[base + k]) : in[base + k];
      ++cnt;
    }
  }
  // threads past the end hold no items: they sit at the end of the order
  const int valid = cnt > 0;
  __shared__ int s_c[MBJ_THREADS];
  if (valid) s_t[threadIdx.x] = v[cnt - 1];
  s_c[threadIdx.x] = valid;
  __syncthreads();
  // inclusive Hillis-Steele scan of the thread totals, in thread order
  for (int d = 1; d < MBJ_THREADS; d <<= 1) {
    T x;
    int hx = 0;
    if (threadIdx.x >= d && s_c[threadIdx.x - d] && s_c[threadIdx.x]) {
      x = USER_OP(s_t[threadIdx.x - d], s_t[threadIdx.x]);
      hx = 1;
    }
    __syncthreads();
    if (hx) s_t[threadIdx.x] = x;
    __syncthreads();
  }
  if (threadIdx.x > 0 && valid) {
    const T pre = s_t[threadIdx.x - 1];
    for (int k = 0; k < cnt; ++k) v[k] = USER_OP(pre, v[k]);
  }
  for (int k = 0; k < cnt; ++k) out[base + k] = v[k];
  // the tile total: the last thread with items
  if (valid && (threadIdx.x == MBJ_THREADS - 1 || !s_c[threadIdx.x + 1]))
    tot[blockIdx.x] = s_t[threadIdx.x];
}
// One block: inclusive scan of the tile totals, in order.
extern "C" __global__ void mbj_scan_totals(T* tot, unsigned tiles) {
  __shared__ T s_t[MBJ_THREADS];
  __shared__ T s_carry;
  for (unsigned c = 0; c < tiles; c += MBJ_THREADS) {
    const unsigned i = c + threadIdx.x;
    const int valid = i < tiles;
    if (valid) s_t[threadIdx.x] = tot[i];
    __syncthreads();
    for (int d = 1; d < MBJ_THREADS; d <<= 1) {
      T x;
      int hx = 0;
      if (valid && threadIdx.x >= d) {
        x = USER_OP(s_t[threadIdx.x - d], s_t[threadIdx.x]);
        hx = 1;
      }
      __syncthreads();
      if (hx) s_t[threadIdx.x] = x;
      __syncthreads();
    }
    if (valid) {
      T r = s_t[threadIdx.x];
      if (c > 0) r = USER_OP(s_carry, r);
      tot[i] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned last = (c + MBJ_THREADS < tiles ? c + MBJ_THREADS : tiles) - 1;
      s_carry = tot[last];
    }
    __syncthreads();
  }
}
// Inclusive: out[i] = P(tile - 1) op local[i].  Exclusive (from the local
// inclusive values in `loc`): out[i] = init op global_inclusive[i - 1].
extern "C" __global__ void mbj_scan_apply(const T* loc, T* out, unsigned long long n,
                                          const T* tot, int exclusive, const T* init) {
  const unsigned long long tile_items = MBJ_THREADS * MBJ_TILE_ITEMS;
  for (unsigned long long i = blockIdx.x * (unsigned long long)MBJ_THREADS + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * MBJ_THREADS) {
    if (!exclusive) {
      const unsigned long long t = i / tile_items;
      out[i] = t > 0 ? USER_OP(tot[t - 1], loc[i]) : loc[i];
    } else if (i == 0) {
      out[0] = *init;
    } else {
      const unsigned long long j = i - 1, t = j / tile_items;
      const T g = t > 0 ? USER_OP(tot[t - 1], loc[j]) : loc[j];
      out[i] = USER_OP(*init, g);
    }
  }
}
)MBJ";

// Stable merge sort of (key, index) pairs under USER_LESS(a, b) -- massively's
// comparator sort (core/ordering/sort.rs:54-455: block sorts, then merge
// passes; ties keep input order).  Tiles of MBS_TILE items are sorted in
// shared memory (each thread's 4 items by insertion, then pairwise merges of
// doubling runs); the merge passes then merge runs of width w into 2w, each
// block producing one tile of the output: its merge-path split in the two
// runs (a binary search in global memory), both slices staged in shared
// memory, each thread merging 4 outputs.  A merge takes the left item unless
// the right one is strictly less, so equal keys keep their input order.
const char* kSortKernels = R"MBJ(
#define MBS_THREADS 256
#define MBS_ITEMS 4
#define MBS_TILE (MBS_THREADS * MBS_ITEMS)
// Items of the merge of a[0, la) and b[0, lb) before output position d that
// come from a (the merge-path split).
template <class K>
__device__ __forceinline__ int mbs_split(const K* a, int la, const K* b, int lb, int d) {
  int lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (!USER_LESS(b[d - 1 - mid], a[mid])) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
// Serial merge of `cnt` outputs starting at split (i, j).
template <class K>
__device__ __forceinline__ void mbs_merge_out(const K* ka, const unsigned* ia, int la,
                                              const K* kb, const unsigned* ib, int lb, int i,
                                              int j, int cnt, K* ko, unsigned* io) {
  for (int c = 0; c < cnt; ++c) {
    const bool left = j >= lb || (i < la && !USER_LESS(kb[j], ka[i]));
    if (left) { ko[c] = ka[i]; io[c] = ia[i]; ++i; }
    else { ko[c] = kb[j]; io[c] = ib[j]; ++j; }
  }
}
// Sorts each tile; idx = the input position of every key.
extern "C" __global__ void mbs_block_sort(const T* keys, unsigned long long n, T* out_k,
                                          unsigned* out_i) {
  __shared__ T sk[2][MBS_TILE];
  __shared__ unsigned si[2][MBS_TILE];
  const unsigned long long t0 = (unsigned long long)blockIdx.x * MBS_TILE;
  const int cnt = (int)(n - t0 < MBS_TILE ? n - t0 : MBS_TILE);
  const int base = threadIdx.x * MBS_ITEMS;
  T k[MBS_ITEMS];
  unsigned ix[MBS_ITEMS];
  int mine = cnt - base;
  mine = mine < 0 ? 0 : (mine > MBS_ITEMS ? MBS_ITEMS : mine);
  for (int q = 0; q < mine; ++q) { k[q] = keys[t0 + base + q]; ix[q] = (unsigned)(t0 + base + q); }
  for (int q = 1; q < mine; ++q) {  // stable insertion sort of the thread's items
    T x = k[q];
    unsigned y = ix[q];
    int r = q - 1;
    while (r >= 0 && USER_LESS(x, k[r])) { k[r + 1] = k[r]; ix[r + 1] = ix[r]; --r; }
    k[r + 1] = x;
    ix[r + 1] = y;
  }
  for (int q = 0; q < mine; ++q) { sk[0][base + q] = k[q]; si[0][base + q] = ix[q]; }
  __syncthreads();
  int src = 0;
  for (int w = MBS_ITEMS; w < MBS_TILE; w <<= 1) {
    // merge runs [a, a + w) and [a + w, a + 2w) (clipped to cnt)
    const int pair = base / (2 * w);
    const int a = pair * 2 * w;
    const int la = a < cnt ? (a + w < cnt ? w : cnt - a) : 0;
    const int b = a + w;
    const int lb = b < cnt ? (b + w < cnt ? w : cnt - b) : 0;
    const int d = base - a;
    const int outs = la + lb - d < MBS_ITEMS ? la + lb - d : MBS_ITEMS;
    if (outs > 0) {
      const int i = mbs_split<T>(sk[src] + a, la, sk[src] + b, lb, d);
      mbs_merge_out<T>(sk[src] + a, si[src] + a, la, sk[src] + b, si[src] + b, lb, i, d - i,
                       outs, sk[src ^ 1] + base, si[src ^ 1] + base);
    }
    __syncthreads();
    src ^= 1;
  }
  for (int q = threadIdx.x; q < cnt; q += MBS_THREADS) {
    out_k[t0 + q] = sk[src][q];
    out_i[t0 + q] = si[src][q];
  }
}
// One merge pass: sorted runs of width w -> 2w.
extern "C" __global__ void mbs_merge_pass(const T* in_k, const unsigned* in_i, T* out_k,
                                          unsigned* out_i, unsigned long long n,
                                          unsigned long long w) {
  __shared__ T sk[2 * MBS_TILE];
  __shared__ unsigned si[2 * MBS_TILE];
  __shared__ int s_split[2];
  const unsigned long long d0 = (unsigned long long)blockIdx.x * MBS_TILE;
  if (d0 >= n) return;
  const unsigned long long a = d0 / (2 * w) * (2 * w);
  const unsigned long long la = a + w < n ? w : n - a;
  const unsigned long long b = a + la;
  const unsigned long long lb = b + w < n ? w : (b < n ? n - b : 0);
  const unsigned long long d1 = d0 + MBS_TILE < a + la + lb ? d0 + MBS_TILE : a + la + lb;
  if (threadIdx.x < 2) {  // merge-path splits of the tile's two ends, in global memory
    const unsigned long long d = (threadIdx.x == 0 ? d0 : d1) - a;
    unsigned long long lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
    while (lo < hi) {
      const unsigned long long mid = (lo + hi) >> 1;
      if (!USER_LESS(in_k[b + d - 1 - mid], in_k[a + mid])) lo = mid + 1;
      else hi = mid;
    }
    s_split[threadIdx.x] = (int)lo;
  }
  __syncthreads();
  const unsigned long long i0 = s_split[0], i1 = s_split[1];
  const unsigned long long j0 = d0 - a - i0, j1 = d1 - a - i1;
  const int na = (int)(i1 - i0), nb = (int)(j1 - j0);
  for (int q = threadIdx.x; q < na; q += MBS_THREADS) {
    sk[q] = in_k[a + i0 + q];
    si[q] = in_i[a + i0 + q];
  }
  for (int q = threadIdx.x; q < nb; q += MBS_THREADS) {
    sk[na + q] = in_k[b + j0 + q];
    si[na + q] = in_i[b + j0 + q];
  }
  __syncthreads();
  const int total = na + nb;
  const int d = threadIdx.x * MBS_ITEMS;
  if (d < total) {
    const int outs = total - d < MBS_ITEMS ? total - d : MBS_ITEMS;
    const int i = mbs_split<T>(sk, na, sk + na, nb, d);
    T ko[MBS_ITEMS];
    unsigned io[MBS_ITEMS];
    mbs_merge_out<T>(sk, si, na, sk + na, si + na, nb, i, d - i, outs, ko, io);
    for (int q = 0; q < outs; ++q) {
      out_k[d0 + d + q] = ko[q];
      out_i[d0 + d + q] = io[q];
    }
  }
}
)MBJ";

const char* kMapKernels = R"MBJ(
extern "C" __global__ void mbj_map(const In* in, Out* out, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * 256ull)
    out[i] = USER_MAP(in[i]);
}
)MBJ";

// Compiles `src` for sm_100a; the CUBIN in `cubin`, or the log in `log`.
int nvrtc_compile(const std::string& src, std::vector<char>& cubin, std::string& log) {
  Nvrtc& n = nvrtc();
  if (!n.ok) return set_error(MB_ERR_LAUNCH, n.why);
  nvrtcProgram_t prog = nullptr;
  if (n.create(&prog, src.c_str(), "mb_user_op.cu", 0, nullptr, nullptr) != 0)
    return set_error(MB_ERR_LAUNCH, "NVRTC could not create the program");
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device"};
  const int rc = n.compile(prog, 3, opts);
  size_t ls = 0;
  n.log_size(prog, &ls);
  log.assign(ls, '\0');
  if (ls) n.log(prog, &log[0]);
  if (rc != 0) {
    n.destroy(&prog);
    return set_error(MB_ERR_LAUNCH, "user operator did not compile: " + log);
  }
  size_t cs = 0;
  n.cubin_size(prog, &cs);
  cubin.resize(cs);
  n.cubin(prog, cubin.data());
  n.destroy(&prog);
  return MB_OK;
}

}  // namespace
}  // namespace mb

struct mb_user_op {
  int kind;       // 0 binary, 1 map, 2 predicate (a comparator)
  int dtype;      // binary / predicate: T; map: In
  int out_dtype;  // map: Out
  cudaLibrary_t lib = nullptr;
  cudaKernel_t k[8] = {};
};

using namespace mb;

namespace {

enum { kReducePartial = 0, kReduceFinal = 1, kScanTiles = 2, kScanTotals = 3, kScanApply = 4,
       kMap = 5, kBlockSort = 6, kMergePass = 7 };
constexpr uint64_t kSortTile = 1024;  // MBS_TILE of kSortKernels

int build_op(int kind, int dtype, int out_dtype, const char* source, const char* name,
             bool load, mb_user_op** out) {
  if (!source || !name) return set_error(MB_ERR_LAUNCH, "missing operator source or name");
  if (!dtype_valid(dtype) || (kind == 1 && !dtype_valid(out_dtype)))
    return set_error(MB_ERR_LAUNCH, "unknown element type");
  if (kind < 0 || kind > 2) return set_error(MB_ERR_LAUNCH, "unknown operator kind");
  std::string src;
  if (kind == 0) {
    src = std::string("typedef ") + ctype_name(dtype) + " T;\n" + source + "\n#define USER_OP " +
          name + "\n" + kBinaryKernels;
  } else if (kind == 2) {
    src = std::string("typedef ") + ctype_name(dtype) + " T;\n" + source +
          "\n#define USER_LESS " + name + "\n" + kSortKernels;
  } else {
    src = std::string("typedef ") + ctype_name(dtype) + " In;\ntypedef " + ctype_name(out_dtype) +
          " Out;\n" + source + "\n#define USER_MAP " + name + "\n" + kMapKernels;
  }
  std::vector<char> cubin;
  std::string log;
  MB_TRY(nvrtc_compile(src, cubin, log));
  if (!load) return MB_OK;
  auto* op = new mb_user_op();
  op->kind = kind;
  op->dtype = dtype;
  op->out_dtype = out_dtype;
  cudaError_t e = cudaLibraryLoadData(&op->lib, cubin.data(), nullptr, nullptr, 0, nullptr,
                                      nullptr, 0);
  if (e != cudaSuccess) {
    delete op;
    return check_cuda(e, "cudaLibraryLoadData");
  }
  const char* names[] = {"mbj_reduce_partial", "mbj_reduce_final", "mbj_scan_tiles",
                         "mbj_scan_totals", "mbj_scan_apply", "mbj_map",
                         "mbs_block_sort", "mbs_merge_pass"};
  for (int i = 0; i < 8; ++i) {
    const int owner = i < 5 ? 0 : (i == 5 ? 1 : 2);  // the kind whose source holds kernel i
    if (owner != kind) continue;
    e = cudaLibraryGetKernel(&op->k[i], op->lib, names[i]);
    if (e != cudaSuccess) {
      cudaLibraryUnload(op->lib);
      delete op;
      return check_cuda(e, "cudaLibraryGetKernel");
    }
  }
  *out = op;
  return MB_OK;
}

int launch(mb_executor* ex, cudaKernel_t k, unsigned grid, unsigned block, void** args) {
  MB_CUDA(cudaLaunchKernel((const void*)k, dim3(grid), dim3(block), args, 0, ex->stream));
  return MB_OK;
}

unsigned grid_for_n(mb_executor* ex, uint64_t n) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ex->device);
  const uint64_t want = (n + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 8));
}

int check_plain(mb_executor* ex, const mb_src* in, int dtype) {
  MB_TRY(check_src(ex, in, "input"));
  MB_TRY(check_len_u32(in->len));
  if (in->kind != MB_SRC_COLUMN || in->map != MB_UN_IDENTITY || in->dtype != dtype ||
      in->vtype != dtype || in->len_dev)
    return set_error(MB_ERR_LAUNCH,
                     "user operators take a plain column of the compiled element type");
  return MB_OK;
}

int scan_user(mb_executor* ex, const mb_src* in, mb_user_op* op, bool exclusive, const void* init,
              mb_col out) {
  MB_TRY(check_exec(ex));
  if (!op || op->kind != 0) return set_error(MB_ERR_LAUNCH, "not a compiled binary operator");
  MB_TRY(check_plain(ex, in, op->dtype));
  MB_TRY(check_col(ex, out, "output"));
  if (out.dtype != op->dtype) return set_error(MB_ERR_LAUNCH, "output element type differs");
  if (out.len < in->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", in->len, out.len);
  uint64_t n = in->len;
  if (n == 0) return MB_OK;
  const size_t es = dtype_size(op->dtype);
  const uint64_t tile = 2048;
  const unsigned tiles = (unsigned)((n + tile - 1) / tile);
  Scratch scratch;
  const size_t tot_b = ((size_t)tiles * es + 255) / 256 * 256;
  const size_t loc_b = exclusive ? (n * es + 255) / 256 * 256 : 0;
  MB_TRY(scratch.alloc(ex, tot_b + loc_b + 256));
  char* tot = scratch.as<char>();
  char* loc = exclusive ? tot + tot_b : (char*)out.data;
  char* initd = tot + tot_b + loc_b;
  if (exclusive) MB_CUDA(cudaMemcpyAsync(initd, init, es, cudaMemcpyHostToDevice, ex->stream));
  const void* inp = in->data;
  void* a0[] = {(void*)&inp, (void*)&loc, (void*)&n, (void*)&tot};
  MB_TRY(launch(ex, op->k[kScanTiles], tiles, 256, a0));
  void* a1[] = {(void*)&tot, (void*)&tiles};
  MB_TRY(launch(ex, op->k[kScanTotals], 1, 256, a1));
  int ex_flag = exclusive ? 1 : 0;
  void* outp = out.data;
  void* a2[] = {(void*)&loc, (void*)&outp, (void*)&n, (void*)&tot, (void*)&ex_flag,
                (void*)&initd};
  MB_TRY(launch(ex, op->k[kScanApply], grid_for_n(ex, n), 256, a2));
  return MB_OK;
}

}  // namespace

extern "C" {

int mb_user_op_compile(mb_executor* ex, int dtype, const char* source, const char* name,
                       mb_user_op** out) {
  MB_TRY(check_exec(ex));
  if (!out) return set_error(MB_ERR_LAUNCH, "missing output handle");
  MB_CUDA(cudaSetDevice(ex->device));
  return build_op(0, dtype, dtype, source, name, true, out);
}

int mb_user_map_compile(mb_executor* ex, int in_dtype, int out_dtype, const char* source,
                        const char* name, mb_user_op** out) {
  MB_TRY(check_exec(ex));
  if (!out) return set_error(MB_ERR_LAUNCH, "missing output handle");
  MB_CUDA(cudaSetDevice(ex->device));
  return build_op(1, in_dtype, out_dtype, source, name, true, out);
}

int mb_user_pred_compile(mb_executor* ex, int dtype, const char* source, const char* name,
                         mb_user_op** out) {
  MB_TRY(check_exec(ex));
  if (!out) return set_error(MB_ERR_LAUNCH, "missing output handle");
  MB_CUDA(cudaSetDevice(ex->device));
  return build_op(2, dtype, dtype, source, name, true, out);
}

int mb_sort_user(mb_executor* ex, const mb_src* keys, mb_user_op* less, const mb_src* values,
                 int nvals, mb_col out_keys, const mb_col* out_values) {
  MB_TRY(check_exec(ex));
  if (!less || less->kind != 2) return set_error(MB_ERR_LAUNCH, "not a compiled comparator");
  MB_TRY(check_plain(ex, keys, less->dtype));
  if (nvals < 0 || nvals > 12) return set_error(MB_ERR_LAUNCH, "values take 0 to 12 columns");
  const uint64_t n0 = keys->len;
  for (int c = 0; c < nvals; ++c) {
    MB_TRY(check_src(ex, &values[c], "values"));
    MB_TRY(check_col(ex, out_values[c], "value output"));
    if (values[c].len != n0)
      return set_error(MB_ERR_LENGTH_MISMATCH, "input lengths differ", n0, values[c].len);
    if (out_values[c].len < n0)
      return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n0,
                       out_values[c].len);
  }
  if (out_keys.data) {
    MB_TRY(check_col(ex, out_keys, "key output"));
    if (out_keys.dtype != less->dtype)
      return set_error(MB_ERR_LAUNCH, "key output element type differs");
    if (out_keys.len < n0)
      return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", n0, out_keys.len);
  }
  uint64_t n = n0;
  if (n == 0) return MB_OK;
  const size_t es = dtype_size(less->dtype);
  const size_t kb = (n * es + 255) / 256 * 256, ib = (n * 4 + 255) / 256 * 256;
  Scratch scratch;
  MB_TRY(scratch.alloc(ex, 2 * (kb + ib)));
  char* k0 = scratch.as<char>();
  char* i0 = k0 + kb;
  char* k1 = i0 + ib;
  char* i1 = k1 + kb;
  const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  const void* kin = keys->data;
  void* a0[] = {(void*)&kin, (void*)&n, (void*)&k0, (void*)&i0};
  MB_TRY(launch(ex, less->k[kBlockSort], (unsigned)tiles, 256, a0));
  for (uint64_t w = kSortTile; w < n; w <<= 1) {
    void* a1[] = {(void*)&k0, (void*)&i0, (void*)&k1, (void*)&i1, (void*)&n, (void*)&w};
    MB_TRY(launch(ex, less->k[kMergePass], (unsigned)tiles, 256, a1));
    std::swap(k0, k1);
    std::swap(i0, i1);
  }
  if (out_keys.data)
    MB_CUDA(cudaMemcpyAsync(out_keys.data, k0, n * es, cudaMemcpyDeviceToDevice, ex->stream));
  mb_src idx{};
  idx.kind = MB_SRC_COLUMN;
  idx.dtype = idx.vtype = MB_U32;
  idx.map = MB_UN_IDENTITY;
  idx.data = i0;
  idx.len = n;
  for (int c = 0; c < nvals; ++c) MB_TRY(mb_gather(ex, &values[c], &idx, nullptr, out_values[c]));
  return MB_OK;
}

int mb_user_op_check(int kind, int dtype, int out_dtype, const char* source, const char* name) {
  mb_user_op* unused = nullptr;
  return build_op(kind, dtype, out_dtype, source, name, false, &unused);
}

int mb_user_op_destroy(mb_user_op* op) {
  if (!op) return MB_OK;
  if (op->lib) cudaLibraryUnload(op->lib);
  delete op;
  return MB_OK;
}

int mb_reduce_user(mb_executor* ex, const mb_src* in, mb_user_op* op, const void* init,
                   void* result_dev, void* result_host) {
  MB_TRY(check_exec(ex));
  if (!op || op->kind != 0) return set_error(MB_ERR_LAUNCH, "not a compiled binary operator");
  if (!init) return set_error(MB_ERR_LAUNCH, "missing init");
  MB_TRY(check_plain(ex, in, op->dtype));
  if (result_host && ex->capturing)
    return set_error(MB_ERR_LAUNCH, "a host-valued result cannot be read inside graph capture");
  const size_t es = dtype_size(op->dtype);
  uint64_t n = in->len;
  const unsigned g = grid_for_n(ex, n);
  Scratch scratch;
  MB_TRY(scratch.alloc(ex, (size_t)g * (es + 4) + 512));
  char* part = scratch.as<char>();
  unsigned* has = (unsigned*)(part + ((size_t)g * es + 15) / 16 * 16);
  char* initd = (char*)(has + g) + 16 - ((uintptr_t)(has + g) & 15);
  char* res = initd + 16;
  MB_CUDA(cudaMemcpyAsync(initd, init, es, cudaMemcpyHostToDevice, ex->stream));
  const void* inp = in->data;
  void* a0[] = {(void*)&inp, (void*)&n, (void*)&part, (void*)&has};
  MB_TRY(launch(ex, op->k[kReducePartial], g, 256, a0));
  unsigned parts = g;
  void* dst = result_dev ? result_dev : (void*)res;
  void* a1[] = {(void*)&part, (void*)&has, (void*)&parts, (void*)&initd, (void*)&dst};
  MB_TRY(launch(ex, op->k[kReduceFinal], 1, 32, a1));
  if (result_host) {
    MB_CUDA(cudaMemcpyAsync(ex->host_pinned, dst, es, cudaMemcpyDeviceToHost, ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
    memcpy(result_host, ex->host_pinned, es);
  }
  return MB_OK;
}

int mb_inclusive_scan_user(mb_executor* ex, const mb_src* in, mb_user_op* op, mb_col out) {
  return scan_user(ex, in, op, false, nullptr, out);
}

int mb_exclusive_scan_user(mb_executor* ex, const mb_src* in, mb_user_op* op, const void* init,
                           mb_col out) {
  if (!init) return set_error(MB_ERR_LAUNCH, "missing init");
  return scan_user(ex, in, op, true, init, out);
}

int mb_map_user(mb_executor* ex, const mb_src* in, mb_user_op* op, mb_col out) {
  MB_TRY(check_exec(ex));
  if (!op || op->kind != 1) return set_error(MB_ERR_LAUNCH, "not a compiled map");
  MB_TRY(check_plain(ex, in, op->dtype));
  MB_TRY(check_col(ex, out, "output"));
  if (out.dtype != op->out_dtype) return set_error(MB_ERR_LAUNCH, "output element type differs");
  if (out.len < in->len)
    return set_error(MB_ERR_OUTPUT_TOO_SHORT, "output is shorter than input", in->len, out.len);
  uint64_t n = in->len;
  if (n == 0) return MB_OK;
  const void* inp = in->data;
  void* outp = out.data;
  void* a[] = {(void*)&inp, (void*)&outp, (void*)&n};
  return launch(ex, op->k[kMap], grid_for_n(ex, n), 256, a);
}

}  // extern "C"
