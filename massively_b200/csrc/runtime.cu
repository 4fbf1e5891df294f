// runtime.cu -- executor, memory pool, errors, copies, synchronisation and
// CUDA-graph capture of the massively_b200 C ABI.
//
// Stands in for massively's Executor / DeviceVec storage layer
// (massively/src/core/runtime.rs:22-389) and its Error enum
// (massively/src/core/error.rs:5-14).  One executor = one device + one CUDA
// stream + a stream-ordered memory pool; every algorithm enqueues on that
// stream, and per-call scratch comes from the pool in stream order, so calls
// are asynchronous and capturable into CUDA graphs.

#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"

namespace {

thread_local std::string g_msg;
thread_local mb_error_detail g_detail{0, 0};
std::atomic<uint64_t> g_next_id{1};

}  // namespace

namespace mb {

int set_error(int code, const std::string& msg, uint64_t left, uint64_t right) {
  g_msg = msg;
  g_detail.left = left;
  g_detail.right = right;
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear sticky-free errors so later calls can proceed
  return set_error(MB_ERR_LAUNCH, m);
}

Scratch::~Scratch() {
  if (ptr && ex) cudaFreeAsync(ptr, ex->stream);
}

int Scratch::alloc(mb_executor* e, size_t bytes) {
  ex = e;
  if (bytes == 0) bytes = 16;
  MB_CUDA(cudaMallocFromPoolAsync(&ptr, bytes, e->pool, e->stream));
  return MB_OK;
}

int check_exec(mb_executor* ex) {
  if (!ex) return set_error(MB_ERR_LAUNCH, "null executor");
  return MB_OK;
}

int check_len_u32(uint64_t n) {
  if (n > 0xFFFFFFFFull) return set_error(MB_ERR_LENGTH_TOO_LARGE, "length does not fit in u32", n);
  return MB_OK;
}

int check_src(mb_executor* ex, const mb_src* s, const char* what) {
  if (!s) return set_error(MB_ERR_UNBOUND_COLUMN, std::string(what) + ": missing input");
  if (s->owner != 0 && s->owner != ex->id)
    return set_error(MB_ERR_FOREIGN_EXECUTOR, "executor does not own this device data");
  if (!dtype_valid(s->dtype) || !dtype_valid(s->vtype))
    return set_error(MB_ERR_LAUNCH, std::string(what) + ": unknown element type");
  if (s->kind < MB_SRC_COLUMN || s->kind > MB_SRC_ADJACENT)
    return set_error(MB_ERR_LAUNCH, std::string(what) + ": unknown view kind");
  if (s->kind == MB_SRC_ADJACENT &&
      (s->map != MB_UN_IDENTITY || !op_valid_for((int)s->b, compute_type(s->vtype))))
    return set_error(MB_ERR_LAUNCH, std::string(what) + ": bad adjacent view");
  bool needs_data = s->kind == MB_SRC_COLUMN || s->kind == MB_SRC_PERMUTE ||
                    s->kind == MB_SRC_REVERSE || s->kind == MB_SRC_REPEAT_EACH ||
                    s->kind == MB_SRC_TILE || s->kind == MB_SRC_ADJACENT;
  if (needs_data && s->data == nullptr && s->len > 0)
    return set_error(MB_ERR_UNBOUND_COLUMN, "column is not bound to device storage");
  if (s->kind == MB_SRC_PERMUTE && s->index == nullptr && s->len > 0)
    return set_error(MB_ERR_UNBOUND_COLUMN, "permute view has no index column");
  if ((s->kind == MB_SRC_REPEAT_EACH || s->kind == MB_SRC_TILE) && s->a == 0 && s->len > 0)
    return set_error(MB_ERR_LAUNCH, std::string(what) + ": zero repeat / tile period");
  return check_len_u32(s->len);
}

int check_col(mb_executor* ex, const mb_col& c, const char* what) {
  if (c.owner != 0 && c.owner != ex->id)
    return set_error(MB_ERR_FOREIGN_EXECUTOR, "executor does not own this device data");
  if (!dtype_valid(c.dtype))
    return set_error(MB_ERR_LAUNCH, std::string(what) + ": unknown element type");
  if (c.data == nullptr && c.len > 0)
    return set_error(MB_ERR_UNBOUND_COLUMN, "column is not bound to device storage");
  return check_len_u32(c.len);
}

int read_u32(mb_executor* ex, const uint32_t* dev, uint32_t* host) {
  if (ex->capturing)
    return set_error(MB_ERR_LAUNCH, "a host-valued result cannot be read inside graph capture");
  MB_CUDA(cudaMemcpyAsync(ex->host_pinned, dev, 4, cudaMemcpyDeviceToHost, ex->stream));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  *host = ex->host_pinned[0];
  return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" {

const char* mb_last_error_message(void) { return g_msg.c_str(); }

void mb_last_error_detail(mb_error_detail* out) {
  if (out) *out = g_detail;
}

int mb_abi_version(void) { return MB_ABI_VERSION; }

int mb_executor_create(int device_ordinal, mb_executor** out) {
  if (!out) return set_error(MB_ERR_LAUNCH, "null output pointer");
  *out = nullptr;
  int count = 0;
  MB_CUDA(cudaGetDeviceCount(&count));
  if (device_ordinal < 0 || device_ordinal >= count)
    return set_error(MB_ERR_LAUNCH, "device ordinal out of range");
  MB_CUDA(cudaSetDevice(device_ordinal));
  mb_executor* ex = new mb_executor();
  ex->id = g_next_id.fetch_add(1);
  ex->device = device_ordinal;
  ex->capturing = false;
  ex->graph = nullptr;
  for (int& t : ex->tune) t = -1;
  cudaError_t e = cudaStreamCreateWithFlags(&ex->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete ex; return check_cuda(e, "cudaStreamCreate"); }
  ex->stream = ex->own_stream;
  // The device's default pool, kept warm: freed blocks stay reserved so
  // stream-ordered scratch costs no driver call after the first use.
  e = cudaDeviceGetDefaultMemPool(&ex->pool, device_ordinal);
  if (e == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    e = cudaMemPoolSetAttribute(ex->pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  if (e == cudaSuccess) e = cudaMalloc(&ex->status_dev, 64);
  if (e == cudaSuccess) e = cudaMemset(ex->status_dev, 0, 64);
  if (e == cudaSuccess) e = cudaMallocHost(&ex->host_pinned, 64);
  if (e != cudaSuccess) {
    cudaStreamDestroy(ex->own_stream);
    delete ex;
    return check_cuda(e, "executor setup");
  }
  *out = ex;
  return MB_OK;
}

int mb_executor_destroy(mb_executor* ex) {
  if (!ex) return MB_OK;
  cudaSetDevice(ex->device);
  cudaStreamSynchronize(ex->stream);
  for (auto& sp : ex->spans) {
    cudaEventDestroy(sp.start);
    cudaEventDestroy(sp.stop);
  }
  if (ex->graph) cudaGraphDestroy(ex->graph);
  cudaFree(ex->status_dev);
  cudaFreeHost(ex->host_pinned);
  cudaStreamDestroy(ex->own_stream);
  delete ex;
  return MB_OK;
}

uint64_t mb_executor_id(const mb_executor* ex) { return ex ? ex->id : 0; }

int mb_sync(mb_executor* ex) {
  MB_TRY(check_exec(ex));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  uint32_t st = 0;
  MB_CUDA(cudaMemcpyAsync(ex->host_pinned, ex->status_dev, 4, cudaMemcpyDeviceToHost, ex->stream));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  st = ex->host_pinned[0];
  if (st != MB_DEV_OK) {
    MB_CUDA(cudaMemsetAsync(ex->status_dev, 0, 4, ex->stream));
    MB_CUDA(cudaStreamSynchronize(ex->stream));
    if (st == MB_DEV_ERR_LOOKBACK)
      return set_error(MB_ERR_LAUNCH, "decoupled look-back wait exceeded its limit");
    return set_error(MB_ERR_LAUNCH, "device-side bounds check failed");
  }
  return MB_OK;
}

int mb_get_stream(mb_executor* ex, void** stream) {
  MB_TRY(check_exec(ex));
  if (stream) *stream = (void*)ex->stream;
  return MB_OK;
}

int mb_set_stream(mb_executor* ex, void* stream) {
  MB_TRY(check_exec(ex));
  ex->stream = (cudaStream_t)stream;
  return MB_OK;
}

int mb_use_own_stream(mb_executor* ex) {
  MB_TRY(check_exec(ex));
  ex->stream = ex->own_stream;
  return MB_OK;
}

int mb_alloc(mb_executor* ex, uint64_t bytes, void** out) {
  MB_TRY(check_exec(ex));
  if (!out) return set_error(MB_ERR_LAUNCH, "null output pointer");
  *out = nullptr;
  if (bytes == 0) bytes = 16;
  MB_CUDA(cudaMallocFromPoolAsync(out, bytes, ex->pool, ex->stream));
  return MB_OK;
}

int mb_free(mb_executor* ex, void* ptr) {
  MB_TRY(check_exec(ex));
  if (ptr) MB_CUDA(cudaFreeAsync(ptr, ex->stream));
  return MB_OK;
}

int mb_copy_to_device(mb_executor* ex, void* dst, const void* src, uint64_t bytes) {
  MB_TRY(check_exec(ex));
  if (bytes) MB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ex->stream));
  return MB_OK;
}

int mb_copy_to_host(mb_executor* ex, void* dst, const void* src, uint64_t bytes) {
  MB_TRY(check_exec(ex));
  if (bytes) MB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ex->stream));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  return MB_OK;
}

int mb_pool_stats(mb_executor* ex, uint64_t* used, uint64_t* reserved) {
  MB_TRY(check_exec(ex));
  uint64_t u = 0, r = 0;
  MB_CUDA(cudaMemPoolGetAttribute(ex->pool, cudaMemPoolAttrUsedMemCurrent, &u));
  MB_CUDA(cudaMemPoolGetAttribute(ex->pool, cudaMemPoolAttrReservedMemCurrent, &r));
  if (used) *used = u;
  if (reserved) *reserved = r;
  return MB_OK;
}

// ----------------------------------------------------------------- graphs --

struct mb_graph {
  cudaGraphExec_t exec;
};

int mb_graph_begin(mb_executor* ex) {
  MB_TRY(check_exec(ex));
  if (ex->capturing) return set_error(MB_ERR_LAUNCH, "graph capture already active");
  if (ex->stream == 0)
    return set_error(MB_ERR_LAUNCH, "the legacy default stream cannot be captured");
  MB_CUDA(cudaStreamBeginCapture(ex->stream, cudaStreamCaptureModeThreadLocal));
  ex->capturing = true;
  return MB_OK;
}

int mb_graph_end(mb_executor* ex, mb_graph** out) {
  MB_TRY(check_exec(ex));
  if (!ex->capturing) return set_error(MB_ERR_LAUNCH, "no graph capture active");
  ex->capturing = false;
  cudaGraph_t g = nullptr;
  MB_CUDA(cudaStreamEndCapture(ex->stream, &g));
  mb_graph* gr = new mb_graph();
  cudaError_t e = cudaGraphInstantiate(&gr->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { delete gr; return check_cuda(e, "cudaGraphInstantiate"); }
  *out = gr;
  return MB_OK;
}

int mb_graph_launch(mb_executor* ex, mb_graph* g) {
  MB_TRY(check_exec(ex));
  if (!g) return set_error(MB_ERR_LAUNCH, "null graph");
  MB_CUDA(cudaGraphLaunch(g->exec, ex->stream));
  return MB_OK;
}

int mb_graph_destroy(mb_graph* g) {
  if (!g) return MB_OK;
  cudaGraphExecDestroy(g->exec);
  delete g;
  return MB_OK;
}

}  // extern "C"

// ---------------------------------------------------------- kernel timing --

int mb_kernel_timing(mb_executor* ex, int enable) {
  if (!ex) return mb::set_error(MB_ERR_LAUNCH, "null executor");
  ex->timing = enable != 0;
  return MB_OK;
}

int mb_kernel_timing_read(mb_executor* ex, int family, uint64_t* launches, double* total_ms) {
  if (!ex) return mb::set_error(MB_ERR_LAUNCH, "null executor");
  MB_CUDA(cudaSetDevice(ex->device));
  MB_CUDA(cudaStreamSynchronize(ex->stream));
  uint64_t count = 0;
  double ms = 0.0;
  std::vector<mb_executor::Span> keep;
  for (auto& sp : ex->spans) {
    if (sp.family != family) {
      keep.push_back(sp);
      continue;
    }
    float t = 0.f;
    cudaError_t e = cudaEventElapsedTime(&t, sp.start, sp.stop);
    cudaEventDestroy(sp.start);
    cudaEventDestroy(sp.stop);
    if (e != cudaSuccess) continue;
    ms += t;
    ++count;
  }
  ex->spans.swap(keep);
  if (launches) *launches = count;
  if (total_ms) *total_ms = ms;
  return MB_OK;
}
