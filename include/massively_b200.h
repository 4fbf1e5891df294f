/*
 * massively_b200.h -- C ABI of the B200-native primitive library.
 *
 * This is the boundary a massively `Executor` backend binds (Rust FFI, ctypes,
 * C++).  Every entry point takes plain pointers and sizes, enqueues work on the
 * executor's CUDA stream, never aborts, and returns an `mb_status` that maps
 * 1:1 onto massively's `Error` enum (massively/src/core/error.rs:5-14).  Details
 * of the last failure on the calling thread are read with
 * `mb_last_error_message()` / `mb_last_error_detail()`.
 *
 * Reference interfaces replaced (paths inside the massively project):
 *   Executor / DeviceVec / DeviceSlice ... massively/src/core/runtime.rs:22-389
 *   lazy views (map, permute, counting..)  massively/src/api/lazy.rs:664-922
 *   vector::* algorithms ................. massively/src/api/algorithm/ (one file per family)
 *   seg::Segmentation / ForEachSegment ... massively/src/seg/segmentation.rs:129,
 *                                          massively/src/seg/mod.rs:159-243
 * Each function below cites the public function it stands in for.
 *
 * Conventions
 *  - Lengths are 64-bit in the ABI but, as in massively (`MIndex = u32`,
 *    massively/src/lib.rs:82), every logical length must fit in u32; larger
 *    lengths return MB_ERR_LENGTH_TOO_LARGE.
 *  - Inputs are `mb_src` descriptors: a device column or a lazy view that the
 *    consuming kernel evaluates in its load (no materialisation).
 *  - Outputs are `mb_col`: a device pointer plus capacity.
 *  - Results whose length is data dependent (copy_where, reduce_by_key, set
 *    ops) are written as a device-resident u32 count (`count_dev`), mirroring
 *    massively's LogicalExtent::Device (massively/src/core/extent.rs:17-36);
 *    a non-null `count_host` additionally synchronises and returns it.
 *  - Device-side failures (a bounded decoupled look-back that ran out of
 *    iterations) set a status word on the executor and surface as
 *    MB_ERR_LAUNCH from the next `mb_sync`.
 */
#ifndef MASSIVELY_B200_H
#define MASSIVELY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MB_ABI_VERSION 1

/* ---------------------------------------------------------------- types -- */

/* Storage element types: massively's MStorageElement set
 * (massively/src/core/value.rs:24). */
typedef enum mb_dtype {
  MB_U8 = 0,
  MB_U16 = 1,
  MB_U32 = 2,
  MB_U64 = 3,
  MB_I8 = 4,
  MB_I16 = 5,
  MB_I32 = 6,
  MB_I64 = 7,
  MB_F32 = 8,
  MB_F64 = 9
} mb_dtype;

/* Status codes: one per massively::Error variant (core/error.rs:5-14). */
typedef enum mb_status {
  MB_OK = 0,
  MB_ERR_LENGTH_MISMATCH = 1,      /* detail: left, right               */
  MB_ERR_OUTPUT_TOO_SHORT = 2,     /* detail: left = input, right = output */
  MB_ERR_LENGTH_TOO_LARGE = 3,     /* detail: left = len                */
  MB_ERR_INVALID_SEGMENTATION = 4,
  MB_ERR_UNBOUND_COLUMN = 5,
  MB_ERR_FOREIGN_EXECUTOR = 6,
  MB_ERR_LAUNCH = 7                /* message: mb_last_error_message()  */
} mb_status;

typedef struct mb_error_detail {
  uint64_t left;
  uint64_t right;
} mb_error_detail;

/* Built-in associative operators (massively `op::ReductionOp`,
 * massively/src/core/reduce.rs:63-66).  Integer ADD and MUL wrap.  MIN
 * returns `b < a ? b : a` and MAX returns `a < b ? b : a` (left operand on
 * ties).  `reduce`, `reduce_by_key` and `seg reduce` additionally require a
 * commutative operator (massively/src/core/reduce.rs:35-38); scans keep
 * operand order, so TAKE_LEFT / TAKE_RIGHT are valid there. */
typedef enum mb_op {
  MB_OP_ADD = 0,
  MB_OP_MUL = 1,
  MB_OP_MIN = 2,
  MB_OP_MAX = 3,
  MB_OP_BIT_AND = 4,
  MB_OP_BIT_OR = 5,
  MB_OP_BIT_XOR = 6,
  MB_OP_TAKE_LEFT = 7,
  MB_OP_TAKE_RIGHT = 8
} mb_op;

/* Built-in unary maps applied inside a load (massively `op::UnaryOp`,
 * massively/src/core/op.rs:33-52, and `op::PredicateOp`).  Predicates yield
 * an MFlag (u32, 1 = true; massively/src/lib.rs:89). */
typedef enum mb_unary {
  MB_UN_IDENTITY = 0, /* value converted to the descriptor's vtype (a cast)  */
  MB_UN_IS_TRUE = 1,  /* x != 0                                              */
  MB_UN_IS_FALSE = 2, /* x == 0                                              */
  MB_UN_IS_EVEN = 3,  /* (x & 1) == 0 on the integer bits                    */
  MB_UN_IS_ODD = 4,   /* (x & 1) != 0                                        */
  MB_UN_NEGATE = 5,   /* -x (wrapping for integers)                          */
  MB_UN_BIT_NOT = 6,  /* ~x (integers)                                       */
  MB_UN_ABS = 7,      /* |x| (wrapping for the minimum signed integer)       */
  MB_UN_IS_NEGATIVE = 8, /* x < 0                                            */
  MB_UN_IS_POSITIVE = 9  /* x > 0                                            */
} mb_unary;

/* Built-in binary predicates (massively `op::BinaryPredicateOp`,
 * massively/src/core/ordering/mod.rs:53-56). */
typedef enum mb_pred2 {
  MB_LESS = 0,       /* a < b (IEEE for floats: -0 == +0, NaN unordered)   */
  MB_GREATER = 1,    /* a > b                                              */
  MB_TOTAL_LESS = 2, /* radix total order: floats as f32::total_cmp        */
  MB_EQUAL = 3       /* a == b (key equality for by-key algorithms)        */
} mb_pred2;

/* Lazy view kinds (massively/src/api/lazy.rs:664-922; expression nodes
 * massively/src/core/read.rs:29-445).  Element i of a view reads:
 *   COLUMN       data[i]
 *   CONSTANT     a (value bits)
 *   COUNTING     a + i                 (u32 / u64 / i32 ... wrapping)
 *   STRIDE       a + i * b
 *   PERMUTE      data[index[i]]
 *   REVERSE      data[len - 1 - i]
 *   REPEAT_EACH  data[i / a]
 *   TILE         data[i % a]
 *   ADJACENT     i == 0 ? data[0] : op(data[i-1], data[i]), op = mb_op id in
 *                `b` (lazy::adjacent_difference, massively/src/api/lazy.rs:
 *                869-902); `map` must be MB_UN_IDENTITY
 * and then applies `map` (mb_unary), converting to `vtype`. */
typedef enum mb_src_kind {
  MB_SRC_COLUMN = 0,
  MB_SRC_CONSTANT = 1,
  MB_SRC_COUNTING = 2,
  MB_SRC_STRIDE = 3,
  MB_SRC_PERMUTE = 4,
  MB_SRC_REVERSE = 5,
  MB_SRC_REPEAT_EACH = 6,
  MB_SRC_TILE = 7,
  MB_SRC_ADJACENT = 8
} mb_src_kind;

typedef struct mb_src {
  int32_t kind;            /* mb_src_kind                                  */
  int32_t dtype;           /* element type stored in `data` / of a, b      */
  int32_t vtype;           /* element type produced after `map`            */
  int32_t map;             /* mb_unary                                     */
  const void* data;        /* device column (offset already applied)       */
  const uint32_t* index;   /* PERMUTE: device index column                 */
  uint64_t len;            /* logical length (capacity)                    */
  uint64_t a;              /* CONSTANT bits / start / repeat / period      */
  uint64_t b;              /* STRIDE step bits                             */
  uint64_t owner;          /* executor id that owns `data`; 0 = unchecked  */
  const uint32_t* len_dev; /* optional device logical length (<= len)      */
} mb_src;

typedef struct mb_col {
  void* data;       /* device pointer                                      */
  int32_t dtype;    /* mb_dtype                                            */
  int32_t pad_;
  uint64_t len;     /* capacity in elements                                */
  uint64_t owner;   /* executor id that owns `data`; 0 = unchecked         */
} mb_col;

typedef struct mb_executor mb_executor;
typedef struct mb_graph mb_graph;

/* ------------------------------------------------------------- errors ---- */

/* Thread-local text and detail of the last non-OK status on this thread. */
const char* mb_last_error_message(void);
void mb_last_error_detail(mb_error_detail* out);
int mb_abi_version(void);

/* ------------------------------------------------------------ runtime ---- */

/* Executor::new (massively/src/core/runtime.rs:49-54): binds a device and a
 * CUDA stream, gives the executor a process-unique id (never 0). */
int mb_executor_create(int device_ordinal, mb_executor** out);
int mb_executor_destroy(mb_executor* exec);
uint64_t mb_executor_id(const mb_executor* exec);
/* Executor::sync (runtime.rs:192-196): waits for the stream and reports a
 * device-side failure recorded since the last sync as MB_ERR_LAUNCH. */
int mb_sync(mb_executor* exec);
/* The stream the executor enqueues on (cudaStream_t, as void*).  Setting a
 * stream makes every later call enqueue there (NULL is the legacy default
 * stream); mb_use_own_stream returns to the executor's own stream. */
int mb_get_stream(mb_executor* exec, void** stream);
int mb_set_stream(mb_executor* exec, void* stream);
int mb_use_own_stream(mb_executor* exec);

/* Executor::alloc / to_device / to_host (runtime.rs:98-177): stream-ordered
 * pool allocations owned by `exec`. */
int mb_alloc(mb_executor* exec, uint64_t bytes, void** out);
int mb_free(mb_executor* exec, void* ptr);
int mb_copy_to_device(mb_executor* exec, void* dst, const void* src, uint64_t bytes);
int mb_copy_to_host(mb_executor* exec, void* dst, const void* src, uint64_t bytes);
/* Bytes currently held by the executor's pool (for admission control). */
int mb_pool_stats(mb_executor* exec, uint64_t* used, uint64_t* reserved);

/* ---------------------------------------------------- transform / fill ---- */

/* vector::copy / vector::map (massively/src/api/algorithm/transform.rs:56-110):
 * evaluates a lazy view into `out`. */
int mb_copy(mb_executor* exec, const mb_src* in, mb_col out);
/* vector::fill (massively/src/api/algorithm/selection.rs:321). */
int mb_fill(mb_executor* exec, const void* value, mb_col out);
/* vector::replace_where (massively/src/api/algorithm/selection.rs:363; core
 * massively/src/core/selection.rs:471-513): out[c][i] = values[c] wherever
 * stencil[i] != 0, for each of the `ncols` (1..12) output columns; other
 * items keep their value.  `values` holds one 8-byte slot per column (value
 * bits in the low bytes).  LENGTH_MISMATCH{stencil, output} when the lengths
 * differ. */
int mb_replace_where(mb_executor* exec, const uint64_t* values, const mb_src* stencil,
                     const mb_col* out, int ncols);
/* vector::transform_where (selection.rs:436; core selection.rs:515-595):
 * out[c][i] = in[c][i] wherever stencil[i] != 0 -- the operator is the
 * input view's `map` (mb_unary), converted to the output's element type --
 * other items keep their value.  LENGTH_MISMATCH{input, stencil} and
 * {input, output} as in massively. */
int mb_transform_where(mb_executor* exec, const mb_src* in, int ncols, const mb_src* stencil,
                       const mb_col* out);

/* ------------------------------------------------------------- scan ------ */

/* vector::inclusive_scan (massively/src/api/algorithm/scan.rs:96; core
 * massively/src/core/scan.rs:1125): out[i] = x0 op x1 op ... op xi. */
int mb_inclusive_scan(mb_executor* exec, const mb_src* in, int op, mb_col out);
/* Inclusive scan that allocates nothing.  No counterpart in massively: it
 * exists for callers that must not allocate device memory during a call --
 * for instance code that runs while another allocator owns all free device
 * memory, or that has to be free of allocation failures and allocator
 * synchronisation in the middle of its work.  Same result as
 * mb_inclusive_scan; the look-back scratch lives in a fixed 1 MiB array in
 * the library's device memory (every device that loads the library holds it
 * until exit) instead of the pool.  Limit: at most 2^27 elements of a 4-byte
 * type or 2^26 of an 8-byte type (MB_ERR_LENGTH_TOO_LARGE beyond).  The first
 * call on a device looks up the array's device address (no allocation);
 * make that first call before any stream capture.  Every call shares the
 * array, so calls that can overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
int mb_inclusive_scan_noalloc(mb_executor* exec, const mb_src* in, int op, mb_col out);
/* vector::exclusive_scan (scan.rs:216; core scan.rs:1180-1234):
 * out[0] = init, out[i] = init op x0 op ... op x(i-1).  `init` points to one
 * host value of the input's vtype. */
int mb_exclusive_scan(mb_executor* exec, const mb_src* in, int op, const void* init,
                      mb_col out);

/* ------------------------------------------------------------- reduce ---- */

/* vector::reduce (massively/src/api/algorithm/reduce.rs:32-50; core
 * massively/src/core/reduce.rs:1074): init op fold(x) in a fixed, run-to-run
 * deterministic tree order.  The result (one vtype value) goes to
 * `result_dev` (device, may be NULL) and, when `result_host` is non-NULL, to
 * the host after a stream synchronisation. */
int mb_reduce(mb_executor* exec, const mb_src* in, int op, const void* init,
              void* result_dev, void* result_host);

/* ---------------------------------------------------------- selection ---- */

/* vector::copy_where / remove_where (massively/src/api/algorithm/
 * selection.rs:146-230; core massively/src/core/selection.rs:363-411):
 * stable compaction of the rows whose stencil flag is non-zero (copy) or
 * zero (remove).  `in` holds `ncols` columns written to `out[0..ncols)`. */
int mb_copy_where(mb_executor* exec, const mb_src* in, int ncols, const mb_src* stencil,
                  const mb_col* out, uint32_t* count_dev, uint32_t* count_host);
int mb_remove_where(mb_executor* exec, const mb_src* in, int ncols, const mb_src* stencil,
                    const mb_col* out, uint32_t* count_dev, uint32_t* count_host);
/* vector::partition (selection.rs:272-300; core selection.rs:413-457): rows
 * whose `pred` (mb_unary predicate over column `pred_col`) holds come first,
 * both halves stable; returns the boundary. */
int mb_partition(mb_executor* exec, const mb_src* in, int ncols, int pred_col, int pred,
                 const mb_col* out, uint32_t* boundary_dev, uint32_t* boundary_host);

/* ------------------------------------------------------ gather/scatter ---- */

/* vector::gather (massively/src/api/algorithm/indexed.rs:172):
 * out[i] = values[indices[i]].  vector::gather_where (indexed.rs:237): only
 * where stencil[i] != 0 (stencil may be NULL). */
int mb_gather(mb_executor* exec, const mb_src* values, const mb_src* indices,
              const mb_src* stencil, mb_col out);
/* vector::scatter (massively/src/api/algorithm/scatter.rs:248):
 * out[indices[i]] = values[i]; scatter_where (scatter.rs:315) with a stencil.
 * Colliding indices leave one unspecified writer, as in massively. */
int mb_scatter(mb_executor* exec, const mb_src* values, const mb_src* indices,
               const mb_src* stencil, mb_col out);
/* vector::scatter_reduce (massively/src/api/algorithm/scatter.rs:332-420;
 * core massively/src/core/scatter_reduce.rs): for every destination d named
 * by `indices`, out[c][d] = out[c][d] op[c] (inits[c] op[c] v_1 op[c] ...),
 * per value column c; other destinations keep their value.  Each op must be
 * associative and commutative (not TAKE_LEFT / TAKE_RIGHT); values[c] and
 * out[c] have the same element type; `inits` holds one 8-byte slot per
 * column (value bits in the low bytes).  Proposals of one destination are
 * combined in an unspecified order (float ADD may round differently from run
 * to run).  An index at or past out[c].len is skipped and reported as a launch
 * error at the next synchronisation. */
int mb_scatter_reduce(mb_executor* exec, const mb_src* values, int nvals, const mb_src* indices,
                      const int* ops, const uint64_t* inits, const mb_col* out);

/* ---------------------------------------------------------- ordering ---- */

/* vector::radix_sort_by_key (massively/src/api/algorithm/by_key.rs:272-325;
 * core massively/src/core/radix.rs:369-546): stable LSD radix order of
 * `nkeys` (1..3) key columns, the first column primary, under the radix
 * encodings of massively/src/core/radix.rs:46-89 (unsigned as is, signed with
 * the sign bit flipped, floats in total order).  Writes the `nvals` (0..12)
 * value columns permuted, and the keys when `out_keys` is non-NULL. */
int mb_radix_sort_by_key(mb_executor* exec, const mb_src* keys, int nkeys,
                         const mb_src* values, int nvals, const mb_col* out_values,
                         const mb_col* out_keys);
/* vector::sort (massively/src/api/algorithm/ordering.rs:64-76; core
 * massively/src/core/ordering/sort.rs:614-696) with a built-in comparator
 * (mb_pred2 LESS, GREATER or TOTAL_LESS): stable. */
int mb_sort(mb_executor* exec, const mb_src* keys, int less, mb_col out);
/* vector::sort_by_key (by_key.rs:226-270; core ordering/mod.rs:325-840):
 * stable comparator sort of `keys`, carrying `nvals` value columns. */
int mb_sort_by_key(mb_executor* exec, const mb_src* keys, int less, const mb_src* values,
                   int nvals, const mb_col* out_keys, const mb_col* out_values);

/* ------------------------------------------------------------- by key ---- */

/* vector::reduce_by_key (massively/src/api/algorithm/by_key.rs:618-724; core
 * massively/src/core/by_key.rs:79-121): for every maximal run of adjacent
 * equal keys (`key_eq` = MB_EQUAL) writes the run's first key and, per value
 * column c, inits[c] op[c] v_head ... op[c] v_tail.  `inits` holds one
 * 8-byte slot per value column (value bits in the low bytes). */
int mb_reduce_by_key(mb_executor* exec, const mb_src* keys, int key_eq, const mb_src* values,
                     int nvals, const int* ops, const uint64_t* inits, mb_col out_keys,
                     const mb_col* out_values, uint32_t* count_dev, uint32_t* count_host);
/* reduce_by_key whose runs also break at segment starts (offsets of
 * `segment_count` segments over the rows).  No counterpart in massively: it
 * lets a batched caller reduce many independent requests' rows in one
 * launch without runs merging across request boundaries. */
int mb_reduce_by_key_segmented(mb_executor* exec, const mb_src* keys, int key_eq,
                               const mb_src* values, int nvals, const int* ops,
                               const uint64_t* inits, const uint32_t* offsets,
                               uint64_t segment_count, mb_col out_keys, const mb_col* out_values,
                               uint32_t* count_dev, uint32_t* count_host);
/* vector::inclusive_scan_by_key / exclusive_scan_by_key (by_key.rs:399-560). */
int mb_inclusive_scan_by_key(mb_executor* exec, const mb_src* keys, int key_eq,
                             const mb_src* values, int op, mb_col out);
int mb_exclusive_scan_by_key(mb_executor* exec, const mb_src* keys, int key_eq,
                             const mb_src* values, int op, const void* init, mb_col out);

/* --------------------------------------------------------- merge / set ---- */

/* vector::unique (massively/src/api/algorithm/ordering.rs:146) and
 * vector::unique_by_key (by_key.rs:759): the first item (row of `values`) of
 * every run of adjacent equal items (keys) under `equal` (MB_EQUAL).  The
 * kept count is written to count_dev (device) and/or count_host. */
int mb_unique(mb_executor* exec, const mb_src* input, int equal, mb_col out, uint32_t* count_dev,
              uint32_t* count_host);
int mb_unique_by_key(mb_executor* exec, const mb_src* keys, const mb_src* values, int nvals,
                     int equal, const mb_col* out_values, uint32_t* count_dev,
                     uint32_t* count_host);

/* vector::lower_bound / vector::upper_bound (massively/src/api/algorithm/
 * search.rs:81-147): for every value, the partition point of the sorted
 * `source` under `less` -- the first index whose element is not less than the
 * value (lower) or that the value is less than (upper).  `out` receives one
 * MIndex (u32) per value. */
int mb_lower_bound(mb_executor* exec, const mb_src* source, const mb_src* values, int less,
                   mb_col out);
int mb_upper_bound(mb_executor* exec, const mb_src* source, const mb_src* values, int less,
                   mb_col out);

/* ------------------------------------- first-index searches and extrema ---- */

/* Each writes one u32 to result_dev (device, stream-ordered: usable inside a
 * graph capture) and / or result_host (synchronises).  An index result is
 * MB_NONE (MIndex::MAX) for massively's None; a flag result is 0 or 1.
 * Predicates `pred` are the mb_unary IS_* ids (IS_EVEN / IS_ODD on integer
 * items only); `equal` is MB_EQUAL; `less` is LESS, GREATER or TOTAL_LESS.
 *
 * mb_find_if         vector::find_if (predicate.rs:218): first passing item.
 * mb_is_partitioned  vector::is_partitioned (predicate.rs:225-260): flag, no
 *                    passing item after a failing one.
 * mb_adjacent_find   vector::adjacent_find (ordering.rs:107): first i with
 *                    x[i] == x[i+1].
 * mb_is_sorted_until vector::is_sorted_until (ordering.rs:213): first i with
 *                    less(x[i], x[i-1]), else the length; is_sorted
 *                    (ordering.rs:256) is "result == length".
 * mb_find_first_of   vector::find_first_of (search.rs:33): first source item
 *                    equal to any needle.
 * mb_mismatch        vector::mismatch (search.rs:231): first i below the
 *                    shorter length with left[i] != right[i]; else the
 *                    shorter length when the lengths differ, else None.
 * mb_equal           vector::equal (search.rs:175): flag.
 * mb_lexicographical_compare  vector::lexicographical_compare
 *                    (search.rs:289): flag, left before right. */
#define MB_NONE 0xFFFFFFFFu
int mb_find_if(mb_executor* exec, const mb_src* input, int pred, uint32_t* result_dev,
               uint32_t* result_host);
int mb_is_partitioned(mb_executor* exec, const mb_src* input, int pred, uint32_t* result_dev,
                      uint32_t* result_host);
int mb_adjacent_find(mb_executor* exec, const mb_src* input, int equal, uint32_t* result_dev,
                     uint32_t* result_host);
int mb_is_sorted_until(mb_executor* exec, const mb_src* input, int less, uint32_t* result_dev,
                       uint32_t* result_host);
int mb_find_first_of(mb_executor* exec, const mb_src* source, const mb_src* needles, int equal,
                     uint32_t* result_dev, uint32_t* result_host);
int mb_mismatch(mb_executor* exec, const mb_src* left, const mb_src* right, int equal,
                uint32_t* result_dev, uint32_t* result_host);
int mb_equal(mb_executor* exec, const mb_src* left, const mb_src* right, int equal,
             uint32_t* result_dev, uint32_t* result_host);
int mb_lexicographical_compare(mb_executor* exec, const mb_src* left, const mb_src* right,
                               int less, uint32_t* result_dev, uint32_t* result_host);

/* vector::min_element / max_element / minmax_element (ordering.rs:300-380,
 * core massively/src/core/arg_reduce.rs): the first minimum, the first
 * maximum, and (minmax: two u32, minimum then maximum) the LAST minimum with
 * the first maximum, as massively's sequential definition gives them; MB_NONE
 * for an empty input.  Under LESS / GREATER a float NaN behaves as in that
 * sequential scan (a NaN at index 0 is the first minimum and maximum; minmax's
 * minimum restarts after the last NaN). */
int mb_min_element(mb_executor* exec, const mb_src* input, int less, uint32_t* result_dev,
                   uint32_t* result_host);
int mb_max_element(mb_executor* exec, const mb_src* input, int less, uint32_t* result_dev,
                   uint32_t* result_host);
int mb_minmax_element(mb_executor* exec, const mb_src* input, int less, uint32_t* result_dev,
                      uint32_t* result_host);

/* vector::merge (massively/src/api/algorithm/merge.rs:109; core
 * massively/src/core/merge.rs:24-1230): stable merge, left first on ties. */
int mb_merge(mb_executor* exec, const mb_src* left, const mb_src* right, int less, mb_col out);
/* vector::merge_by_key (merge.rs:195-282). */
int mb_merge_by_key(mb_executor* exec, const mb_src* left_keys, const mb_src* left_values,
                    const mb_src* right_keys, const mb_src* right_values, int nvals, int less,
                    mb_col out_keys, const mb_col* out_values);
/* vector::set_union / set_intersection / set_difference
 * (massively/src/api/algorithm/set.rs:47-195; core massively/src/core/
 * set.rs:14-401), multiset semantics. */
int mb_set_union(mb_executor* exec, const mb_src* left, const mb_src* right, int less,
                 mb_col out, uint32_t* count_dev, uint32_t* count_host);
int mb_set_intersection(mb_executor* exec, const mb_src* left, const mb_src* right, int less,
                        mb_col out, uint32_t* count_dev, uint32_t* count_host);
int mb_set_difference(mb_executor* exec, const mb_src* left, const mb_src* right, int less,
                      mb_col out, uint32_t* count_dev, uint32_t* count_host);

/* ------------------------------------------------------------ segments ---- */

/* Segmentation::from_offsets (massively/src/seg/segmentation.rs:196-232):
 * offsets must be non-empty, start at 0 and be non-decreasing; returns the
 * value count (one synchronisation, as in massively). */
int mb_segmentation_validate_offsets(mb_executor* exec, const uint32_t* offsets,
                                     uint64_t offset_count, uint32_t* value_count);
/* Segmentation::from_lengths (segmentation.rs:238-280): offsets (count + 1
 * entries) from per-segment lengths; fails with LENGTH_TOO_LARGE when the
 * total does not fit in u32. */
int mb_segmentation_from_lengths(mb_executor* exec, const mb_src* lengths, uint32_t* offsets,
                                 uint32_t* value_count);
/* Segmentation::segment_ids (flat value -> segment index). */
int mb_segmentation_segment_ids(mb_executor* exec, const uint32_t* offsets,
                                uint64_t segment_count, uint32_t* ids, uint64_t value_count);
/* Segmentation::lengths and local_indices (segmentation.rs:346-411). */
int mb_segmentation_lengths(mb_executor* exec, const uint32_t* offsets, uint64_t segment_count,
                            uint32_t* lengths);
int mb_segmentation_local_indices(mb_executor* exec, const uint32_t* offsets,
                                  uint64_t segment_count, uint32_t* local, uint64_t value_count);
/* Segmentation::from_segment_ids (segmentation.rs:290-335): ids must be
 * non-decreasing and below segment_count; offsets[s] = lower_bound(ids, s)
 * for s = 0..segment_count (segment_count + 1 entries, one synchronisation). */
int mb_segmentation_from_segment_ids(mb_executor* exec, const mb_src* ids, uint64_t segment_count,
                                     uint32_t* offsets);

/* ForEachSegment(InclusiveScan(op)) / ExclusiveScan(op, init)
 * (massively/src/seg/mod.rs:525-572). */
int mb_seg_inclusive_scan(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                          uint64_t segment_count, int op, mb_col out);
int mb_seg_exclusive_scan(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                          uint64_t segment_count, int op, const void* init, mb_col out);
/* ForEachSegment(Reduce(op, init)) (massively/src/seg/mod.rs:676-897): one
 * value per segment; empty segments yield `init`. */
int mb_seg_reduce(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                  uint64_t segment_count, int op, const void* init, mb_col out);
/* ForEachSegment(Sort(less)) (massively/src/seg/mod.rs:379-425): stable sort
 * inside every segment, offsets unchanged. */
/* ForEachSegment(CountIf / FindIf / AdjacentFind / AllOf / AnyOf / NoneOf /
 * IsSorted / IsSortedUntil) (massively/src/seg/mod.rs:211-245; oracle
 * verification/oracle/src/seg.rs:171-283): one u32 per segment into `out`.
 * COUNT_IF counts the items `op` (an IS_* predicate) passes; FIND_IF gives
 * the first passing local index, ADJACENT_FIND the first i with
 * x[i] == x[i+1] (`op` = MB_EQUAL), IS_SORTED_UNTIL the first i with
 * less(x[i], x[i-1]) (`op` = LESS / GREATER / TOTAL_LESS) -- each the
 * segment's length when there is none; ALL_OF / ANY_OF / NONE_OF / IS_SORTED
 * give MFlags. */
enum {
  MB_SEG_COUNT_IF = 0,
  MB_SEG_FIND_IF = 1,
  MB_SEG_ADJACENT_FIND = 2,
  MB_SEG_IS_SORTED_UNTIL = 3,
  MB_SEG_ALL_OF = 4,
  MB_SEG_ANY_OF = 5,
  MB_SEG_NONE_OF = 6,
  MB_SEG_IS_SORTED = 7
};
int mb_seg_query(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                 uint64_t segment_count, int query, int op, mb_col out);
/* ForEachSegment(Reverse) and ForEachSegment(AdjacentDifference(op))
 * (massively/src/seg/mod.rs:177, 191; oracle seg.rs:41-46, 90-107): the
 * same offsets; `out` holds the transformed values. */
int mb_seg_reverse(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                   uint64_t segment_count, mb_col out);
int mb_seg_adjacent_difference(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                               uint64_t segment_count, int op, mb_col out);
/* ForEachSegment(Filter(pred) / Take(k) / Unique(equal)) (seg/mod.rs:195-205;
 * oracle seg.rs:109-153): a stable subsequence of every segment.  `kind` 0 =
 * filter (`param` an IS_* predicate), 1 = take (`param` = k), 2 = unique
 * (`param` = MB_EQUAL).  Writes the kept values to `out` (capacity: the input
 * length) and the new offsets (segment_count + 1 entries) to new_offsets;
 * the kept count goes to count_dev and / or count_host. */
int mb_seg_keep(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                uint64_t segment_count, int kind, int param, mb_col out, uint32_t* new_offsets,
                uint32_t* count_dev, uint32_t* count_host);
int mb_seg_sort(mb_executor* exec, const mb_src* values, const uint32_t* offsets,
                uint64_t segment_count, int less, mb_col out);

/* -------------------------------------------------------------- random ---- */

/* util::random::uniform_u32 / uniform_u64 (massively/src/api/util/
 * random.rs:12-22, 331-385): the PCG-hash stream, element i of the view at
 * `offset + i`.  Integer streams are bit-exact with massively's. */
int mb_random_uniform_u32(mb_executor* exec, uint32_t min, uint32_t max, uint64_t seed,
                          uint64_t offset, mb_col out);
int mb_random_uniform_u64(mb_executor* exec, uint64_t min, uint64_t max, uint64_t seed,
                          uint64_t offset, mb_col out);

/* ------------------------------------------------------ batched graphs ---- */

/* Captures every call made on `exec` between begin and end into a CUDA graph
 * that `mb_graph_launch` replays on the executor's stream.  Calls that return
 * a host value (count_host, result_host, validation) must not be captured. */
int mb_graph_begin(mb_executor* exec);
int mb_graph_end(mb_executor* exec, mb_graph** out);
int mb_graph_launch(mb_executor* exec, mb_graph* graph);
int mb_graph_destroy(mb_graph* graph);

/* ------------------------------------------------------------- tuning ---- */

/* Selects the kernel configuration (tile shape) used by an algorithm family
 * for later calls on `exec`; -1 restores the built-in default.  `family` is
 * one of the MB_TUNE_* ids; `config` is below mb_tune_config_count(family). */
enum {
  MB_TUNE_SCAN = 0,
  MB_TUNE_RADIX = 1,
  MB_TUNE_REDUCE = 2,
  MB_TUNE_SELECT = 3,
  MB_TUNE_SEG = 4, /* ForEachSegment(Reduce): tile-local folds or a carried look-back */
  MB_TUNE_SEARCH = 5 /* lower_bound / upper_bound: line levels or a two-level binary search */
};
int mb_tune_config_count(int family);
int mb_tune_set(mb_executor* exec, int family, int config);
int mb_tune_get(mb_executor* exec, int family);
/* Human-readable description of one configuration (static string). */
const char* mb_tune_describe(int family, int config);

/* ----------------------------------------------------- user operators ---- */

/* massively's operators are user `#[cube]` trait impls (op::ReductionOp,
 * op::UnaryOp; massively/src/core/op.rs:33-96) compiled into its kernels.
 * Beyond the built-in ids above, an operator can be given as CUDA C source
 * and is compiled at run time (NVRTC, sm_100a):
 *  - mb_user_op_compile: `source` defines `__device__ T name(T a, T b)`
 *    over the element type `dtype` (T is typedef'd before it); the operator
 *    is associative (scans) and also commutative (reduce);
 *  - mb_user_map_compile: `source` defines `__device__ Out name(In x)`.
 * The handle is valid on every device and is released by
 * mb_user_op_destroy.  mb_user_op_check only compiles (no device needed) and
 * reports a compile error with NVRTC's log as the message.  The algorithms
 * take a plain column of the compiled type: reduce (vector::reduce,
 * init op fold), inclusive / exclusive scan (vector::inclusive_scan /
 * exclusive_scan), map (vector::map). */
typedef struct mb_user_op mb_user_op;
int mb_user_op_compile(mb_executor* exec, int dtype, const char* source, const char* name,
                       mb_user_op** out);
int mb_user_map_compile(mb_executor* exec, int in_dtype, int out_dtype, const char* source,
                        const char* name, mb_user_op** out);
int mb_user_op_check(int kind, int dtype, int out_dtype, const char* source, const char* name);
int mb_user_op_destroy(mb_user_op* op);
int mb_reduce_user(mb_executor* exec, const mb_src* in, mb_user_op* op, const void* init,
                   void* result_dev, void* result_host);
int mb_inclusive_scan_user(mb_executor* exec, const mb_src* in, mb_user_op* op, mb_col out);
int mb_exclusive_scan_user(mb_executor* exec, const mb_src* in, mb_user_op* op, const void* init,
                           mb_col out);
int mb_map_user(mb_executor* exec, const mb_src* in, mb_user_op* op, mb_col out);
/* A user comparator (massively `op::BinaryPredicateOp`, core/ordering/
 * mod.rs:53-56): `source` defines `__device__ bool name(T a, T b)`, a strict
 * weak order ("a before b").  mb_sort_user is vector::sort / sort_by_key
 * under it (massively/src/api/algorithm/ordering.rs:64-76, by_key.rs:
 * 226-270; core massively/src/core/ordering/sort.rs:54-455): a stable merge
 * sort of a plain key column of the compiled type, writing the sorted keys
 * (when out_keys.data is non-NULL) and the `nvals` (0..12) value columns
 * permuted alike; ties keep their input order.  mb_user_op_check takes kind
 * 2 for a comparator. */
int mb_user_pred_compile(mb_executor* exec, int dtype, const char* source, const char* name,
                         mb_user_op** out);
int mb_sort_user(mb_executor* exec, const mb_src* keys, mb_user_op* less, const mb_src* values,
                 int nvals, mb_col out_keys, const mb_col* out_values);

/* ------------------------------------------------------- kernel timing ---- */

/* No counterpart in massively (which has no tracing).  While enabled, the
 * executor brackets each launch of its dominant kernels with CUDA events on
 * its stream (never inside a graph capture).  mb_kernel_timing_read
 * synchronises the stream and returns, for one MB_KF_* family, how many
 * launches were recorded since the last read of that family and their summed
 * device time in milliseconds, then forgets them.  Used by the benchmark for
 * the per-kernel roofline. */
enum {
  MB_KF_RADIX_ONESWEEP = 0,  /* one onesweep digit pass */
  MB_KF_RADIX_HISTOGRAM = 1, /* the all-digit histogram */
  MB_KF_SCAN = 2,            /* inclusive / exclusive scan */
  MB_KF_SELECT = 3,          /* copy_where / remove_where / partition */
  MB_KF_SEARCH = 4,          /* first-index searches and extrema (predicate.cu) */
  MB_KF_SEG_SORT = 5         /* the segmented sort of 4-byte values (segsort.cu) */
};
int mb_kernel_timing(mb_executor* exec, int enable);
int mb_kernel_timing_read(mb_executor* exec, int family, uint64_t* launches, double* total_ms);

/* ------------------------------------------------ failure detection ---- */

/* No counterpart in massively.  Enqueues one of the library's own bounded
 * waits against a condition that never comes, to show that it ends: kind 0
 * runs the radix digit look-back of four tiles whose first predecessor never
 * publishes; kind 1 waits on an mbarrier for bulk-copy bytes that no copy
 * delivers.  Each wait gives up after the 2 s spin limit, records the
 * failure and returns (no copy is in flight, the context stays usable); the
 * next mb_sync reports MB_ERR_LAUNCH ("decoupled look-back wait exceeded its
 * limit") and clears it. */
int mb_check_bounded_waits(mb_executor* exec, int kind);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MASSIVELY_B200_H */
