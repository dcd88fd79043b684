/*
 * ionp_cuda.h -- C ABI of the B200 ufunc engine (libionp_cuda.so).
 *
 * This is the seam the reference's Rust engine API occupies:
 * ionp_core::ufunc::{binary_op, unary_op, math_unary_op, math_binary_op,
 * reduce_axis, argext, write_out} over `&NdArray`, returning
 * `Result<NdArray, IonpError>` (Son0fSun/anionpy, ionp-core/src/ufunc.rs).
 * Arrays are plain descriptors over device memory; no C++ or torch types
 * cross this boundary. Every entry point returns an int32 status
 * (IONP_OK = 0); the message of the last failure on the calling thread is
 * available from ionp_last_error_message().
 *
 * Conventions (the reference's, ionp-core/src/shape.rs:1-5 and
 * ionp-core/src/array.rs:24-40):
 *   - strides and offsets are in ELEMENTS, not bytes;
 *   - `data` is the base of the allocation, `offset` the first element;
 *   - dtype codes follow ionp-core/src/dtype.rs:14 (complex excluded).
 * The caller owns every buffer; outputs are allocated by the caller after
 * host-side planning (shape, dtype and layout from the query functions).
 */
#ifndef IONP_CUDA_H
#define IONP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IONP_MAX_DIMS 32

/* dtype codes (ionp-core/src/dtype.rs:14-28) */
enum {
    IONP_BOOL = 0, IONP_INT8, IONP_INT16, IONP_INT32, IONP_INT64,
    IONP_UINT8, IONP_UINT16, IONP_UINT32, IONP_UINT64,
    IONP_FLOAT16, IONP_FLOAT32, IONP_FLOAT64
};

/* op codes: BinaryOp (ufunc.rs:43-65) in declaration order, then the
 * MathBinaryOp / UnaryOp / MathUnaryOp members this engine implements. */
enum {
    IONP_ADD = 0, IONP_SUBTRACT, IONP_MULTIPLY, IONP_DIVIDE, IONP_MAXIMUM, IONP_MINIMUM,
    IONP_GREATER, IONP_GREATER_EQUAL, IONP_LESS, IONP_LESS_EQUAL, IONP_EQUAL, IONP_NOT_EQUAL,
    IONP_LOGICAL_AND, IONP_LOGICAL_OR, IONP_LOGICAL_XOR,
    IONP_BITWISE_AND, IONP_BITWISE_OR, IONP_BITWISE_XOR,
    IONP_FLOOR_DIVIDE, IONP_LEFT_SHIFT, IONP_RIGHT_SHIFT,
    IONP_REMAINDER = 32, IONP_FMOD = 33,
    IONP_NEGATIVE = 64, IONP_ABSOLUTE = 65, IONP_INVERT = 66, IONP_LOGICAL_NOT = 67,
    IONP_SQRT = 80, IONP_EXP = 81, IONP_LOG = 82, IONP_SIN = 83, IONP_COS = 84
};

/* status codes: 1:1 with IonpError variants (ionp-core/src/error.rs:8-40),
 * plus device-side failures. */
enum {
    IONP_OK = 0,
    IONP_ERR_BROADCAST = 1,   /* IonpError::Broadcast  -> ValueError */
    IONP_ERR_TYPE = 2,        /* IonpError::Type       -> TypeError */
    IONP_ERR_VALUE = 3,       /* IonpError::Value      -> ValueError */
    IONP_ERR_NO_LOOP = 4,     /* IonpError::NoUfuncLoop -> UFuncTypeError */
    IONP_ERR_AXIS = 5,        /* IonpError::AxisError  -> AxisError */
    IONP_ERR_CUDA = 6,        /* a CUDA runtime call failed */
    IONP_ERR_TIMEOUT = 7,     /* a bounded device-side wait ran out */
    IONP_ERR_OOM = 8,         /* device allocation failed */
    IONP_ERR_UNSUPPORTED = 9, /* dtype/op outside this engine (e.g. complex) */
    IONP_ERR_INVALID = 10,    /* malformed descriptor or argument */
    IONP_ERR_INDEX = 11       /* IonpError::Index      -> IndexError */
};

/* FPE category bits (ionp-core/src/fpe.rs:43-48) */
enum { IONP_FPE_DIVIDE = 1, IONP_FPE_OVER = 2, IONP_FPE_UNDER = 4, IONP_FPE_INVALID = 8 };

/* casting rules for ionp_can_cast (ionp-core/src/dtype.rs:823) */
enum { IONP_CAST_NO = 0, IONP_CAST_EQUIV = 1, IONP_CAST_SAFE = 2, IONP_CAST_SAME_KIND = 3, IONP_CAST_UNSAFE = 4 };

typedef struct IonpArr {
    int32_t dtype;
    int32_t ndim;
    int64_t shape[IONP_MAX_DIMS];
    int64_t strides[IONP_MAX_DIMS]; /* elements */
    int64_t offset;                 /* elements */
    void* data;                     /* device pointer: base of the allocation */
} IonpArr;

typedef void* IonpStream; /* a cudaStream_t; NULL = the legacy default stream */

/* ---------------------------------------------------------------- queries */
/* promote_dtype (ionp-core/src/dtype.rs:297) */
int32_t ionp_promote(int32_t a, int32_t b, int32_t* out);
/* binary_out_dtype (ufunc.rs:1101) / math_binary_out_dtype (ufunc.rs:1785) */
int32_t ionp_binary_out_dtype(int32_t op, int32_t a, int32_t b, int32_t* out);
/* unary_out_dtype (ufunc.rs:1608) / math_unary_out_dtype (ufunc.rs:1682) */
int32_t ionp_unary_out_dtype(int32_t op, int32_t a, int32_t* out);
/* reduce_family_compute_dtype (ufunc.rs:2080) + supports_reduce_family (ufunc.rs:106) */
int32_t ionp_reduce_compute_dtype(int32_t op, int32_t a, int32_t* out);
/* can_cast (ionp-core/src/dtype.rs:823); *out = 0/1 */
int32_t ionp_can_cast(int32_t from, int32_t to, int32_t rule, int32_t* out);
/* One scalar converted with the reference's cast rules (Buffer::cast_to,
 * ionp-core/src/buffer.rs:64-330): used for initial= values. Host memory. */
int32_t ionp_cast_scalar(const void* src, int32_t src_dtype, void* dst, int32_t dst_dtype);
/* Element strides of the order='K' result of a call over `nops` operands
 * (ionp-py/src/lib.rs:1290-1330, ionp-core/src/array.rs:1153). */
int32_t ionp_order_k_strides(int32_t nops, const IonpArr* const* ops, int32_t ndim, const int64_t* out_shape,
                             int64_t* out_strides);
/* Shape and element strides of a reduction result
 * (ionp-core/src/array.rs:845-930, relayout_for_reduction). */
int32_t ionp_reduce_layout(const IonpArr* a, const int32_t* axes, int32_t naxes, int32_t keepdims,
                           int32_t* out_ndim, int64_t* out_shape, int64_t* out_strides);

/* ---------------------------------------------------------------- compute */
/* Element-wise binary ufunc: binary_op (ufunc.rs:3628) or math_binary_op
 * (ufunc.rs:5733) followed by write_out (ufunc.rs:10112).
 *   out   : caller-allocated, shape = broadcast(a, b) or wider (out= may
 *           broadcast up), any strides; its dtype may differ from the loop
 *           dtype (the value is cast on store, as write_into_out_ufunc does).
 *   where : NULL, or a bool mask broadcastable to out (masked store).
 *   fpe   : NULL, or a host word that receives the OR of IONP_FPE_* bits of
 *           the reference's post-hoc detector for this op
 *           (ionp-py/src/lib.rs:9077-9138); non-NULL makes the call wait for
 *           the stream. */
int32_t ionp_binary(int32_t op, const IonpArr* a, const IonpArr* b, IonpArr* out, const IonpArr* where,
                    uint32_t* fpe, IonpStream stream);
/* Element-wise unary ufunc: unary_op (ufunc.rs:3824) / math_unary_op
 * (ufunc.rs:4606). Same out/where/fpe conventions as ionp_binary. */
int32_t ionp_unary(int32_t op, const IonpArr* a, IonpArr* out, const IonpArr* where, uint32_t* fpe,
                   IonpStream stream);
/* ionp_binary / ionp_unary that never wait for the stream. `fpe` (NULL, or
 * a host word, best from ionp_host_alloc) receives the same detector bits,
 * written by a copy in stream order: read it after the stream has
 * synchronized. For ops without a detector it is set to 0 before the call
 * returns. No counterpart in the reference, whose calls are synchronous;
 * these let a caller overlap copies and kernels of consecutive calls and
 * still get the reference's FPE categories (fpe_check_after_call,
 * ionp-py/src/lib.rs:9077-9138). */
int32_t ionp_binary_nowait(int32_t op, const IonpArr* a, const IonpArr* b, IonpArr* out, const IonpArr* where,
                           uint32_t* fpe, IonpStream stream);
int32_t ionp_unary_nowait(int32_t op, const IonpArr* a, IonpArr* out, const IonpArr* where, uint32_t* fpe,
                          IonpStream stream);
/* Element-wise dtype conversion/copy of `a` into `out` (same shape, any
 * strides): Buffer::cast_to (ionp-core/src/buffer.rs:210). */
int32_t ionp_cast(const IonpArr* a, IonpArr* out, IonpStream stream);
/* ndarray.astype (ionp-py/src/lib.rs:5960-6003): the cast above preceded
 * by detect_cast_overflow (ionp-core/src/fpe.rs:398). fpe (NULL, or a host
 * word) receives IONP_FPE_INVALID when a float source holds a NaN, an
 * infinity or a value outside the integer destination's range; other
 * casts never flag. A non-NULL fpe makes the call wait for the stream. */
int32_t ionp_astype(const IonpArr* a, IonpArr* out, uint32_t* fpe, IonpStream stream);
/* ufunc.reduce: reduce_axis (ufunc.rs:7634).
 *   axes          : normalized, sorted, unique (normalize_reduce_axes, ufunc.rs:7551)
 *   compute_dtype : -1 = reduce_family_compute_dtype, else the dtype= override
 *   initial       : NULL, or a HOST pointer to one value of the compute dtype
 *   where         : NULL, or a mask broadcastable to a (any dtype, cast to bool)
 *   out           : caller-allocated, the kept shape (keepdims or not), any
 *                   strides; value cast on store when its dtype differs. */
int32_t ionp_reduce(int32_t op, const IonpArr* a, const int32_t* axes, int32_t naxes, int32_t keepdims,
                    int32_t compute_dtype, const void* initial, const IonpArr* where, IonpArr* out,
                    IonpStream stream);
/* ufunc.reduce that allocates no device memory. This entry point has no
 * counterpart in the reference; it exists for callers that cannot let the
 * library call cudaMalloc (a process that reserves its device memory up front
 * and forbids later allocations, a host runtime that owns every device byte
 * and passes in only its own buffers, a latency-critical loop that cannot
 * afford an allocation's implicit synchronisation). It computes what
 * ionp_reduce computes -- same arguments, minus the dtype override and the
 * where= mask, with compute_dtype = reduce_family_compute_dtype -- but keeps
 * the partial results of long runs in one fixed device array of
 * IONP_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads
 * the library holds until the process exits. It never calls cudaMalloc,
 * cudaFree or the library's caching allocator.
 *   - Handles the layouts the row (pairwise-tree) kernels reduce in place:
 *     the reduced axes form one run holding the smallest strides, input in
 *     the compute dtype (integer add/multiply widening on load is allowed),
 *     non-empty reduced extent. Others return IONP_ERR_UNSUPPORTED.
 *   - Returns IONP_ERR_VALUE when the partials of a call would exceed
 *     IONP_NOALLOC_SCRATCH_BYTES (at most 2^17 float64 partials: e.g. one
 *     output up to 2^33 elements, or up to 2^17 outputs of runs longer than
 *     65536 elements).
 *   - The first call on a device looks up the array's device address with
 *     that device current; make that first call before any stream capture.
 *     With CUDA's lazy module loading (the default) that first call also
 *     loads the library's kernels and the array onto the device, which the
 *     driver allocates: a caller that reserves its whole memory budget up
 *     front should make one warm-up call (any supported reduction) first.
 *   - The address is cached per device for the life of the process; do not
 *     reset the device (cudaDeviceReset) while using this entry point.
 *   - All calls share the one array: calls that overlap on the GPU (on
 *     different streams, or from several threads) race on it. Serialise them
 *     on one stream. */
#define IONP_NOALLOC_SCRATCH_BYTES (1u << 20)
int32_t ionp_reduce_noalloc(int32_t op, const IonpArr* a, const int32_t* axes, int32_t naxes, int32_t keepdims,
                            const void* initial, IonpArr* out, IonpStream stream);
/* ufunc.accumulate / cumsum / cumprod: accumulate_axis (ufunc.rs:7967):
 * every fiber along `axis` (0 <= axis < ndim) folded in order, acc = x0,
 * acc = op(acc, x_i), in reduce_family_compute_dtype (ufunc.rs:2080).
 * out: a's shape, any strides, cast on store. */
int32_t ionp_accumulate(int32_t op, const IonpArr* a, int32_t axis, IonpArr* out, IonpStream stream);
/* ufunc.reduceat: reduceat_binary_axis (ufunc.rs:8450): segment k of every
 * fiber is x[indices[k]] .. x[indices[k+1] - 1] (to the axis end for the
 * last), folded in order, or x[indices[k]] alone when indices[k+1] <=
 * indices[k]. indices: HOST int64 array, each in [0, a.shape[axis]), else
 * IONP_ERR_INDEX. out: a's shape with the axis extent nindices. */
int32_t ionp_reduceat(int32_t op, const IonpArr* a, int32_t axis, const int64_t* indices, int64_t nindices,
                      IonpArr* out, IonpStream stream);
/* ufunc.at, in place on `target`: at_binary (ufunc.rs:9577),
 * at_math_binary (ufunc.rs:9932; remainder, fmod), at_unary (ufunc.rs:9301)
 * and at_math_unary (ufunc.rs:9805). For i in order,
 * target[indices[i], ...] = op(target[indices[i], ...], values[i, ...]),
 * values broadcast against (nindices,) + target.shape[1:] as a whole;
 * repeated indices apply in order; computed in the target's dtype
 * (comparisons: 0/1 of it; logical ops: in bool) or, when the ufunc
 * promotes, on a whole-target copy in the promoted dtype that is cast back
 * element by element. Unary ops (values NULL) apply once per occurrence.
 * indices: HOST int64, negative counts from the end, each within axis 0
 * (a 0-d target takes nindices = 0 and applies once), else IONP_ERR_INDEX.
 * Values that share memory with the target are read as they were before
 * the call. No FPE report (the reference's .at has none). */
int32_t ionp_at(int32_t op, IonpArr* target, const int64_t* indices, int64_t nindices, const IonpArr* values,
                IonpStream stream);
/* argmin (is_max=0) / argmax (is_max=1): argext (ufunc.rs:8131) behind
 * do_argext (ionp-py/src/reductions.rs:1198). axis = -1 means the flattened
 * C-order ravel (axis=None); out is int64 with the kept shape. */
int32_t ionp_argext(int32_t is_max, const IonpArr* a, int32_t axis, int32_t keepdims, IonpArr* out,
                    IonpStream stream);

/* ---------------------------------------------------------------- batches */
/* Many small calls as one persistent kernel over a device queue of call
 * descriptors, captured in a CUDA graph. No counterpart in the reference,
 * which runs each call on its own (ionp-py/src/lib.rs:9205 __call__,
 * lib.rs:9959 reduce); every call computes exactly what ionp_binary /
 * ionp_reduce compute for it.
 *
 * A schedule is a point of a 48-point space: block tile {128,256,512,1024} x
 * vector width {1,2,4} (16-byte units) x elements per thread {1,4} x
 * reduction split {1,2}. It changes how a call is cut into tiles and mapped
 * to threads, never a result bit. Index order: block tile slowest, split
 * fastest (ionp_schedule_from_index). */
typedef struct IonpSchedule {
    int32_t block_tile, vec_width, elems_per_thread, red_split;
} IonpSchedule;
#define IONP_NUM_SCHEDULES 48
int32_t ionp_schedule_from_index(int32_t idx, IonpSchedule* s);

typedef struct IonpBatch IonpBatch;
int32_t ionp_batch_create(IonpBatch** b);
int32_t ionp_batch_destroy(IonpBatch* b);
/* Binary call: add, subtract, multiply, maximum, less, logical_and; any
 * dtypes, broadcasting and strides (at most 4 merged dims, fewer than 2^31
 * output elements). sched NULL = the default schedule. */
int32_t ionp_batch_add_binary(IonpBatch* b, int32_t op, const IonpArr* a, const IonpArr* bb, IonpArr* out,
                              const IonpSchedule* sched, int32_t* call_id);
/* add.reduce / maximum.reduce over one axis of a C-contiguous array into a
 * C-contiguous output of the compute dtype. */
int32_t ionp_batch_add_reduce(IonpBatch* b, int32_t op, const IonpArr* a, int32_t axis, int32_t keepdims, IonpArr* out,
                              const IonpSchedule* sched, int32_t* call_id);
int32_t ionp_batch_set_schedule(IonpBatch* b, int32_t call, const IonpSchedule* sched);
/* Plans the tiles and uploads the queue (run does it when needed). */
int32_t ionp_batch_finalize(IonpBatch* b, IonpStream stream);
/* Runs every call: one persistent kernel; use_graph=1 captures the run once
 * in a CUDA graph and replays the graph afterwards. */
int32_t ionp_batch_run(IonpBatch* b, int32_t use_graph, IonpStream stream);
/* The same calls, one ionp_binary / ionp_reduce launch per call (default
 * schedules): the baseline the batch is measured against. */
int32_t ionp_batch_run_per_call(IonpBatch* b, IonpStream stream);
/* FPE words (IONP_FPE_* bits) of every call of the last run, caller order.
 * The batch pairs operands by broadcasting; for float multiply calls whose
 * operands are not trailing-aligned the reference's detector pairs them by
 * flat index, which ionp_binary reproduces and the batch does not. */
int32_t ionp_batch_fpe(IonpBatch* b, uint32_t* words, IonpStream stream);
/* info[0] calls, [1] tiles, [2] grid, [3] dynamic shared bytes,
 * [4] algorithmic bytes of one run */
int32_t ionp_batch_info(IonpBatch* b, int64_t* info);
/* Device microseconds of one call under each schedule as a batch sees it
 * (the autotuner's measurement): the call is queued enough times in one
 * launch for four tiles per resident CTA (at most 4096 copies, all fitting a
 * 1 GiB pool), each copy on its own operand region of the pool, so copies
 * stream from HBM like distinct calls; reps launches between two events;
 * time per copy. Only shapes, strides and dtypes matter: the pool's
 * contents are arbitrary. */
int32_t ionp_batch_time_call(IonpBatch* b, int32_t call, int32_t nsched, const IonpSchedule* scheds, int32_t reps,
                             float* us_out, IonpStream stream);

/* Feature vector of one queued call for the schedule picker. */
#define IONP_PICKER_FEATURES 32
int32_t ionp_batch_features(IonpBatch* b, int32_t call, float* features);

/* ------------------------------------------------------- schedule picker net */
/* A 3-layer perceptron (FP32, ReLU hidden layers) with hand-written forward,
 * backward and Adam kernels; it predicts each schedule's log-time from a
 * call's features. No counterpart in the reference. x, t, mask and y are
 * DEVICE float arrays, row-major [batch][features] / [batch][outputs]. */
typedef struct IonpMlp IonpMlp;
int32_t ionp_mlp_create(IonpMlp** m, int32_t nin, int32_t hidden, int32_t nout, uint64_t seed);
int32_t ionp_mlp_destroy(IonpMlp* m);
int32_t ionp_mlp_num_params(IonpMlp* m, int64_t* n);
/* which = 0: parameters; 1: gradients of the last gradients/train step.
 * Layout: W1[nin][h], b1[h], W2[h][h], b2[h], W3[h][nout], b3[nout]. */
int32_t ionp_mlp_get(IonpMlp* m, int32_t which, float* host, int64_t n);
int32_t ionp_mlp_set_params(IonpMlp* m, const float* host, int64_t n);
int32_t ionp_mlp_forward(IonpMlp* m, const float* x, int32_t batch, float* y, IonpStream stream);
/* mean squared error over the (masked) outputs and its gradients; loss may be
 * NULL (then the call does not wait for the stream) */
int32_t ionp_mlp_gradients(IonpMlp* m, const float* x, const float* t, const float* mask, int32_t batch, float* loss,
                           IonpStream stream);
/* gradients + one Adam step (beta 0.9 / 0.999, eps 1e-8, decoupled-free L2 weight_decay) */
int32_t ionp_mlp_train_step(IonpMlp* m, const float* x, const float* t, const float* mask, int32_t batch, float lr,
                            float weight_decay, float* loss, IonpStream stream);

/* ---------------------------------------------------------------- memory */
/* Caching device allocator (the device counterpart of Buffer's Vec<T>,
 * ionp-core/src/buffer.rs:18): one pool per device (blocks are allocated
 * on, and reused only on, the device current at ionp_alloc), size-classed
 * free lists, stream-ordered reuse (a block freed on one stream is reused
 * on another only after an event wait). A failed cudaMalloc releases the
 * device's cached blocks and retries once, then returns IONP_ERR_OOM. */
int32_t ionp_alloc(void** ptr, size_t bytes, IonpStream stream);
int32_t ionp_free(void* ptr, IonpStream stream);
/* current device's pool, bytes: [0] in use, [1] cached (free), [2] peak in
 * use, [3] cudaMalloc calls */
int32_t ionp_alloc_stats(uint64_t* stats4);
int32_t ionp_alloc_trim(void);

/* ---------------------------------------------------------------- runtime */
/* Thin runtime helpers so hosts need no CUDA bindings of their own. */
enum { IONP_H2D = 0, IONP_D2H = 1, IONP_D2D = 2 };
int32_t ionp_memcpy(void* dst, const void* src, size_t bytes, int32_t kind, IonpStream stream);
int32_t ionp_stream_create(IonpStream* stream);
int32_t ionp_stream_destroy(IonpStream stream);
int32_t ionp_stream_synchronize(IonpStream stream);
int32_t ionp_device_synchronize(void);
/* pinned host memory (page-locked; fast, asynchronous copies) */
int32_t ionp_host_alloc(void** ptr, size_t bytes);
int32_t ionp_host_free(void* ptr);
/* events for device-side timing on a stream */
int32_t ionp_event_create(void** ev);
int32_t ionp_event_destroy(void* ev);
int32_t ionp_event_record(void* ev, IonpStream stream);
int32_t ionp_event_elapsed_ms(void* start, void* stop, float* ms);
/* select the CUDA device used by the calling host thread */
int32_t ionp_set_device(int32_t device);
/* device name / SM count / whether a device is present (count=0 if none) */
int32_t ionp_device_info(int32_t* count, int32_t* sm_count, char* name, size_t len);

/* ---------------------------------------------------------------- misc */
/* Copies the last error message of the calling thread (NUL-terminated). */
int32_t ionp_last_error_message(char* buf, size_t len);
/* Number of kernels this library has launched since load (all streams). */
uint64_t ionp_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* IONP_CUDA_H */
