// Host-side helpers shared by the engine translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/ionp_cuda.h"

namespace ionp {

// --- errors ---------------------------------------------------------------
int32_t set_err(int32_t status, const std::string& msg);
int32_t cuda_err(cudaError_t e, const char* where);
std::string fmt_shape(const int64_t* shape, int nd);
const char* op_name(int op);

// --- dtype rules ------------------------------------------------------------
bool dt_valid(int d);
int promote(int a, int b);
int32_t binary_loop(int op, int a, int b, int* cd, int* rd);   // loop and result dtype
int32_t unary_loop(int op, int a, int* cd, int* rd);
int32_t reduce_cd(int op, int a, int* cd);
bool can_cast(int from, int to, int rule);
const char* dt_name(int d);
int dt_bytes(int d);
// host copy of the reference cast of one scalar (buffer.rs casts)
void host_cast_scalar(const void* src, int sd, void* dst, int dd);

// --- arrays -----------------------------------------------------------------
int32_t check_arr(const IonpArr* a, const char* what);
inline int64_t numel(const IonpArr* a) {
    int64_t n = 1;
    for (int i = 0; i < a->ndim; ++i) n *= a->shape[i];
    return n;
}
inline const char* elem_ptr(const IonpArr* a) {
    return (const char*)a->data + a->offset * (int64_t)dt_bytes(a->dtype);
}
// broadcast_strides_to (shape.rs:113): strides of `a` viewed with `shape`
bool bcast_strides(const IonpArr* a, int nd, const int64_t* shape, int64_t* out);

// Dim merging of an element-wise call: up to 4 operands (output first) over
// one shape; drops unit dims, orders dims by |output stride| (outermost
// first) and merges neighbours whose strides chain for every operand.
struct MergeIn {
    int nd;
    int64_t shape[IONP_MAX_DIMS];
    int nops;
    int64_t st[4][IONP_MAX_DIMS];
};
struct MergeOut {
    int nd;
    int64_t shape[IONP_MAX_DIMS];
    int64_t st[4][IONP_MAX_DIMS];
};
MergeOut merge_dims(const MergeIn& in);

// element-wise cast/copy of a into out with an optional bool mask
int32_t cast_impl(const IonpArr* a, IonpArr* out, const IonpArr* where, cudaStream_t s);

// --- tracing ------------------------------------------------------------------
// An NVTX range over the scope (a C-ABI call, a batch run), named after the
// entry point; on only when the environment sets IONP_NVTX=1 (read once), so
// a profiler's timeline can show each call, and nothing is done otherwise.
struct NvtxRange {
    bool on;
    explicit NvtxRange(const char* name);
    ~NvtxRange();
};

// --- scratch memory from the caching allocator -------------------------------
void* scratch_alloc(size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);

// FPE word helpers: device flag word from the allocator, read back after the
// stream drains.
// One device word per device that kernels set when a bounded wait of theirs
// gives up (a bulk copy that never completes); null if it cannot be had.
// ionp_stream_synchronize / ionp_device_synchronize report it as
// IONP_ERR_TIMEOUT and clear it.
uint32_t* async_error_word();
int32_t check_async_error();

struct FlagWord {
    uint32_t* d = nullptr;
    cudaStream_t s = nullptr;
    int32_t open(cudaStream_t st);
    int32_t read(uint32_t* host);
    // stream-ordered copy into a caller's (pinned) host word; no wait
    int32_t read_async(uint32_t* host);
    // read() or read_async() by the call's mode
    int32_t deliver(uint32_t* host, bool nowait) { return nowait ? read_async(host) : read(host); }
    ~FlagWord();
};

}  // namespace ionp
