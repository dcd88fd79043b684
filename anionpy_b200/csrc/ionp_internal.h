// Internal plan structures shared by the host engine (ionp_engine.cu) and
// the kernel files. Not part of the C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/ionp_cuda.h"

namespace ionp {

constexpr int EW_MAXD = 4;  // merged dims handled by the element-wise kernels

// One operand of an element-wise launch after dim merging: pointer to its
// first element, runtime dtype and element strides over the merged dims.
struct EwOperand {
    const void* p;
    int32_t dt;
    int64_t st[EW_MAXD];
};

// Element-wise launch descriptor (passed by value to the kernels).
struct EwDesc {
    int32_t nd;                 // merged dims (1..EW_MAXD)
    int64_t shape[EW_MAXD];
    int64_t n;                  // total elements
    EwOperand a, b, m;          // m = where mask (p == nullptr: none)
    void* o;                    // output first element
    int32_t odt;
    int64_t so[EW_MAXD];
};

// Result of the host check for the vectorised contiguous path.
struct ContigInfo {
    bool ok;            // all operands same dtype as the loop, unit/zero strides, 16B aligned
    bool a_scalar, b_scalar;
};

// Launchers (defined in the kernel files). Return a cudaError_t.
cudaError_t launch_binary(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* dflags, cudaStream_t s);
cudaError_t launch_unary(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* dflags, cudaStream_t s);
// streaming multiprocessors of the current device (queried once per device)
int sm_count();
cudaError_t launch_cast(const EwDesc& d, cudaStream_t s);
cudaError_t launch_cast_check(const EwDesc& d, double lo, double hi, uint32_t* flags, cudaStream_t s);
// FPE detector with the reference's flat `x[i % len]` operand pairing, for
// calls where it differs from true broadcasting (fpe.rs:173-300).
struct FpeQuirkDesc {
    int kind;               // 1 divide family, 2 integer remainder, 3 float multiply
    int out_is_float;
    int64_t n;              // max(len_a, len_b, len_out)
    int64_t la, lb, lo;
    const void* a; int32_t da; int32_t nda; int64_t sha[32]; int64_t sta[32];
    const void* b; int32_t dbt; int32_t ndb; int64_t shb[32]; int64_t stb[32];
    const void* o; int32_t dout; int32_t ndo; int64_t sho[32]; int64_t sto[32];
};
cudaError_t launch_fpe_quirk(const FpeQuirkDesc& d, uint32_t* dflags, cudaStream_t s);

void count_launch(int k = 1);

}  // namespace ionp
