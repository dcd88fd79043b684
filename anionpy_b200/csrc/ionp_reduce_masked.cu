// where= reduction kernels.
#include "ionp_reduce_launch.cuh"

namespace ionp {

template <int OPV>
static cudaError_t masked_op(const RedDesc& d, cudaStream_t s) {
    int64_t g = (d.nout + 127) / 128;
    if (g < 1) g = 1;
    if (g > sm_count() * 16) g = sm_count() * 16;
#define IONP_DTCASE(D)                                                     \
    case D:                                                                \
        if constexpr (red_any_valid(OPV, D)) {                             \
            k_red_masked<OPV, D><<<(int)g, 128, 0, s>>>(d);                \
            count_launch();                                                \
            return cudaGetLastError();                                     \
        }                                                                  \
        break;
    switch (d.cd) { IONP_DTS(IONP_DTCASE) }
#undef IONP_DTCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce_masked(const RedDesc& d, cudaStream_t s) {
#define IONP_OPCASE(OP) case OP: return masked_op<OP>(d, s);
    switch (d.op) { IONP_RED_OPS(IONP_OPCASE) }
#undef IONP_OPCASE
    return cudaErrorInvalidValue;
}

}  // namespace ionp
