// Binary element-wise kernel instantiations: cmp group.
#include "ionp_ew_launch.cuh"

namespace ionp {

cudaError_t launch_binary_cmp(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_GREATER: return launch_bin_op<OP_GREATER>(cd, d, ci, f, s);
        case OP_GREATER_EQUAL: return launch_bin_op<OP_GREATER_EQUAL>(cd, d, ci, f, s);
        case OP_LESS: return launch_bin_op<OP_LESS>(cd, d, ci, f, s);
        case OP_LESS_EQUAL: return launch_bin_op<OP_LESS_EQUAL>(cd, d, ci, f, s);
        case OP_EQUAL: return launch_bin_op<OP_EQUAL>(cd, d, ci, f, s);
        case OP_NOT_EQUAL: return launch_bin_op<OP_NOT_EQUAL>(cd, d, ci, f, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
