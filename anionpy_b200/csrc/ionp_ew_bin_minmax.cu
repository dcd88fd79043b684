// Binary element-wise kernel instantiations: minmax group.
#include "ionp_ew_launch.cuh"

namespace ionp {

cudaError_t launch_binary_minmax(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_MAXIMUM: return launch_bin_op<OP_MAXIMUM>(cd, d, ci, f, s);
        case OP_MINIMUM: return launch_bin_op<OP_MINIMUM>(cd, d, ci, f, s);
        case OP_LOGICAL_AND: return launch_bin_op<OP_LOGICAL_AND>(cd, d, ci, f, s);
        case OP_LOGICAL_OR: return launch_bin_op<OP_LOGICAL_OR>(cd, d, ci, f, s);
        case OP_LOGICAL_XOR: return launch_bin_op<OP_LOGICAL_XOR>(cd, d, ci, f, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
