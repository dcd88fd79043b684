// Binary element-wise kernel instantiations: arith group.
#include "ionp_ew_launch.cuh"

namespace ionp {

cudaError_t launch_binary_arith(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_ADD: return launch_bin_op<OP_ADD>(cd, d, ci, f, s);
        case OP_SUBTRACT: return launch_bin_op<OP_SUBTRACT>(cd, d, ci, f, s);
        case OP_MULTIPLY: return launch_bin_op<OP_MULTIPLY>(cd, d, ci, f, s);
        case OP_DIVIDE: return launch_bin_op<OP_DIVIDE>(cd, d, ci, f, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
