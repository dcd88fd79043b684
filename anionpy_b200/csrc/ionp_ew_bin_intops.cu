// Binary element-wise kernel instantiations: intops group.
#include "ionp_ew_launch.cuh"

namespace ionp {

cudaError_t launch_binary_intops(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_BITWISE_AND: return launch_bin_op<OP_BITWISE_AND>(cd, d, ci, f, s);
        case OP_BITWISE_OR: return launch_bin_op<OP_BITWISE_OR>(cd, d, ci, f, s);
        case OP_BITWISE_XOR: return launch_bin_op<OP_BITWISE_XOR>(cd, d, ci, f, s);
        case OP_LEFT_SHIFT: return launch_bin_op<OP_LEFT_SHIFT>(cd, d, ci, f, s);
        case OP_RIGHT_SHIFT: return launch_bin_op<OP_RIGHT_SHIFT>(cd, d, ci, f, s);
        case OP_FLOOR_DIVIDE: return launch_bin_op<OP_FLOOR_DIVIDE>(cd, d, ci, f, s);
        case OP_REMAINDER: return launch_bin_op<OP_REMAINDER>(cd, d, ci, f, s);
        case OP_FMOD: return launch_bin_op<OP_FMOD>(cd, d, ci, f, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
