// Row (tree) reduction kernels: bitwise, logical and bool equal/not_equal.
#include "ionp_reduce_row_impl.cuh"

namespace ionp {

cudaError_t launch_reduce_row_b(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s, bool top) {
    switch (d.op) {
        case OP_BITWISE_AND: return row_op<OP_BITWISE_AND>(d, tpr, smem, grid, s, top);
        case OP_BITWISE_OR: return row_op<OP_BITWISE_OR>(d, tpr, smem, grid, s, top);
        case OP_BITWISE_XOR: return row_op<OP_BITWISE_XOR>(d, tpr, smem, grid, s, top);
        case OP_LOGICAL_AND: return row_op<OP_LOGICAL_AND>(d, tpr, smem, grid, s, top);
        case OP_LOGICAL_OR: return row_op<OP_LOGICAL_OR>(d, tpr, smem, grid, s, top);
        case OP_LOGICAL_XOR: return row_op<OP_LOGICAL_XOR>(d, tpr, smem, grid, s, top);
        case OP_EQUAL: return row_op<OP_EQUAL>(d, tpr, smem, grid, s, top);
        case OP_NOT_EQUAL: return row_op<OP_NOT_EQUAL>(d, tpr, smem, grid, s, top);
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
