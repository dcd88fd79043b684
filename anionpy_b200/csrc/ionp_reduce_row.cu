// Row (tree) reduction kernels: add / multiply / maximum / minimum.
#include "ionp_reduce_row_impl.cuh"

namespace ionp {

bool reduce_row_supported(int op, int cd) { return red_row_valid(op, cd); }

cudaError_t launch_reduce_row_b(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s, bool top);

static cudaError_t row_dispatch(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s, bool top) {
    switch (d.op) {
        case OP_ADD: return row_op<OP_ADD>(d, tpr, smem, grid, s, top);
        case OP_MULTIPLY: return row_op<OP_MULTIPLY>(d, tpr, smem, grid, s, top);
        case OP_MAXIMUM: return row_op<OP_MAXIMUM>(d, tpr, smem, grid, s, top);
        case OP_MINIMUM: return row_op<OP_MINIMUM>(d, tpr, smem, grid, s, top);
    }
    return launch_reduce_row_b(d, tpr, smem, grid, s, top);
}

cudaError_t launch_reduce_row(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s) {
    return row_dispatch(d, tpr, smem, grid, s, false);
}
cudaError_t launch_reduce_row_top(const RedDesc& d, cudaStream_t s) { return row_dispatch(d, 0, 0, 0, s, true); }

}  // namespace ionp
