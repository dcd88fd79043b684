// Row (tree) reduction launch templates, included by the per-op-group
// translation units ionp_reduce_row_*.cu.
#pragma once
#include "ionp_reduce_launch.cuh"
#include "ionp_reduce_rowst.cuh"

namespace ionp {

constexpr bool red_castld_ok(int op, int cd) { return (op == OP_ADD || op == OP_MULTIPLY) && (cd == DT_I64 || cd == DT_U64); }

template <int OP, int CD, bool C>
static cudaError_t row_t2(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s) {
    if constexpr (!C) {
        cudaError_t e = launch_row_wide<OP, CD>(d, s);
        if (e != cudaErrorNotSupported) return e;
    }
    switch (tpr) {
        case 1: k_red_row<OP, CD, 1, C><<<grid, RED_THREADS, smem, s>>>(d); break;
        case 32: k_red_row<OP, CD, 32, C><<<grid, RED_THREADS, smem, s>>>(d); break;
        default: {
            auto k = k_red_row<OP, CD, 256, C>;
            if (smem > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess) return e;
            }
            k<<<grid, RED_THREADS, smem, s>>>(d);
        } break;
    }
    count_launch();
    return cudaGetLastError();
}

template <int OP, int CD>
static cudaError_t row_top_t(const RedDesc& d, cudaStream_t s) {
    typedef typename RPol<OP, CD>::A A;
    if constexpr (red_assoc(OP, CD)) {
        if (d.K <= 6 && d.nout >= sm_count() * 8) {
            int64_t g = (d.nout + RED_THREADS - 1) / RED_THREADS;
            if (g > sm_count() * 16) g = sm_count() * 16;
            k_red_row_top_small<OP, CD><<<(int)g, RED_THREADS, 0, s>>>(d);
            count_launch();
            return cudaGetLastError();
        }
    }
    if constexpr (!red_assoc(OP, CD)) {
        // many outputs of few parts: one thread per output, the tree unrolled
        if (d.K >= 1 && d.K <= 5 && d.nout >= sm_count() * 8) {
            int64_t g = (d.nout + RED_THREADS - 1) / RED_THREADS;
            if (g > sm_count() * 16) g = sm_count() * 16;
            switch (d.K) {
                case 1: k_red_row_top_tree<OP, CD, 1><<<(int)g, RED_THREADS, 0, s>>>(d); break;
                case 2: k_red_row_top_tree<OP, CD, 2><<<(int)g, RED_THREADS, 0, s>>>(d); break;
                case 3: k_red_row_top_tree<OP, CD, 3><<<(int)g, RED_THREADS, 0, s>>>(d); break;
                case 4: k_red_row_top_tree<OP, CD, 4><<<(int)g, RED_THREADS, 0, s>>>(d); break;
                default: k_red_row_top_tree<OP, CD, 5><<<(int)g, RED_THREADS, 0, s>>>(d); break;
            }
            count_launch();
            return cudaGetLastError();
        }
    }
    if (d.K > 2 * TOP_CHUNK_LOG) return cudaErrorInvalidValue;   // planners cap K far below this
    const size_t smem = row_top_smem<A>(d.K);                    // at most 32 KiB
    int grid = (int)(d.nout < sm_count() * 8 ? d.nout : sm_count() * 8);
    k_red_row_top<OP, CD><<<grid, RED_THREADS, smem, s>>>(d);
    count_launch();
    return cudaGetLastError();
}

template <int OPV>
static cudaError_t row_op(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s, bool top) {
    const bool castld = d.adt != d.cd;
#define IONP_DTCASE(D)                                                                  \
    case D:                                                                             \
        if constexpr (red_row_valid(OPV, D)) {                                          \
            if (top) return row_top_t<OPV, D>(d, s);                                    \
            if constexpr (red_castld_ok(OPV, D)) {                                      \
                if (castld) return row_t2<OPV, D, true>(d, tpr, smem, grid, s);         \
            }                                                                           \
            if (castld) return cudaErrorInvalidValue;                                   \
            return row_t2<OPV, D, false>(d, tpr, smem, grid, s);                        \
        }                                                                               \
        break;
    switch (d.cd) { IONP_DTS(IONP_DTCASE) }
#undef IONP_DTCASE
    return cudaErrorInvalidValue;
}

}  // namespace ionp
