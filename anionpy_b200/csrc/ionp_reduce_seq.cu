// Sequential (column) reduction kernels and the general wide x narrow kernel.
#include "ionp_reduce_row_impl.cuh"

namespace ionp {

static int seq_grid(int64_t nout, int threads) {
    int64_t g = (nout + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > sm_count() * 16) g = sm_count() * 16;
    return (int)g;
}

// The staged column kernel applies to one narrow axis over one contiguous
// kept axis, 4- or 8-byte elements, 16-byte aligned rows.
static bool col_staged_ok(const RedDesc& d, int es) {
    if (d.adt != d.cd || (es != 4 && es != 8)) return false;
    if (d.nr != 1 || d.nk != 1 || d.kst[0] != 1 || d.rst[0] <= 0) return false;
    if (d.kshape[0] % (16 / es) != 0 || (d.rst[0] * es) % 16 != 0) return false;
    if (reinterpret_cast<uintptr_t>(d.a) % 16 != 0) return false;
    // with 64K or more outputs one thread per output already keeps enough
    // loads in flight; the staged kernel pays off below that
    return d.rshape[0] >= 64 && d.kshape[0] >= 128 / es && d.nout < 65536;
}

template <int OPV, int D>
static cudaError_t col_staged(const RedDesc& d, cudaStream_t s) {
    typedef typename DT<D>::T T;
    const size_t smem = colst_smem<T>();
    auto k = k_red_col_staged<OPV, D>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int64_t tiles = (d.kshape[0] + colst_cols<T>() - 1) / colst_cols<T>();
    const int64_t cap = (int64_t)sm_count() * COLST_CTAS;
    int grid = (int)(tiles < cap ? tiles : cap);
    k<<<grid, RED_THREADS, smem, s>>>(d);
    count_launch();
    return cudaGetLastError();
}

template <int OPV>
static cudaError_t col_op(const RedDesc& d, cudaStream_t s) {
    const bool castld = d.adt != d.cd;
    const int grid = seq_grid(d.nout, RED_THREADS);
    // fewer than 64K outputs over one long narrow axis of 4- or 8-byte
    // elements: one thread per output, two register batches of loads
    if (!castld && d.nr == 1 && d.nout < 65536 && d.rshape[0] >= 256 && dt_size(d.cd) >= 4) {
        const int pgrid = seq_grid(d.nout, COLP_THREADS);
#define IONP_U64CASE(D)                                                                  \
        case D:                                                                          \
            if constexpr (red_any_valid(OPV, D) && (sizeof(typename DT<D>::T) >= 4)) {   \
                k_red_col_pipe<OPV, D, sizeof(typename DT<D>::T) == 4 ? 64 : 32><<<pgrid, COLP_THREADS, 0, s>>>(d); \
                count_launch();                                                          \
                return cudaGetLastError();                                               \
            }                                                                            \
            break;
        switch (d.cd) { IONP_DTS(IONP_U64CASE) }
#undef IONP_U64CASE
    }
    if (col_staged_ok(d, dt_size(d.cd))) {
#define IONP_STCASE(D)                                                                   \
        case D:                                                                          \
            if constexpr (red_any_valid(OPV, D) && (sizeof(typename DT<D>::T) >= 4))     \
                return col_staged<OPV, D>(d, s);                                         \
            break;
        switch (d.cd) { IONP_DTS(IONP_STCASE) }
#undef IONP_STCASE
    }
#define IONP_DTCASE(D)                                                                          \
    case D:                                                                                     \
        if constexpr (red_any_valid(OPV, D)) {                                                  \
            if constexpr (red_castld_ok(OPV, D)) {                                              \
                if (castld) { k_red_col<OPV, D, true><<<grid, RED_THREADS, 0, s>>>(d); count_launch(); return cudaGetLastError(); } \
            }                                                                                   \
            if (castld) return cudaErrorInvalidValue;                                           \
            k_red_col<OPV, D, false><<<grid, RED_THREADS, 0, s>>>(d);                           \
            count_launch();                                                                     \
            return cudaGetLastError();                                                          \
        }                                                                                       \
        break;
    switch (d.cd) { IONP_DTS(IONP_DTCASE) }
#undef IONP_DTCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce_col(const RedDesc& d, cudaStream_t s) {
#define IONP_OPCASE(OP) case OP: return col_op<OP>(d, s);
    switch (d.op) { IONP_RED_OPS(IONP_OPCASE) }
#undef IONP_OPCASE
    return cudaErrorInvalidValue;
}

template <int OPV>
static cudaError_t col_split_op(const RedDesc& d, cudaStream_t s) {
    const int64_t ntask = d.nout << d.K;
    int64_t g = (ntask + RED_THREADS - 1) / RED_THREADS;
    if (g > sm_count() * 8) g = sm_count() * 8;
    const int grid = (int)(g < 1 ? 1 : g);
#define IONP_DTCASE(D)                                                  \
    case D:                                                             \
        if constexpr (red_assoc(OPV, D)) {                              \
            k_red_col_split<OPV, D><<<grid, RED_THREADS, 0, s>>>(d);    \
            count_launch();                                             \
            return cudaGetLastError();                                  \
        }                                                               \
        break;
    switch (d.cd) { IONP_DTS(IONP_DTCASE) }
#undef IONP_DTCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce_col_split(const RedDesc& d, cudaStream_t s) {
#define IONP_OPCASE(OP) case OP: return col_split_op<OP>(d, s);
    switch (d.op) { IONP_RED_OPS(IONP_OPCASE) }
#undef IONP_OPCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce_gen(const RedDesc& d, cudaStream_t s) {
    int grid = seq_grid(d.nout, 128);
    switch (d.cd) {
        case DT_F32: if (d.op == OP_ADD) { k_red_gen<OP_ADD, DT_F32><<<grid, 128, 0, s>>>(d); count_launch(); return cudaGetLastError(); } break;
        case DT_F64: if (d.op == OP_ADD) { k_red_gen<OP_ADD, DT_F64><<<grid, 128, 0, s>>>(d); count_launch(); return cudaGetLastError(); } break;
        case DT_F16:
            switch (d.op) {
                case OP_ADD: k_red_gen<OP_ADD, DT_F16><<<grid, 128, 0, s>>>(d); break;
                case OP_MULTIPLY: k_red_gen<OP_MULTIPLY, DT_F16><<<grid, 128, 0, s>>>(d); break;
                case OP_SUBTRACT: k_red_gen<OP_SUBTRACT, DT_F16><<<grid, 128, 0, s>>>(d); break;
                case OP_DIVIDE: k_red_gen<OP_DIVIDE, DT_F16><<<grid, 128, 0, s>>>(d); break;
                default: return cudaErrorInvalidValue;
            }
            count_launch();
            return cudaGetLastError();
    }
    return cudaErrorInvalidValue;
}

}  // namespace ionp
