// Instantiations and launchers of the argmin/argmax kernels.
#include "ionp_reduce_launch.cuh"

namespace ionp {

template <int CD, bool MAX>
static cudaError_t arg_t(const RedDesc& d, int mode, int tpr, cudaStream_t s) {
    if (mode == 1) {  // column scan
        int64_t g = (d.nout + RED_THREADS - 1) / RED_THREADS;
        if (g > 148 * 16) g = 148 * 16;
        k_argext_col<CD, MAX><<<(int)(g < 1 ? 1 : g), RED_THREADS, 0, s>>>(d);
        count_launch();
        return cudaGetLastError();
    }
    if (mode == 2) {  // top of a split scan
        int64_t g = (d.nout + 127) / 128;
        if (g > 148 * 16) g = 148 * 16;
        k_argext_top<CD, MAX><<<(int)(g < 1 ? 1 : g), 128, 0, s>>>(d);
        count_launch();
        return cudaGetLastError();
    }
    const int64_t ntasks = d.nout << d.K;
    const int groups = RED_THREADS / tpr;
    int64_t g = (ntasks + groups - 1) / groups;
    if (g > 148 * 16) g = 148 * 16;
    int grid = (int)(g < 1 ? 1 : g);
    switch (tpr) {
        case 1: k_argext<CD, MAX, 1><<<grid, RED_THREADS, 0, s>>>(d); break;
        case 32: k_argext<CD, MAX, 32><<<grid, RED_THREADS, 0, s>>>(d); break;
        default: k_argext<CD, MAX, 256><<<grid, RED_THREADS, 0, s>>>(d); break;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_argext(const RedDesc& d, int is_max, int mode, int tpr, cudaStream_t s) {
#define IONP_DTCASE(D) \
    case D: return is_max ? arg_t<D, true>(d, mode, tpr, s) : arg_t<D, false>(d, mode, tpr, s);
    switch (d.cd) { IONP_DTS(IONP_DTCASE) }
#undef IONP_DTCASE
    return cudaErrorInvalidValue;
}

}  // namespace ionp
