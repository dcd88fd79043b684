// Instantiations and launchers of the argmin/argmax kernels.
#include "ionp_reduce_launch.cuh"

#include <algorithm>

namespace ionp {

template <int CD, bool MAX>
static cudaError_t arg_t(const RedDesc& d, int mode, int tpr, cudaStream_t s) {
    if (mode == 1) {  // column scan, split 2^K ways when d.K > 0
        int64_t g = ((d.nout << d.K) + RED_THREADS - 1) / RED_THREADS;
        if (g > sm_count() * 16) g = sm_count() * 16;
        k_argext_col<CD, MAX><<<(int)(g < 1 ? 1 : g), RED_THREADS, 0, s>>>(d);
        count_launch();
        return cudaGetLastError();
    }
    if (mode == 2) {  // top of a split scan
        if (d.K <= 6) {
            int64_t g = (d.nout + RED_THREADS - 1) / RED_THREADS;
            if (g > sm_count() * 16) g = sm_count() * 16;
            k_argext_top_small<CD, MAX><<<(int)(g < 1 ? 1 : g), RED_THREADS, 0, s>>>(d);
        } else {
            int64_t g = d.nout;
            if (g > sm_count() * 8) g = sm_count() * 8;
            k_argext_top<CD, MAX><<<(int)(g < 1 ? 1 : g), RED_THREADS, 0, s>>>(d);
        }
        count_launch();
        return cudaGetLastError();
    }
    if (mode == 3) {  // many short contiguous rows
        const int64_t m = d.w * (int64_t)sizeof(typename DT<CD>::T) / 16;
        const int64_t R = std::min<int64_t>(2048, 2048 / m);
        const int64_t nwin = (d.nout + R - 1) / R;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nwin, (int64_t)sm_count() * 2));
        auto k = k_argext_nar<CD, MAX>;
        const size_t smem = 3 * 32768;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<grid, RED_THREADS, smem, s>>>(d);
        count_launch();
        return cudaGetLastError();
    }
    const int64_t ntasks = d.nout << d.K;
    const int groups = RED_THREADS / tpr;
    int64_t g = (ntasks + groups - 1) / groups;
    if (g > sm_count() * 16) g = sm_count() * 16;
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
