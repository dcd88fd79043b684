// ufunc.accumulate (cumsum / cumprod) and ufunc.reduceat: folds in order
// along one axis.
//
// accumulate_axis (ionp-core/src/ufunc.rs:7967-8035) and reduceat_binary_axis
// (ufunc.rs:8450-8483, reduceat_axis_generic 8322) walk every fiber parallel
// to the axis (one position of every other axis) and fold it left to right:
// acc = x0, then acc = f(acc, x_i). The fold is the scalar op table of the
// ufunc call (BinOp), in the compute dtype of reduce_family_compute_dtype
// (ufunc.rs:2080); inputs are converted on load, results on store.
//
//  k_scan_fiber  one thread per fiber, in order along the axis. Every op;
//                the only exact form for float add / multiply and the other
//                order-dependent folds (subtract, divide, shifts, ...).
//  k_scan_part, k_scan_carry, k_scan_apply
//                folds that are associative bit for bit (wrapping integer
//                add / multiply, bitwise and logical ops, integer and float
//                maximum / minimum, whose first NaN and tie rules hold for
//                any grouping) over few long fibers: each fiber is cut into
//                P parts; pass 1 folds each part, pass 2 turns a fiber's part
//                totals into exclusive carries in order, pass 3 rescans each
//                part from its carry. Equal to the sequential fold.
//  k_reduceat    one thread per (segment, fiber): out[k] = the fold of
//                x[idx_k], ..., x[next_k - 1] (next_k = idx_{k+1}, or the axis
//                length for the last segment), or x[idx_k] alone when
//                next_k <= idx_k.
#include <algorithm>
#include <cstring>
#include <vector>
#include "ionp_host.h"
#include "ionp_ew_launch.cuh"

namespace ionp {

constexpr int SC_MAXD = 6;   // kept dims of one launch (more: a host loop)
constexpr int SC_THREADS = 256;

struct ScanDesc {
    const void* a;
    int32_t adt;
    void* o;
    int32_t odt;
    int64_t len, sa, so;            // axis extent and element strides along it
    int32_t nk;
    int64_t kshape[SC_MAXD], kst[SC_MAXD], kost[SC_MAXD];
    int64_t nfib;
    const int64_t* idx;             // reduceat: segment starts (device)
    int64_t nseg;
    int64_t parts;                  // split scan: parts per fiber
    void* carry;                    // split scan: nfib * parts values
};

__device__ __forceinline__ void fiber_offsets(const ScanDesc& d, int64_t f, int64_t* ia, int64_t* io) {
    int64_t a = 0, o = 0;
    for (int k = d.nk - 1; k >= 0; --k) {
        const int64_t q = f / d.kshape[k];
        const int64_t i = f - q * d.kshape[k];
        f = q;
        a += i * d.kst[k];
        o += i * d.kost[k];
    }
    *ia = a;
    *io = o;
}

template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_scan_fiber(ScanDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < d.nfib; f += stride) {
        int64_t ia, io;
        fiber_offsets(d, f, &ia, &io);
        T acc = load_cast<CD>(d.a, ia, d.adt);
        store_cast<CD>(d.o, io, d.odt, acc);
        for (int64_t i = 1; i < d.len; ++i) {
            acc = (T)BinOp<OP, CD>::apply(acc, load_cast<CD>(d.a, ia + i * d.sa, d.adt));
            store_cast<CD>(d.o, io + i * d.so, d.odt, acc);
        }
    }
}

__device__ __forceinline__ void part_range(const ScanDesc& d, int64_t p, int64_t* lo, int64_t* hi) {
    *lo = p * d.len / d.parts;
    *hi = (p + 1) * d.len / d.parts;
}

// pass 1: the fold of every (fiber, part)
template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_scan_part(ScanDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t n = d.nfib * d.parts, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int64_t f = t / d.parts, p = t - f * d.parts;
        int64_t ia, io, lo, hi;
        fiber_offsets(d, f, &ia, &io);
        part_range(d, p, &lo, &hi);
        if (hi <= lo) continue;
        T acc = load_cast<CD>(d.a, ia + lo * d.sa, d.adt);
        for (int64_t i = lo + 1; i < hi; ++i) acc = (T)BinOp<OP, CD>::apply(acc, load_cast<CD>(d.a, ia + i * d.sa, d.adt));
        reinterpret_cast<T*>(d.carry)[t] = acc;
    }
}

// pass 2: per fiber, slot p >= 1 becomes the fold of parts 0 .. p-1
template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_scan_carry(ScanDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < d.nfib; f += stride) {
        T* c = reinterpret_cast<T*>(d.carry) + f * d.parts;
        T run = c[0];
        for (int64_t p = 1; p < d.parts; ++p) {
            int64_t lo, hi;
            part_range(d, p, &lo, &hi);
            const T mine = c[p];
            c[p] = run;
            if (hi > lo) run = (T)BinOp<OP, CD>::apply(run, mine);
        }
    }
}

// pass 3: every part rescanned from its carry
template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_scan_apply(ScanDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t n = d.nfib * d.parts, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int64_t f = t / d.parts, p = t - f * d.parts;
        int64_t ia, io, lo, hi;
        fiber_offsets(d, f, &ia, &io);
        part_range(d, p, &lo, &hi);
        if (hi <= lo) continue;
        T acc;
        if (p == 0) {
            acc = load_cast<CD>(d.a, ia, d.adt);
        } else {
            acc = (T)BinOp<OP, CD>::apply(reinterpret_cast<const T*>(d.carry)[t], load_cast<CD>(d.a, ia + lo * d.sa, d.adt));
        }
        store_cast<CD>(d.o, io + lo * d.so, d.odt, acc);
        for (int64_t i = lo + 1; i < hi; ++i) {
            acc = (T)BinOp<OP, CD>::apply(acc, load_cast<CD>(d.a, ia + i * d.sa, d.adt));
            store_cast<CD>(d.o, io + i * d.so, d.odt, acc);
        }
    }
}

template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_reduceat(ScanDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t n = d.nfib * d.nseg, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int64_t k = t / d.nfib, f = t - k * d.nfib;
        int64_t ia, io;
        fiber_offsets(d, f, &ia, &io);
        const int64_t start = d.idx[k];
        const int64_t next = k + 1 < d.nseg ? d.idx[k + 1] : d.len;
        T acc = load_cast<CD>(d.a, ia + start * d.sa, d.adt);
        for (int64_t j = start + 1; j < next; ++j) acc = (T)BinOp<OP, CD>::apply(acc, load_cast<CD>(d.a, ia + j * d.sa, d.adt));
        store_cast<CD>(d.o, io + k * d.so, d.odt, acc);
    }
}

// Folds that give the same bits under any grouping (see the file comment).
template <int OP, int CD> constexpr bool scan_assoc() {
    if (OP == OP_MAXIMUM || OP == OP_MINIMUM) return true;
    if (op_is_logical(OP)) return true;
    if (OP == OP_BITWISE_AND || OP == OP_BITWISE_OR || OP == OP_BITWISE_XOR) return true;
    if (OP == OP_ADD || OP == OP_MULTIPLY) return !dt_is_float(CD);
    return false;
}
// Ops with a fold in the compute dtype: the ufunc's own loop exists for
// (CD, CD) and returns CD (comparisons fold only over bool).
template <int OP, int CD> constexpr bool scan_valid() {
    if (op_is_compare(OP)) return CD == DT_BOOL;
    if constexpr (bin_valid<OP, CD>()) return BinOp<OP, CD>::OUT_DT == CD;
    return false;
}

inline int sc_grid(int64_t items) {
    int64_t g = (items + SC_THREADS - 1) / SC_THREADS;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148LL * 8));
}

template <int OP, int CD>
cudaError_t scan_t(int mode, ScanDesc d, cudaStream_t s) {
    if constexpr (!scan_valid<OP, CD>()) {
        return cudaErrorInvalidValue;
    } else {
        if (mode == 1) {  // reduceat
            k_reduceat<OP, CD><<<sc_grid(d.nfib * d.nseg), SC_THREADS, 0, s>>>(d);
            count_launch();
            return cudaGetLastError();
        }
        if constexpr (scan_assoc<OP, CD>()) {
            if (d.parts > 1) {
                k_scan_part<OP, CD><<<sc_grid(d.nfib * d.parts), SC_THREADS, 0, s>>>(d);
                k_scan_carry<OP, CD><<<sc_grid(d.nfib), SC_THREADS, 0, s>>>(d);
                k_scan_apply<OP, CD><<<sc_grid(d.nfib * d.parts), SC_THREADS, 0, s>>>(d);
                count_launch(3);
                return cudaGetLastError();
            }
        }
        k_scan_fiber<OP, CD><<<sc_grid(d.nfib), SC_THREADS, 0, s>>>(d);
        count_launch();
        return cudaGetLastError();
    }
}

template <int OP>
cudaError_t scan_op(int mode, int cd, const ScanDesc& d, cudaStream_t s) {
#define IONP_CASE(D) case D: return scan_t<OP, D>(mode, d, s);
    switch (cd) {
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
    }
#undef IONP_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_scan(int mode, int op, int cd, const ScanDesc& d, cudaStream_t s) {
    switch (op) {
        case OP_ADD: return scan_op<OP_ADD>(mode, cd, d, s);
        case OP_SUBTRACT: return scan_op<OP_SUBTRACT>(mode, cd, d, s);
        case OP_MULTIPLY: return scan_op<OP_MULTIPLY>(mode, cd, d, s);
        case OP_DIVIDE: return scan_op<OP_DIVIDE>(mode, cd, d, s);
        case OP_MAXIMUM: return scan_op<OP_MAXIMUM>(mode, cd, d, s);
        case OP_MINIMUM: return scan_op<OP_MINIMUM>(mode, cd, d, s);
        case OP_GREATER: return scan_op<OP_GREATER>(mode, cd, d, s);
        case OP_GREATER_EQUAL: return scan_op<OP_GREATER_EQUAL>(mode, cd, d, s);
        case OP_LESS: return scan_op<OP_LESS>(mode, cd, d, s);
        case OP_LESS_EQUAL: return scan_op<OP_LESS_EQUAL>(mode, cd, d, s);
        case OP_EQUAL: return scan_op<OP_EQUAL>(mode, cd, d, s);
        case OP_NOT_EQUAL: return scan_op<OP_NOT_EQUAL>(mode, cd, d, s);
        case OP_LOGICAL_AND: return scan_op<OP_LOGICAL_AND>(mode, cd, d, s);
        case OP_LOGICAL_OR: return scan_op<OP_LOGICAL_OR>(mode, cd, d, s);
        case OP_LOGICAL_XOR: return scan_op<OP_LOGICAL_XOR>(mode, cd, d, s);
        case OP_BITWISE_AND: return scan_op<OP_BITWISE_AND>(mode, cd, d, s);
        case OP_BITWISE_OR: return scan_op<OP_BITWISE_OR>(mode, cd, d, s);
        case OP_BITWISE_XOR: return scan_op<OP_BITWISE_XOR>(mode, cd, d, s);
        case OP_FLOOR_DIVIDE: return scan_op<OP_FLOOR_DIVIDE>(mode, cd, d, s);
        case OP_LEFT_SHIFT: return scan_op<OP_LEFT_SHIFT>(mode, cd, d, s);
        case OP_RIGHT_SHIFT: return scan_op<OP_RIGHT_SHIFT>(mode, cd, d, s);
    }
    return cudaErrorInvalidValue;
}

// Shared host planning of ionp_accumulate and ionp_reduceat: `out` holds
// the fold of every fiber of `a` along `axis` (accumulate: out's shape is
// a's; reduceat: out's axis extent is the number of segments).
int32_t fiber_call(int mode, int32_t op, const IonpArr* a, int32_t axis, const int64_t* idx_host, int64_t nidx,
                   IonpArr* out, const char* what, cudaStream_t s) {
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    const int nd = a->ndim;
    if (nd == 0) return set_err(IONP_ERR_TYPE, std::string("cannot ") + what + " on a scalar");
    if (axis < 0 || axis >= nd) return set_err(IONP_ERR_AXIS, "axis " + std::to_string(axis) + " is out of bounds for array of dimension " + std::to_string(nd));
    int cd;
    if ((st = reduce_cd(op, a->dtype, &cd))) return st;
    if (out->ndim != nd) return set_err(IONP_ERR_VALUE, "out has the wrong number of dimensions");
    for (int i = 0; i < nd; ++i) {
        const int64_t want = (mode == 1 && i == axis) ? nidx : a->shape[i];
        if (out->shape[i] != want) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
    }
    if (numel(out) == 0) return IONP_OK;
    const int64_t len = a->shape[axis];
    int64_t* idx_dev = nullptr;
    if (mode == 1) {
        for (int64_t k = 0; k < nidx; ++k)
            if (idx_host[k] < 0 || idx_host[k] >= len)
                return set_err(IONP_ERR_INDEX, "index " + std::to_string(idx_host[k]) + " out-of-bounds in " +
                                                   op_name(op) + ".reduceat [0, " + std::to_string(len) + ")");
    }
    // kept dims, C order, unit dims dropped, adjacent dims merged when
    // both the input and the output strides chain
    struct KD { int64_t n, st, ost; };
    std::vector<KD> v;
    for (int i = 0; i < nd; ++i) {
        if (i == axis || a->shape[i] == 1) continue;
        KD x{a->shape[i], a->strides[i], out->strides[i]};
        if (!v.empty() && v.back().st == x.st * x.n && v.back().ost == x.ost * x.n) {
            v.back().n *= x.n; v.back().st = x.st; v.back().ost = x.ost;
            continue;
        }
        v.push_back(x);
    }
    ScanDesc d;
    memset(&d, 0, sizeof(d));
    d.adt = a->dtype;
    d.odt = out->dtype;
    d.len = len;
    d.sa = a->strides[axis];
    d.so = out->strides[axis];
    d.nseg = nidx;
    const int lead = (int)v.size() > SC_MAXD ? (int)v.size() - SC_MAXD : 0;
    d.nk = (int)v.size() - lead;
    d.nfib = 1;
    for (int i = 0; i < d.nk; ++i) {
        d.kshape[i] = v[lead + i].n; d.kst[i] = v[lead + i].st; d.kost[i] = v[lead + i].ost;
        d.nfib *= d.kshape[i];
    }
    int64_t nlead = 1;
    for (int i = 0; i < lead; ++i) nlead *= v[i].n;
    // associative folds over few long fibers: parts of >= 1024 elements,
    // enough (fiber, part) threads for every SM
    void* carry = nullptr;
    if (mode == 0 && d.nfib < 148 * 256 && len >= 4096) {
        int64_t parts = std::min<int64_t>(len / 1024, (148LL * 1024 + d.nfib - 1) / d.nfib);
        if (parts > 1) {
            d.parts = parts;
            carry = scratch_alloc((size_t)(d.nfib * parts) * 8 + 64, s);
            if (!carry) return IONP_ERR_OOM;
            d.carry = carry;
        }
    }
    if (mode == 1 && nidx > 0) {
        idx_dev = (int64_t*)scratch_alloc((size_t)nidx * 8, s);
        if (!idx_dev) { if (carry) scratch_free(carry, s); return IONP_ERR_OOM; }
        st = cuda_err(cudaMemcpyAsync(idx_dev, idx_host, (size_t)nidx * 8, cudaMemcpyHostToDevice, s), "reduceat indices");
        d.idx = idx_dev;
    }
    for (int64_t q = 0; q < nlead && !st; ++q) {
        int64_t rem = q, oa = 0, oo = 0;
        for (int i = lead - 1; i >= 0; --i) {
            const int64_t id = rem % v[i].n;
            rem /= v[i].n;
            oa += id * v[i].st;
            oo += id * v[i].ost;
        }
        d.a = elem_ptr(a) + oa * dt_bytes(a->dtype);
        d.o = (char*)elem_ptr(out) + oo * dt_bytes(out->dtype);
        st = cuda_err(launch_scan(mode, op, cd, d, s), mode == 1 ? "reduceat launch" : "accumulate launch");
    }
    if (carry) scratch_free(carry, s);
    if (idx_dev) scratch_free(idx_dev, s);
    return st;
}

}  // namespace ionp

using namespace ionp;

extern "C" int32_t ionp_accumulate(int32_t op, const IonpArr* a, int32_t axis, IonpArr* out, IonpStream stream) {
    return fiber_call(0, op, a, axis, nullptr, 0, out, "accumulate", (cudaStream_t)stream);
}

extern "C" int32_t ionp_reduceat(int32_t op, const IonpArr* a, int32_t axis, const int64_t* indices, int64_t nindices,
                                 IonpArr* out, IonpStream stream) {
    if (nindices < 0 || (nindices > 0 && !indices)) return set_err(IONP_ERR_INVALID, "bad indices");
    return fiber_call(1, op, a, axis, indices, nindices, out, "reduceat", (cudaStream_t)stream);
}
