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
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)sm_count() * 8));
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
    if (mode == 0 && d.nfib < sm_count() * 256 && len >= 4096) {
        int64_t parts = std::min<int64_t>(len / 1024, ((int64_t)sm_count() * 1024 + d.nfib - 1) / d.nfib);
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
    NvtxRange nvtx_("ionp_accumulate");
    return fiber_call(0, op, a, axis, nullptr, 0, out, "accumulate", (cudaStream_t)stream);
}

extern "C" int32_t ionp_reduceat(int32_t op, const IonpArr* a, int32_t axis, const int64_t* indices, int64_t nindices,
                                 IonpArr* out, IonpStream stream) {
    NvtxRange nvtx_("ionp_reduceat");
    if (nindices < 0 || (nindices > 0 && !indices)) return set_err(IONP_ERR_INVALID, "bad indices");
    return fiber_call(1, op, a, axis, indices, nindices, out, "reduceat", (cudaStream_t)stream);
}

namespace ionp {

// ---------------------------------------------------------------------------
// ufunc.at: target[idx_i, ...] = op(target[idx_i, ...], values[i, ...]) for
// i in order (at_binary, ionp-core/src/ufunc.rs:9577-9733). Repeated indices
// apply in order, so each distinct row is one chain: the host groups the
// index positions by row (first occurrence order of rows, positions
// ascending within a row) and one thread takes one (row, element) pair,
// folding the row's values in order in the compute dtype CD:
//  * logical ops: CD bool (the target element read as bool, the result
//    written back as 0/1 of the target dtype);
//  * comparisons: CD the target dtype, the bool result written back as
//    0/1 of it after every step;
//  * other ops: CD = the ufunc's result dtype for (target, values); when it
//    differs from the target's, the reference casts the whole target to CD,
//    applies the updates, and casts the whole target back, so every element
//    makes the round trip (done by the host as two casts before this
//    kernel); the updates then chain in CD and are cast back once.
// ---------------------------------------------------------------------------
struct AtDesc {
    void* t;                        // target row 0, element 0
    int32_t tdt;
    int64_t tst0;                   // target stride along axis 0
    const void* v;                  // values, broadcast to (n, row...)
    int32_t vdt;
    int64_t vst0;
    int32_t nr;                     // row dims (merged)
    int64_t rshape[SC_MAXD], rtst[SC_MAXD], rvst[SC_MAXD];
    int64_t rown;                   // elements per row
    int64_t nrows;                  // distinct rows
    const int64_t* row;             // [nrows] target row index
    const int64_t* start;           // [nrows + 1] into pos
    const int64_t* pos;             // value positions, grouped by row
};

template <int CD> __device__ __forceinline__ typename DT<CD>::T from_bool(bool b) {
    if constexpr (CD == DT_F16) return b ? (uint16_t)0x3C00 : (uint16_t)0;
    else return (typename DT<CD>::T)(b ? 1 : 0);
}

template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_at(AtDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t n = d.nrows * d.rown, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int64_t r = t / d.rown;
        int64_t e = t - r * d.rown, to = 0, vo = 0;
        for (int k = d.nr - 1; k >= 0; --k) {
            const int64_t q = e / d.rshape[k], i = e - q * d.rshape[k];
            e = q;
            to += i * d.rtst[k];
            vo += i * d.rvst[k];
        }
        const int64_t tp = d.row[r] * d.tst0 + to;
        T acc = load_cast<CD>(d.t, tp, d.tdt);
        for (int64_t k = d.start[r]; k < d.start[r + 1]; ++k) {
            const T x = load_cast<CD>(d.v, d.pos[k] * d.vst0 + vo, d.vdt);
            if constexpr (op_is_compare(OP)) acc = from_bool<CD>((bool)BinOp<OP, CD>::apply(acc, x));
            else acc = (T)BinOp<OP, CD>::apply(acc, x);
        }
        store_cast<CD>(d.t, tp, d.tdt, acc);
    }
}

template <int OP, int CD> constexpr bool at_valid() {
    if (op_is_logical(OP)) return CD == DT_BOOL;
    if (op_is_compare(OP)) return true;
    if constexpr (bin_valid<OP, CD>()) return BinOp<OP, CD>::OUT_DT == CD;
    return false;
}

template <int OP>
cudaError_t at_op(int cd, const AtDesc& d, cudaStream_t s) {
#define IONP_CASE(D)                                                                              \
    case D:                                                                                       \
        if constexpr (at_valid<OP, D>()) {                                                        \
            k_at<OP, D><<<sc_grid(d.nrows * d.rown), SC_THREADS, 0, s>>>(d);                      \
            count_launch();                                                                       \
            return cudaGetLastError();                                                            \
        }                                                                                         \
        break;
    switch (cd) {
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
    }
#undef IONP_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_at(int op, int cd, const AtDesc& d, cudaStream_t s) {
    switch (op) {
        case OP_ADD: return at_op<OP_ADD>(cd, d, s);
        case OP_SUBTRACT: return at_op<OP_SUBTRACT>(cd, d, s);
        case OP_MULTIPLY: return at_op<OP_MULTIPLY>(cd, d, s);
        case OP_DIVIDE: return at_op<OP_DIVIDE>(cd, d, s);
        case OP_MAXIMUM: return at_op<OP_MAXIMUM>(cd, d, s);
        case OP_MINIMUM: return at_op<OP_MINIMUM>(cd, d, s);
        case OP_GREATER: return at_op<OP_GREATER>(cd, d, s);
        case OP_GREATER_EQUAL: return at_op<OP_GREATER_EQUAL>(cd, d, s);
        case OP_LESS: return at_op<OP_LESS>(cd, d, s);
        case OP_LESS_EQUAL: return at_op<OP_LESS_EQUAL>(cd, d, s);
        case OP_EQUAL: return at_op<OP_EQUAL>(cd, d, s);
        case OP_NOT_EQUAL: return at_op<OP_NOT_EQUAL>(cd, d, s);
        case OP_LOGICAL_AND: return at_op<OP_LOGICAL_AND>(cd, d, s);
        case OP_LOGICAL_OR: return at_op<OP_LOGICAL_OR>(cd, d, s);
        case OP_LOGICAL_XOR: return at_op<OP_LOGICAL_XOR>(cd, d, s);
        case OP_BITWISE_AND: return at_op<OP_BITWISE_AND>(cd, d, s);
        case OP_BITWISE_OR: return at_op<OP_BITWISE_OR>(cd, d, s);
        case OP_BITWISE_XOR: return at_op<OP_BITWISE_XOR>(cd, d, s);
        case OP_FLOOR_DIVIDE: return at_op<OP_FLOOR_DIVIDE>(cd, d, s);
        case OP_LEFT_SHIFT: return at_op<OP_LEFT_SHIFT>(cd, d, s);
        case OP_RIGHT_SHIFT: return at_op<OP_RIGHT_SHIFT>(cd, d, s);
        case OP_REMAINDER: return at_op<OP_REMAINDER>(cd, d, s);
        case OP_FMOD: return at_op<OP_FMOD>(cd, d, s);
    }
    return cudaErrorInvalidValue;
}

// Unary .at (at_unary, ufunc.rs:9301; at_math_unary, ufunc.rs:9805): every
// occurrence of a row applies op once more to its elements, each time
// computed in CD and written back in the target's dtype (logical_not: CD
// bool, the target read as bool).
template <int OP, int CD>
__global__ void __launch_bounds__(SC_THREADS) k_at_unary(AtDesc d) {
    typedef UnOp<OP, CD> U;
    const int64_t n = d.nrows * d.rown, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int64_t r = t / d.rown;
        int64_t e = t - r * d.rown, to = 0;
        for (int k = d.nr - 1; k >= 0; --k) {
            const int64_t q = e / d.rshape[k], i = e - q * d.rshape[k];
            e = q;
            to += i * d.rtst[k];
        }
        const int64_t tp = d.row[r] * d.tst0 + to, c = d.start[r + 1] - d.start[r];
        for (int64_t k = 0; k < c; ++k) store_cast<U::OUT_DT>(d.t, tp, d.tdt, U::apply(load_cast<CD>(d.t, tp, d.tdt)));
    }
}

template <int OP>
cudaError_t at_un_op(int cd, const AtDesc& d, cudaStream_t s) {
    constexpr bool MATH = OP >= OP_SQRT;
#define IONP_CASE(D)                                                                              \
    case D:                                                                                       \
        if constexpr (!MATH || dt_is_float(D)) {                                                  \
            k_at_unary<OP, D><<<sc_grid(d.nrows * d.rown), SC_THREADS, 0, s>>>(d);                \
            count_launch();                                                                       \
            return cudaGetLastError();                                                            \
        }                                                                                         \
        break;
    switch (cd) {
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
    }
#undef IONP_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_at_unary(int op, int cd, const AtDesc& d, cudaStream_t s) {
    switch (op) {
        case OP_NEGATIVE: return at_un_op<OP_NEGATIVE>(cd, d, s);
        case OP_ABSOLUTE: return at_un_op<OP_ABSOLUTE>(cd, d, s);
        case OP_INVERT: return at_un_op<OP_INVERT>(cd, d, s);
        case OP_LOGICAL_NOT: return at_un_op<OP_LOGICAL_NOT>(cd, d, s);
        case OP_SQRT: return at_un_op<OP_SQRT>(cd, d, s);
        case OP_EXP: return at_un_op<OP_EXP>(cd, d, s);
        case OP_LOG: return at_un_op<OP_LOG>(cd, d, s);
        case OP_SIN: return at_un_op<OP_SIN>(cd, d, s);
        case OP_COS: return at_un_op<OP_COS>(cd, d, s);
    }
    return cudaErrorInvalidValue;
}

// [lo, hi) bytes an array's elements can touch
static void byte_span(const IonpArr* a, uintptr_t* lo, uintptr_t* hi) {
    const int64_t b = dt_bytes(a->dtype);
    int64_t mn = 0, mx = 0;
    for (int i = 0; i < a->ndim; ++i) {
        const int64_t ext = (a->shape[i] - 1) * a->strides[i];
        if (ext < 0) mn += ext; else mx += ext;
    }
    const uintptr_t base = (uintptr_t)elem_ptr(a);
    *lo = base + mn * b;
    *hi = base + (mx + 1) * b;
}

static IonpArr c_contig_like(const IonpArr* a, int dtype, void* data) {
    IonpArr r;
    memset(&r, 0, sizeof(r));
    r.dtype = dtype;
    r.ndim = a->ndim;
    int64_t acc = 1;
    for (int i = a->ndim - 1; i >= 0; --i) {
        r.shape[i] = a->shape[i];
        r.strides[i] = acc;
        acc *= a->shape[i] > 0 ? a->shape[i] : 1;
    }
    r.data = data;
    return r;
}

// One .at pass over `t` (already in its compute dtype unless comparisons /
// logical ops, which the kernel casts per element).
static int32_t at_pass(int32_t op, int cd, bool unary, const IonpArr* t, const IonpArr* v, const int64_t* vst,
                       const std::vector<int64_t>& rows, cudaStream_t s) {
    const int nd = t->ndim;
    if (rows.empty()) return IONP_OK;
    // group index positions by row: rows ascending, positions ascending
    std::vector<int64_t> order(rows.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int64_t)i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return rows[x] < rows[y]; });
    std::vector<int64_t> urow, start;
    for (size_t i = 0; i < order.size(); ++i) {
        if (i == 0 || rows[order[i]] != rows[order[i - 1]]) {
            urow.push_back(rows[order[i]]);
            start.push_back((int64_t)i);
        }
    }
    start.push_back((int64_t)order.size());
    const int64_t G = (int64_t)urow.size();
    // row dims: unit dims dropped, neighbours merged when both strides chain
    struct RD { int64_t n, ts, vs; };
    std::vector<RD> rd;
    int64_t rown = 1;
    for (int i = 1; i < nd; ++i) {
        rown *= t->shape[i];
        if (t->shape[i] == 1) continue;
        RD x{t->shape[i], t->strides[i], v ? vst[i] : 0};
        if (!rd.empty() && rd.back().ts == x.ts * x.n && rd.back().vs == x.vs * x.n) {
            rd.back().n *= x.n; rd.back().ts = x.ts; rd.back().vs = x.vs;
            continue;
        }
        rd.push_back(x);
    }
    if (rown == 0) return IONP_OK;
    std::vector<int64_t> host;
    host.reserve(urow.size() + start.size() + order.size());
    host.insert(host.end(), urow.begin(), urow.end());
    host.insert(host.end(), start.begin(), start.end());
    host.insert(host.end(), order.begin(), order.end());
    int64_t* dev = (int64_t*)scratch_alloc(host.size() * 8, s);
    if (!dev) return IONP_ERR_OOM;
    int32_t st = cuda_err(cudaMemcpyAsync(dev, host.data(), host.size() * 8, cudaMemcpyHostToDevice, s), "at indices");
    AtDesc d;
    memset(&d, 0, sizeof(d));
    d.tdt = t->dtype;
    d.tst0 = nd ? t->strides[0] : 0;
    d.vdt = v ? v->dtype : 0;
    d.vst0 = (v && nd) ? vst[0] : 0;
    d.row = dev;
    d.start = dev + G;
    d.pos = dev + 2 * G + 1;
    d.nrows = G;
    const int lead = (int)rd.size() > SC_MAXD ? (int)rd.size() - SC_MAXD : 0;
    d.nr = (int)rd.size() - lead;
    d.rown = 1;
    for (int i = 0; i < d.nr; ++i) {
        d.rshape[i] = rd[lead + i].n; d.rtst[i] = rd[lead + i].ts; d.rvst[i] = rd[lead + i].vs;
        d.rown *= d.rshape[i];
    }
    int64_t nlead = 1;
    for (int i = 0; i < lead; ++i) nlead *= rd[i].n;
    for (int64_t q = 0; q < nlead && !st; ++q) {
        int64_t rem = q, ot = 0, ov = 0;
        for (int i = lead - 1; i >= 0; --i) {
            const int64_t id = rem % rd[i].n;
            rem /= rd[i].n;
            ot += id * rd[i].ts;
            ov += id * rd[i].vs;
        }
        d.t = (char*)elem_ptr(t) + ot * dt_bytes(t->dtype);
        d.v = v ? elem_ptr(v) + ov * dt_bytes(v->dtype) : nullptr;
        st = cuda_err(unary ? launch_at_unary(op, cd, d, s) : launch_at(op, cd, d, s), "at launch");
    }
    scratch_free(dev, s);
    return st;
}

}  // namespace ionp

extern "C" int32_t ionp_at(int32_t op, IonpArr* target, const int64_t* indices, int64_t nindices,
                           const IonpArr* values, IonpStream stream) {
    NvtxRange nvtx_("ionp_at");
    int32_t st;
    if ((st = check_arr(target, "target"))) return st;
    if (values && (st = check_arr(values, "values"))) return st;
    if (nindices < 0 || (nindices > 0 && !indices)) return set_err(IONP_ERR_INVALID, "bad indices");
    cudaStream_t s = (cudaStream_t)stream;
    const bool unary = op >= OP_NEGATIVE && op <= OP_COS;
    const bool math_un = op >= OP_SQRT && op <= OP_COS;
    if (!unary && !(op >= OP_ADD && op <= OP_RIGHT_SHIFT) && op != OP_REMAINDER && op != OP_FMOD)
        return set_err(IONP_ERR_UNSUPPORTED, std::string("op ") + std::to_string(op) + " has no .at in this engine");
    if (unary && values) return set_err(IONP_ERR_INVALID, "unary ufunc .at() takes no third argument");
    if (!unary && !values) return set_err(IONP_ERR_INVALID, "binary ufunc .at() requires a values argument");
    const int tdt = target->dtype;
    int cd = 0, rd = 0;
    if (math_un && (st = unary_loop(op, tdt, &cd, &rd))) return st;   // checked before the indices
    // normalize_at_indices (ufunc.rs:9250)
    const int nd = target->ndim;
    std::vector<int64_t> rows;
    if (nd == 0) {
        if (nindices)
            return set_err(IONP_ERR_INDEX, "too many indices for array: array is 0-dimensional, but " +
                                               std::to_string(nindices) + " were indexed");
        rows.push_back(0);
    } else {
        const int64_t n = target->shape[0];
        rows.resize((size_t)nindices);
        for (int64_t i = 0; i < nindices; ++i) {
            const int64_t x = indices[i], y = x < 0 ? x + n : x;
            if (y < 0 || y >= n)
                return set_err(IONP_ERR_INDEX, "index " + std::to_string(x) + " is out of bounds for axis 0 with size " +
                                                   std::to_string(n));
            rows[i] = y;
        }
    }
    bool slow = false;
    if (unary) {
        if (op == OP_LOGICAL_NOT) cd = DT_BOOL;
        else if (!math_un) {
            if ((st = unary_loop(op, tdt, &cd, &rd))) return st;
            if (rd != tdt)
                return set_err(IONP_ERR_TYPE, std::string("'.at' would change dtype from ") + dt_name(tdt) + " to " +
                                                  dt_name(rd) + ", which is not supported");
        }
    } else if (op_is_logical(op)) {
        cd = DT_BOOL;
    } else if (op_is_compare(op)) {
        if (!dt_valid(values->dtype) || !dt_valid(tdt)) return set_err(IONP_ERR_UNSUPPORTED, "unsupported dtype");
        cd = tdt;
    } else {
        if ((st = binary_loop(op, tdt, values->dtype, &cd, &rd))) return st;
        cd = rd;
        slow = cd != tdt;
    }
    // values broadcast against (len(indices),) + row shape as a whole
    int64_t vshape[IONP_MAX_DIMS], vst[IONP_MAX_DIMS];
    int vnd = 0;
    if (!unary) {
        if (nd) {
            vshape[0] = nindices;
            for (int i = 1; i < nd; ++i) vshape[i] = target->shape[i];
            vnd = nd;
        }
        if (!bcast_strides(values, vnd, vshape, vst))
            return set_err(IONP_ERR_BROADCAST, "array is not broadcastable to correct shape");
        if (!nd) vst[0] = 0;
    }
    if (numel(target) == 0) return IONP_OK;
    if (slow) {
        // compute on a whole-target copy in the promoted dtype, then cast
        // every element back (the reference's round trip)
        void* buf = scratch_alloc((size_t)numel(target) * dt_bytes(cd), s);
        if (!buf) return IONP_ERR_OOM;
        IonpArr tmp = c_contig_like(target, cd, buf);
        st = cast_impl(target, &tmp, nullptr, s);
        if (!st) st = at_pass(op, cd, false, &tmp, values, vst, rows, s);
        if (!st) st = cast_impl(&tmp, target, nullptr, s);
        scratch_free(buf, s);
        return st;
    }
    // values that share memory with the target are read as they were
    // before the call: take a copy first
    void* vcopy = nullptr;
    IonpArr vc;
    const IonpArr* vv = values;
    if (values && numel(values) > 0) {
        uintptr_t tl, th, vl, vh;
        byte_span(target, &tl, &th);
        byte_span(values, &vl, &vh);
        if (vl < th && tl < vh) {
            vcopy = scratch_alloc((size_t)numel(values) * dt_bytes(values->dtype), s);
            if (!vcopy) return IONP_ERR_OOM;
            vc = c_contig_like(values, values->dtype, vcopy);
            if ((st = cast_impl(values, &vc, nullptr, s))) { scratch_free(vcopy, s); return st; }
            if (!bcast_strides(&vc, vnd, vshape, vst)) { scratch_free(vcopy, s); return set_err(IONP_ERR_BROADCAST, "array is not broadcastable to correct shape"); }
            if (!nd) vst[0] = 0;
            vv = &vc;
        }
    }
    st = at_pass(op, cd, unary, target, vv, vst, rows, s);
    if (vcopy) scratch_free(vcopy, s);
    return st;
}
