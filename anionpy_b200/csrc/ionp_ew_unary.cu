// Unary element-wise kernels, the dtype-cast kernel, the FPE detector for
// non-trailing broadcasts, and the binary dispatcher over op groups.
#include "ionp_ew_launch.cuh"

namespace ionp {

cudaError_t launch_binary_arith(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s);
cudaError_t launch_binary_cmp(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s);
cudaError_t launch_binary_minmax(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s);
cudaError_t launch_binary_intops(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s);

cudaError_t launch_binary(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_ADD: case OP_SUBTRACT: case OP_MULTIPLY: case OP_DIVIDE:
            return launch_binary_arith(op, cd, d, ci, f, s);
        case OP_GREATER: case OP_GREATER_EQUAL: case OP_LESS: case OP_LESS_EQUAL: case OP_EQUAL: case OP_NOT_EQUAL:
            return launch_binary_cmp(op, cd, d, ci, f, s);
        case OP_MAXIMUM: case OP_MINIMUM: case OP_LOGICAL_AND: case OP_LOGICAL_OR: case OP_LOGICAL_XOR:
            return launch_binary_minmax(op, cd, d, ci, f, s);
        default:
            return launch_binary_intops(op, cd, d, ci, f, s);
    }
}

// ---------------------------------------------------------------------------
// unary
// ---------------------------------------------------------------------------
template <int OP, int CD> constexpr bool un_valid() {
    if (OP == OP_LOGICAL_NOT) return CD == DT_BOOL;
    if (OP == OP_NEGATIVE) return CD != DT_BOOL;
    if (OP == OP_ABSOLUTE) return true;
    if (OP == OP_INVERT) return !dt_is_float(CD);
    return dt_is_float(CD);  // sqrt / exp / log / sin / cos
}

template <int OP, int CD>
cudaError_t launch_un_t(const EwDesc& d, const ContigInfo& ci, uint32_t* flags, cudaStream_t s) {
    typedef typename DT<CD>::T T;
    typedef typename UnOp<OP, CD>::R R;
    constexpr bool HAS_FPE = un_has_fpe<OP>();
    const bool fpe = HAS_FPE && flags != nullptr;
    if (d.n == 0) return cudaSuccess;
    if (ci.ok) {
        int64_t nv = d.n / Vec16<T>::N;
        int g = ew_grid(nv > 0 ? (nv + 1) / 2 : d.n);
        if constexpr (HAS_FPE) {
            if (fpe) { k_un_contig<OP, CD, true><<<g, EW_THREADS, 0, s>>>((const T*)d.a.p, (R*)d.o, d.n, flags); count_launch(); return cudaGetLastError(); }
        }
        k_un_contig<OP, CD, false><<<g, EW_THREADS, 0, s>>>((const T*)d.a.p, (R*)d.o, d.n, flags);
        count_launch();
        return cudaGetLastError();
    }
    int64_t inner = d.shape[d.nd - 1];
    int g = ew_grid(inner >= 64 ? (d.n + 3) / 4 : d.n);
    if constexpr (HAS_FPE) {
        if (fpe) { k_un_nd<OP, CD, true><<<g, EW_THREADS, 0, s>>>(d, flags); count_launch(); return cudaGetLastError(); }
    }
    k_un_nd<OP, CD, false><<<g, EW_THREADS, 0, s>>>(d, flags);
    count_launch();
    return cudaGetLastError();
}

template <int OP>
cudaError_t launch_un_op(int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* flags, cudaStream_t s) {
#define IONP_CASE(D)                                                            \
    case D:                                                                     \
        if constexpr (un_valid<OP, D>()) return launch_un_t<OP, D>(d, ci, flags, s); \
        break;
    switch (cd) {
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
    }
#undef IONP_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_unary(int op, int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* f, cudaStream_t s) {
    switch (op) {
        case OP_NEGATIVE: return launch_un_op<OP_NEGATIVE>(cd, d, ci, f, s);
        case OP_ABSOLUTE: return launch_un_op<OP_ABSOLUTE>(cd, d, ci, f, s);
        case OP_INVERT: return launch_un_op<OP_INVERT>(cd, d, ci, f, s);
        case OP_LOGICAL_NOT: return launch_un_op<OP_LOGICAL_NOT>(cd, d, ci, f, s);
        case OP_SQRT: return launch_un_op<OP_SQRT>(cd, d, ci, f, s);
        case OP_EXP: return launch_un_op<OP_EXP>(cd, d, ci, f, s);
        case OP_LOG: return launch_un_op<OP_LOG>(cd, d, ci, f, s);
        case OP_SIN: return launch_un_op<OP_SIN>(cd, d, ci, f, s);
        case OP_COS: return launch_un_op<OP_COS>(cd, d, ci, f, s);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// cast / copy: out = a.cast_to(out.dtype), any strides on both sides
// ---------------------------------------------------------------------------
template <int DD>
__global__ void __launch_bounds__(EW_THREADS) k_cast(EwDesc d) {
    const int nd = d.nd;
    const int64_t inner = d.shape[nd - 1];
    const int64_t sa = d.a.st[nd - 1], so = d.so[nd - 1];
    typedef typename DT<DD>::T D;
    if (inner >= 64) {
        constexpr int ILP = 4;
        const int64_t tile = (int64_t)blockDim.x * ILP;
        const int64_t tpr = (inner + tile - 1) / tile;
        const int64_t ntiles = (d.n / inner) * tpr;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            int64_t row = t / tpr, cb = t - row * tpr;
            Offs base = unravel(d, row, 1);
            int64_t c0 = cb * tile + threadIdx.x;
#pragma unroll
            for (int u = 0; u < ILP; ++u) {
                int64_t c = c0 + u * blockDim.x;
                if (c < inner && (!d.m.p || ((const uint8_t*)d.m.p)[base.m + c * d.m.st[nd - 1]]))
                    ((D*)d.o)[base.o + c * so] = load_cast<DD>(d.a.p, base.a + c * sa, d.a.dt);
            }
        }
    } else {
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
            Offs f = unravel(d, i, 0);
            if (!d.m.p || ((const uint8_t*)d.m.p)[f.m]) ((D*)d.o)[f.o] = load_cast<DD>(d.a.p, f.a, d.a.dt);
        }
    }
}

// detect_cast_overflow (ionp-core/src/fpe.rs:398-424): a float source
// element that is not finite or lies outside [lo, hi] (the destination
// integer type's range as float64) sets FPE_INVALID. Every element is
// widened to float64 first, as the reference's to_f64_lossy does.
template <int SD>
__global__ void __launch_bounds__(EW_THREADS) k_cast_check(EwDesc d, double lo, double hi, uint32_t* flags) {
    typedef typename DT<SD>::T S;
    bool bad = false;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
        const Offs f = unravel(d, i, 0);
        const S v = ((const S*)d.a.p)[f.a];
        double x;
        if constexpr (SD == DT_F16) x = (double)h2f(v);
        else x = (double)v;
        if (!(x >= lo && x <= hi)) bad = true;
    }
    flush_flags(bad ? FPE_INVALID : 0u, flags);
}

cudaError_t launch_cast_check(const EwDesc& d, double lo, double hi, uint32_t* flags, cudaStream_t s) {
    if (d.n == 0) return cudaSuccess;
    const int g = ew_grid(d.n);
    switch (d.a.dt) {
        case DT_F16: k_cast_check<DT_F16><<<g, EW_THREADS, 0, s>>>(d, lo, hi, flags); break;
        case DT_F32: k_cast_check<DT_F32><<<g, EW_THREADS, 0, s>>>(d, lo, hi, flags); break;
        case DT_F64: k_cast_check<DT_F64><<<g, EW_THREADS, 0, s>>>(d, lo, hi, flags); break;
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cast(const EwDesc& d, cudaStream_t s) {
    // (k_cast<DD> is instantiated for all 12 output dtypes by design)
    if (d.n == 0) return cudaSuccess;
    int64_t inner = d.shape[d.nd - 1];
    int g = ew_grid(inner >= 64 ? (d.n + 3) / 4 : d.n);
    switch (d.odt) {
#define IONP_CASE(D) case D: k_cast<D><<<g, EW_THREADS, 0, s>>>(d); break;
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
#undef IONP_CASE
        default: return cudaErrorInvalidValue;
    }
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FPE detector with the reference's flat pairing x[i % len_x] over the
// C-order ravel of each operand (fpe.rs:173-300). Values are compared as
// f64, exactly as to_f64_lossy does.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ld_as_f64(const void* p, int dt, int64_t e) {
    switch (dt) {
        case DT_BOOL: return ((const uint8_t*)p)[e] ? 1.0 : 0.0;
        case DT_I8: return (double)((const int8_t*)p)[e];
        case DT_I16: return (double)((const int16_t*)p)[e];
        case DT_I32: return (double)((const int32_t*)p)[e];
        case DT_I64: return (double)((const int64_t*)p)[e];
        case DT_U8: return (double)((const uint8_t*)p)[e];
        case DT_U16: return (double)((const uint16_t*)p)[e];
        case DT_U32: return (double)((const uint32_t*)p)[e];
        case DT_U64: return (double)((const uint64_t*)p)[e];
        case DT_F16: return (double)h2f(((const h16*)p)[e]);
        case DT_F32: return (double)((const float*)p)[e];
        default: return ((const double*)p)[e];
    }
}
__device__ __forceinline__ int64_t c_offset(int64_t flat, int nd, const int64_t* sh, const int64_t* st) {
    int64_t off = 0;
    for (int k = nd - 1; k >= 0; --k) {
        int64_t q = flat / sh[k];
        off += (flat - q * sh[k]) * st[k];
        flat = q;
    }
    return off;
}
__device__ __forceinline__ bool tiny_or_inf(const void* p, int dt, int64_t e, bool* inf) {
    if (dt == DT_F16) { h16 h = ((const h16*)p)[e]; *inf = (h & 0x7FFFu) == 0x7C00u; return (h & 0x7C00u) == 0; }
    if (dt == DT_F32) { uint32_t u = fb(((const float*)p)[e]); *inf = (u & 0x7FFFFFFFu) == 0x7F800000u; return (u & 0x7F800000u) == 0; }
    if (dt == DT_F64) { uint64_t u = db(((const double*)p)[e]); *inf = (u & 0x7FFFFFFFFFFFFFFFull) == 0x7FF0000000000000ull; return (u & 0x7FF0000000000000ull) == 0; }
    *inf = false;
    return false;
}

__global__ void __launch_bounds__(EW_THREADS) k_fpe_quirk(FpeQuirkDesc d, uint32_t* flags) {
    uint32_t bits = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
        int64_t ia = d.la == 1 ? 0 : i % d.la, ib = d.lb == 1 ? 0 : i % d.lb;
        double x = ld_as_f64(d.a, d.da, c_offset(ia, d.nda, d.sha, d.sta));
        double y = ld_as_f64(d.b, d.dbt, c_offset(ib, d.ndb, d.shb, d.stb));
        if (d.kind == 1) {
            if (y == 0.0) bits |= FPE_DIVIDE | ((x == 0.0 && d.out_is_float) ? FPE_INVALID : 0u);
        } else if (d.kind == 2) {
            if (y == 0.0) bits |= FPE_DIVIDE;
        } else {
            bool fin = !isnan_d(x) && !isinf(x) && !isnan_d(y) && !isinf(y) && x != 0.0 && y != 0.0;
            if (fin) {
                int64_t io = d.lo == 1 ? 0 : i % d.lo;
                bool inf;
                bool tiny = tiny_or_inf(d.o, d.dout, c_offset(io, d.ndo, d.sho, d.sto), &inf);
                if (inf) bits |= FPE_OVER;
                else if (tiny) bits |= FPE_UNDER;
            }
        }
    }
    flush_flags(bits, flags);
}

cudaError_t launch_fpe_quirk(const FpeQuirkDesc& d, uint32_t* flags, cudaStream_t s) {
    if (d.n == 0) return cudaSuccess;
    k_fpe_quirk<<<ew_grid(d.n), EW_THREADS, 0, s>>>(d, flags);
    count_launch();
    return cudaGetLastError();
}

}  // namespace ionp
