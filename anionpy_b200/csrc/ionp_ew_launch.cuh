// Launch helpers that instantiate the element-wise kernels for the legal
// (op, loop dtype) pairs of the reference's dtype tables.
#pragma once
#include "ionp_ew.cuh"

namespace ionp {

// Loop dtypes each binary op can be dispatched on (binary_out_dtype,
// ufunc.rs:1101, and the int_same / bool_same / float_same arms that exist).
template <int OP, int CD> constexpr bool bin_valid() {
    if (op_is_compare(OP)) return true;
    if (op_is_logical(OP)) return CD == DT_BOOL;
    if (OP == OP_ADD || OP == OP_MULTIPLY || OP == OP_MAXIMUM || OP == OP_MINIMUM) return true;
    if (OP == OP_SUBTRACT) return CD != DT_BOOL;
    if (OP == OP_DIVIDE) return dt_is_float(CD);
    if (OP == OP_BITWISE_AND || OP == OP_BITWISE_OR || OP == OP_BITWISE_XOR) return !dt_is_float(CD);
    if (OP == OP_LEFT_SHIFT || OP == OP_RIGHT_SHIFT) return dt_is_sint(CD) || dt_is_uint(CD);
    if (OP == OP_FLOOR_DIVIDE || OP == OP_REMAINDER || OP == OP_FMOD) return CD != DT_BOOL;
    return false;
}

// Whether the vector tile kernel applies: whole tiles, every array either
// row- or column-contiguous with its other stride and its base a multiple of
// 16 bytes (so each vector a tile row starts is aligned).
template <class T> inline bool trv_ok(const EwDesc& d) {
    constexpr int TL = TrV<T>::TILE, VW = TrV<T>::VW;
    if (d.shape[0] % TL || d.shape[1] % TL) return false;
    auto fits = [&](const void* p, int64_t s0, int64_t s1) {
        if (reinterpret_cast<uintptr_t>(p) % 16) return false;
        if (s1 == 1) return s0 > 0 && s0 % VW == 0;
        if (s0 == 1) return s1 > 0 && s1 % VW == 0;
        return false;
    };
    return fits(d.a.p, d.a.st[0], d.a.st[1]) && fits(d.b.p, d.b.st[0], d.b.st[1]) && fits(d.o, d.so[0], d.so[1]);
}

template <int OP, int CD>
cudaError_t launch_bin_t(const EwDesc& d, const ContigInfo& ci, uint32_t* flags, cudaStream_t s) {
    typedef typename DT<CD>::T T;
    typedef typename BinOp<OP, CD>::R R;
    constexpr bool HAS_FPE = FpeKind<OP, CD>::value != 0;
    const bool fpe = HAS_FPE && flags != nullptr;
    if (d.n == 0) return cudaSuccess;
    if (ci.ok) {
        int64_t nv = d.n / Vec16<T>::N;
        int g = ew_grid(nv > 0 ? (nv + 1) / 2 : d.n);
        const T* a = (const T*)d.a.p;
        const T* b = (const T*)d.b.p;
        R* o = (R*)d.o;
        if constexpr (OP == OP_FLOOR_DIVIDE && CD == DT_F64) {
            if (fpe) k_bin_contig3<OP, CD, true><<<g, EW_THREADS, 0, s>>>(a, b, o, d.n, ci.a_scalar, ci.b_scalar, flags);
            else k_bin_contig3<OP, CD, false><<<g, EW_THREADS, 0, s>>>(a, b, o, d.n, ci.a_scalar, ci.b_scalar, flags);
        } else {
            if (HAS_FPE && fpe) k_bin_contig<OP, CD, HAS_FPE><<<g, EW_THREADS, 0, s>>>(a, b, o, d.n, ci.a_scalar, ci.b_scalar, flags);
            else k_bin_contig<OP, CD, false><<<g, EW_THREADS, 0, s>>>(a, b, o, d.n, ci.a_scalar, ci.b_scalar, flags);
        }
        count_launch();
        return cudaGetLastError();
    }
    const bool same = d.a.dt == CD && d.b.dt == CD && d.odt == BinOp<OP, CD>::OUT_DT && d.m.p == nullptr;
    // two merged dims with operands contiguous along different dims: tiles
    // through shared memory
    if (same && d.nd == 2 && d.shape[0] >= TR_TILE && d.shape[1] >= TR_TILE) {
        auto colc = [](int64_t s0, int64_t s1) { return s0 == 1 && s1 != 1; };
        const bool ca = colc(d.a.st[0], d.a.st[1]), cb = colc(d.b.st[0], d.b.st[1]), co = colc(d.so[0], d.so[1]);
        if (ca != co || cb != co) {
            if constexpr ((sizeof(T) == 4 || sizeof(T) == 8) && sizeof(R) == sizeof(T)) {
                if (trv_ok<T>(d)) {
                    constexpr int TL = TrV<T>::TILE;
                    const int64_t tiles = (d.shape[0] / TL) * (d.shape[1] / TL);
                    // one operand across the output: 4-byte types, and the
                    // division family of 8-byte types (arithmetic-heavy,
                    // where overlapping the next tile's loads pays)
                    constexpr bool DIVF = OP == OP_FLOOR_DIVIDE || OP == OP_REMAINDER || OP == OP_FMOD || OP == OP_DIVIDE;
                    if constexpr (sizeof(T) == 4 || DIVF) {
                        if ((ca != co) != (cb != co)) {
                            const int g = (int)(tiles < sm_count() * 8 ? tiles : sm_count() * 8);
                            if constexpr (HAS_FPE) {
                                if (fpe) { k_bin_trv1<OP, CD, true><<<g, EW_THREADS, 0, s>>>(d, flags); count_launch(); return cudaGetLastError(); }
                            }
                            k_bin_trv1<OP, CD, false><<<g, EW_THREADS, 0, s>>>(d, flags);
                            count_launch();
                            return cudaGetLastError();
                        }
                    }
                    const int g = (int)(tiles < sm_count() * 6 ? tiles : sm_count() * 6);
                    if constexpr (HAS_FPE) {
                        if (fpe) { k_bin_trv<OP, CD, true><<<g, EW_THREADS, 0, s>>>(d, flags); count_launch(); return cudaGetLastError(); }
                    }
                    k_bin_trv<OP, CD, false><<<g, EW_THREADS, 0, s>>>(d, flags);
                    count_launch();
                    return cudaGetLastError();
                }
            }
            const int64_t tiles = ((d.shape[0] + TR_TILE - 1) / TR_TILE) * ((d.shape[1] + TR_TILE - 1) / TR_TILE);
            const int g = (int)(tiles < sm_count() * 8 ? tiles : sm_count() * 8);
            if constexpr (HAS_FPE) {
                if (fpe) { k_bin_tr<OP, CD, true><<<g, EW_THREADS, 0, s>>>(d, flags); count_launch(); return cudaGetLastError(); }
            }
            k_bin_tr<OP, CD, false><<<g, EW_THREADS, 0, s>>>(d, flags);
            count_launch();
            return cudaGetLastError();
        }
    }
    if (same && d.nd == 1) {
        constexpr int U = sizeof(T) >= 8 ? 4 : 8;
        const int g = ew_grid((d.n + U - 1) / U);
        if constexpr (HAS_FPE) {
            if (fpe) { k_bin_run<OP, CD, true><<<g, EW_THREADS, 0, s>>>(d, flags); count_launch(); return cudaGetLastError(); }
        }
        k_bin_run<OP, CD, false><<<g, EW_THREADS, 0, s>>>(d, flags);
        count_launch();
        return cudaGetLastError();
    }
    int64_t inner = d.shape[d.nd - 1];
    int g = ew_grid(inner >= 64 ? (d.n + 3) / 4 : d.n);
    if constexpr (HAS_FPE) {
        if (fpe) {
            if (same) k_bin_nd<OP, CD, true, true><<<g, EW_THREADS, 0, s>>>(d, flags);
            else k_bin_nd<OP, CD, true, false><<<g, EW_THREADS, 0, s>>>(d, flags);
            count_launch();
            return cudaGetLastError();
        }
    }
    if (same) k_bin_nd<OP, CD, false, true><<<g, EW_THREADS, 0, s>>>(d, flags);
    else k_bin_nd<OP, CD, false, false><<<g, EW_THREADS, 0, s>>>(d, flags);
    count_launch();
    return cudaGetLastError();
}

template <int OP>
cudaError_t launch_bin_op(int cd, const EwDesc& d, const ContigInfo& ci, uint32_t* flags, cudaStream_t s) {
#define IONP_CASE(D)                                                             \
    case D:                                                                      \
        if constexpr (bin_valid<OP, D>()) return launch_bin_t<OP, D>(d, ci, flags, s); \
        break;
    switch (cd) {
        IONP_CASE(DT_BOOL) IONP_CASE(DT_I8) IONP_CASE(DT_I16) IONP_CASE(DT_I32) IONP_CASE(DT_I64)
        IONP_CASE(DT_U8) IONP_CASE(DT_U16) IONP_CASE(DT_U32) IONP_CASE(DT_U64)
        IONP_CASE(DT_F16) IONP_CASE(DT_F32) IONP_CASE(DT_F64)
    }
#undef IONP_CASE
    return cudaErrorInvalidValue;
}

}  // namespace ionp
