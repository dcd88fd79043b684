// Unary op table (ufunc.rs:3824-3975 unary_op, 4237-4367 math_unary_f32/f64);
// exp/log/sin/cos are the C-library restatements of ionp_libm.cuh.
#pragma once
#include "ionp_scalar.cuh"
#include "ionp_libm.cuh"

namespace ionp {

template <int OP, int CD> struct UnOp {
    typedef typename DT<CD>::T T;
    static constexpr int OUT_DT = (OP == OP_LOGICAL_NOT) ? DT_BOOL : CD;
    typedef typename DT<OUT_DT>::T R;
    static __device__ __forceinline__ R apply(T x) {
        if constexpr (OP == OP_LOGICAL_NOT) return (R)(x == 0);
        else if constexpr (OP == OP_NEGATIVE || OP == OP_ABSOLUTE || OP == OP_INVERT) {
            constexpr bool NEG = OP == OP_NEGATIVE, ABS = OP == OP_ABSOLUTE;
            if constexpr (CD == DT_BOOL) return ABS ? x : (R)(x == 0);
            else if constexpr (dt_is_sint(CD)) return NEG ? w_sub<T>((T)0, x) : ABS ? (x < 0 ? w_sub<T>((T)0, x) : x) : (T)~x;
            else if constexpr (dt_is_uint(CD)) return NEG ? w_sub<T>((T)0, x) : ABS ? x : (T)~x;
            else if constexpr (CD == DT_F16) return NEG ? (T)(x ^ 0x8000u) : (T)(x & 0x7FFFu);
            else return NEG ? neg_bits(x) : abs_bits(x);
        } else {
            // math unary on float loop dtypes; float16 goes through f32
            if constexpr (CD == DT_F16) return f2h(f32op(h2f(x)));
            else if constexpr (CD == DT_F32) return f32op(x);
            else return f64op(x);
        }
    }
    static __device__ __forceinline__ float f32op(float x) {
        if constexpr (OP == OP_SQRT) return x_sqrt(x);
        else if constexpr (OP == OP_EXP) return lm::exp32(x);
        else if constexpr (OP == OP_LOG) return lm::log32(x);
        else if constexpr (OP == OP_SIN) return lm::sin32(x);
        else return lm::cos32(x);
    }
    static __device__ __forceinline__ double f64op(double x) {
        if constexpr (OP == OP_SQRT) return x_sqrt(x);
        else if constexpr (OP == OP_EXP) return lm::exp64(x);
        else if constexpr (OP == OP_LOG) return lm::log64(x);
        else if constexpr (OP == OP_SIN) return lm::sin64(x);
        else return lm::cos64(x);
    }
    // detect_sqrt / detect_log (fpe.rs:359-396): x < 0 -> invalid,
    // log(0) -> divide.
    static __device__ __forceinline__ uint32_t fpe(T x) {
        if constexpr (OP == OP_SQRT || OP == OP_LOG) {
            bool neg, zero;
            if constexpr (CD == DT_F16) { neg = (x & 0x8000u) && (x & 0x7FFFu) && !isnan_h(x); zero = (x & 0x7FFFu) == 0; }
            else { neg = x < (T)0; zero = x == (T)0; }
            uint32_t b = neg ? FPE_INVALID : 0u;
            if constexpr (OP == OP_LOG) b |= zero ? FPE_DIVIDE : 0u;
            return b;
        } else {
            return 0u;
        }
    }
};

template <int OP> constexpr bool un_has_fpe() { return OP == OP_SQRT || OP == OP_LOG; }

}  // namespace ionp
