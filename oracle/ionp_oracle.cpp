// TEST INFRASTRUCTURE ONLY -- the parity oracle. Nothing in the product path
// (anionpy_b200/, include/) may link, import or call this file; only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg use it, and only as
// the checker.
//
// A plain C++ restatement, on the host, of anionpy's CPU ufunc engine
// (Son0fSun/anionpy, ionp-core/src/ufunc.rs and friends), loop for loop:
// the same dtype promotion, the same per-kind scalar op tables, the same
// broadcast walk, the same reduction fold orders (numpy's pairwise sum on the
// "wide" run, sequential folds on "narrow" axes, f16 widening rules, masked
// runs), the same argmin/argmax scan and the same post-hoc FPE detectors.
// Each function cites the reference file:line it follows.
//
// Floating point NaN results follow x86-64 SSE semantics, which is what the
// reference's compiled Rust does on the x86 hosts this runs on: an operation
// with a NaN operand returns the first NaN operand, quieted; an invalid
// operation on non-NaN operands returns the "real indefinite" default NaN
// (sign bit set). These are applied explicitly below so the oracle does not
// depend on how gcc orders commutative operands.
//
// Transcendentals (exp/log/sin) call glibc's libm directly, which is what
// Rust's f32::exp/ln/sin and f64::exp/ln/sin lower to on Linux
// (ionp-core/src/ufunc.rs:4237-4367).
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off, no fast-math).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <functional>

extern "C" {

// Array descriptor: element strides and offset (the reference's convention,
// ionp-core/src/shape.rs:1-5), data = base of the allocation.
typedef struct {
    int32_t dtype;
    int32_t ndim;
    int64_t shape[32];
    int64_t strides[32];
    int64_t offset;
    void* data;
} OrArr;

}

namespace {

// ---------------------------------------------------------------------------
// dtype codes, in the order of ionp-core/src/dtype.rs:14 (complex excluded)
// ---------------------------------------------------------------------------
enum { D_BOOL = 0, D_I8, D_I16, D_I32, D_I64, D_U8, D_U16, D_U32, D_U64, D_F16, D_F32, D_F64, D_NUM };

enum Kind { K_BOOL, K_INT, K_UINT, K_FLOAT };

static Kind kind_of(int d) {
    if (d == D_BOOL) return K_BOOL;
    if (d >= D_I8 && d <= D_I64) return K_INT;
    if (d >= D_U8 && d <= D_U64) return K_UINT;
    return K_FLOAT;
}
static int bits_of(int d) {
    switch (d) {
        case D_BOOL: return 8;
        case D_I8: case D_U8: return 8;
        case D_I16: case D_U16: case D_F16: return 16;
        case D_I32: case D_U32: case D_F32: return 32;
        default: return 64;
    }
}
static int int_of(int b) { return b == 8 ? D_I8 : b == 16 ? D_I16 : b == 32 ? D_I32 : D_I64; }
static int uint_of(int b) { return b == 8 ? D_U8 : b == 16 ? D_U16 : b == 32 ? D_U32 : D_U64; }
static int float_of(int b) { return b <= 16 ? D_F16 : b == 32 ? D_F32 : D_F64; }
static int itemsize(int d) { return d == D_BOOL ? 1 : bits_of(d) / 8; }

// int_uint_table (dtype.rs:260-293): (signed bits, unsigned bits) -> dtype
static int int_uint_table(int ib, int ub) {
    if (ub < ib) return int_of(ib);
    if (ub == 64) return D_F64;
    return int_of(ub * 2);
}
// int_equiv_float_bits: the float width that holds an integer of this width
static int int_equiv_float_bits(int b) { return b == 8 ? 16 : b == 16 ? 32 : 64; }

// promote_dtype (dtype.rs:297-367), numeric kinds only.
static int promote(int a, int b) {
    if (a == b) return a;
    Kind ka = kind_of(a), kb = kind_of(b);
    if (ka == K_BOOL) return b;
    if (kb == K_BOOL) return a;
    if (ka == K_INT && kb == K_INT) return int_of(std::max(bits_of(a), bits_of(b)));
    if (ka == K_UINT && kb == K_UINT) return uint_of(std::max(bits_of(a), bits_of(b)));
    if (ka == K_INT && kb == K_UINT) return int_uint_table(bits_of(a), bits_of(b));
    if (ka == K_UINT && kb == K_INT) return int_uint_table(bits_of(b), bits_of(a));
    if (ka == K_FLOAT && kb == K_FLOAT) return float_of(std::max(bits_of(a), bits_of(b)));
    if (kb == K_FLOAT) return float_of(std::max(int_equiv_float_bits(bits_of(a)), bits_of(b)));
    return float_of(std::max(bits_of(a), int_equiv_float_bits(bits_of(b))));
}

// ---------------------------------------------------------------------------
// op codes (shared numbering with the product's C ABI)
// ---------------------------------------------------------------------------
enum {
    OP_ADD = 0, OP_SUBTRACT, OP_MULTIPLY, OP_DIVIDE, OP_MAXIMUM, OP_MINIMUM,
    OP_GREATER, OP_GREATER_EQUAL, OP_LESS, OP_LESS_EQUAL, OP_EQUAL, OP_NOT_EQUAL,
    OP_LOGICAL_AND, OP_LOGICAL_OR, OP_LOGICAL_XOR,
    OP_BITWISE_AND, OP_BITWISE_OR, OP_BITWISE_XOR,
    OP_FLOOR_DIVIDE, OP_LEFT_SHIFT, OP_RIGHT_SHIFT,
    OP_REMAINDER = 32, OP_FMOD = 33,
    OP_NEGATIVE = 64, OP_ABSOLUTE = 65, OP_INVERT = 66, OP_LOGICAL_NOT = 67,
    OP_SQRT = 80, OP_EXP = 81, OP_LOG = 82, OP_SIN = 83, OP_COS = 84,
};

// status codes
enum { ST_OK = 0, ST_BROADCAST = 1, ST_TYPE = 2, ST_VALUE = 3, ST_NO_LOOP = 4, ST_AXIS = 5, ST_UNSUPPORTED = 9 };

static bool is_compare(int op) { return op >= OP_GREATER && op <= OP_NOT_EQUAL; }
static bool is_logical(int op) { return op >= OP_LOGICAL_AND && op <= OP_LOGICAL_XOR; }
static bool is_bitwise(int op) { return op >= OP_BITWISE_AND && op <= OP_BITWISE_XOR; }
static bool is_shift(int op) { return op == OP_LEFT_SHIFT || op == OP_RIGHT_SHIFT; }

// binary_out_dtype (ufunc.rs:1101-1224), numeric dtypes.
static int binary_out_dtype(int op, int a, int b, int* out) {
    if (is_compare(op) || is_logical(op)) { *out = D_BOOL; return ST_OK; }
    int p = promote(a, b);
    Kind k = kind_of(p);
    if (is_bitwise(op)) {
        if (k == K_INT || k == K_UINT || k == K_BOOL) { *out = p; return ST_OK; }
        return ST_TYPE;
    }
    if (is_shift(op)) {
        if (p == D_BOOL) { *out = D_I8; return ST_OK; }
        if (k == K_INT || k == K_UINT) { *out = p; return ST_OK; }
        return ST_TYPE;
    }
    if (op == OP_SUBTRACT && p == D_BOOL) return ST_TYPE;
    if (op == OP_DIVIDE) { *out = (k == K_FLOAT) ? p : D_F64; return ST_OK; }
    if (op == OP_FLOOR_DIVIDE) { *out = (p == D_BOOL) ? D_I8 : p; return ST_OK; }
    *out = p;
    return ST_OK;
}

// math_binary_out_dtype (ufunc.rs:1785-1960) for the non-float-promoting
// members used here (remainder, fmod).
static int math_binary_out_dtype(int, int a, int b, int* out) {
    int p = promote(a, b);
    *out = (p == D_BOOL) ? D_I8 : p;
    return ST_OK;
}

// unary_out_dtype (ufunc.rs:1608-1650) and math_unary_out_dtype (1682-1783).
static int unary_out_dtype(int op, int a, int* out) {
    switch (op) {
        case OP_LOGICAL_NOT: *out = D_BOOL; return ST_OK;
        case OP_NEGATIVE: if (a == D_BOOL) return ST_TYPE; *out = a; return ST_OK;
        case OP_INVERT: if (kind_of(a) == K_FLOAT) return ST_TYPE; *out = a; return ST_OK;
        case OP_ABSOLUTE: *out = a; return ST_OK;
        case OP_SQRT: case OP_EXP: case OP_LOG: case OP_SIN: case OP_COS:
            if (a == D_BOOL || a == D_I8 || a == D_U8) *out = D_F16;
            else if (a == D_I16 || a == D_U16) *out = D_F32;
            else if (kind_of(a) != K_FLOAT) *out = D_F64;
            else *out = a;
            return ST_OK;
    }
    return ST_UNSUPPORTED;
}

// ---------------------------------------------------------------------------
// float16 <-> float32/64 and x86 NaN rules
// ---------------------------------------------------------------------------
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint64_t dbits(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
static inline double bitsd(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }

static const uint32_t F32_DEFAULT_NAN = 0xFFC00000u;            // x86 "real indefinite"
static const uint64_t F64_DEFAULT_NAN = 0xFFF8000000000000ull;

static inline float quietf(float x) { return bitsf(fbits(x) | 0x00400000u); }
static inline double quietd(double x) { return bitsd(dbits(x) | 0x0008000000000000ull); }

// half::f16::to_f32 (IEEE conversion, exact; NaN quieted, payload kept).
static float h2f(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1F, m = h & 0x3FF;
    if (e == 0x1F) return bitsf(m == 0 ? (sign | 0x7F800000u) : (sign | 0x7FC00000u | (m << 13)));
    if (e == 0) {
        if (m == 0) return bitsf(sign);
        float v = (float)m * 5.9604644775390625e-8f;  // m * 2^-24, exact
        return sign ? -v : v;
    }
    return bitsf(sign | ((e + 112u) << 23) | (m << 13));
}
static double h2d(uint16_t h) { return (double)h2f(h); }

// half::f16::from_f64: round-to-nearest-even from double; NaN keeps the top
// payload bits and is quieted.
static uint16_t d2h(double d) {
    uint64_t b = dbits(d);
    uint16_t sign = (uint16_t)((b >> 48) & 0x8000u);
    uint64_t ex = (b >> 52) & 0x7FF, man = b & ((1ull << 52) - 1);
    if (ex == 0x7FF) {
        if (man == 0) return sign | 0x7C00;
        return (uint16_t)(sign | 0x7E00 | (uint16_t)((man >> 42) & 0x3FF));
    }
    if (ex == 0) return sign;  // double subnormals are far below half's range
    int e = (int)ex - 1023;
    if (e > 15) return sign | 0x7C00;
    uint64_t m = man | (1ull << 52);
    if (e >= -14) {
        uint64_t q = m >> 42, rem = m & ((1ull << 42) - 1), half = 1ull << 41;
        if (rem > half || (rem == half && (q & 1))) q++;
        uint32_t he = (uint32_t)(e + 15);
        if (q == 2048) { q = 1024; he++; }
        if (he >= 31) return sign | 0x7C00;
        return (uint16_t)(sign | (he << 10) | (q & 0x3FF));
    }
    int shift = 28 - e;  // value / 2^-24 = m * 2^(e - 52 + 24)
    if (shift > 60) return sign;
    uint64_t q = m >> shift, rem = m & ((1ull << shift) - 1), half = 1ull << (shift - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    return (uint16_t)(sign | q);
}
static uint16_t f2h(float f) { return d2h((double)f); }

// x86 f64 -> f32 (cvtsd2ss): RNE; NaN keeps the top payload bits, quieted.
static float d2f(double d) {
    if (std::isnan(d)) {
        uint64_t b = dbits(d);
        uint32_t s = (uint32_t)(b >> 32) & 0x80000000u;
        return bitsf(s | 0x7FC00000u | (uint32_t)((b >> 29) & 0x7FFFFFu));
    }
    return (float)d;
}
// x86 f32 -> f64 (cvtss2sd): exact; NaN quieted with payload kept.
static double f2d(float f) {
    if (std::isnan(f)) {
        uint64_t s = (uint64_t)(fbits(f) & 0x80000000u) << 32;
        return bitsd(s | 0x7FF8000000000000ull | ((uint64_t)(fbits(f) & 0x7FFFFFu) << 29));
    }
    return (double)f;
}

// Binary float primitives with the x86 NaN rule made explicit.
template <class F> struct FT;
template <> struct FT<float> {
    static float dnan() { return bitsf(F32_DEFAULT_NAN); }
    static float quiet(float x) { return quietf(x); }
};
template <> struct FT<double> {
    static double dnan() { return bitsd(F64_DEFAULT_NAN); }
    static double quiet(double x) { return quietd(x); }
};
template <class F> static inline F nan2(F x, F y) {
    if (x != x) return FT<F>::quiet(x);
    if (y != y) return FT<F>::quiet(y);
    return FT<F>::dnan();
}
template <class F> static inline F fadd(F x, F y) { F r = x + y; return r == r ? r : nan2(x, y); }
template <class F> static inline F fsub(F x, F y) { F r = x - y; return r == r ? r : nan2(x, y); }
template <class F> static inline F fmul(F x, F y) { F r = x * y; return r == r ? r : nan2(x, y); }
template <class F> static inline F fdiv(F x, F y) { F r = x / y; return r == r ? r : nan2(x, y); }
static inline float o_fmod(float x, float y) { return fmodf(x, y); }   // glibc, as Rust `%` calls
static inline double o_fmod(double x, double y) { return fmod(x, y); }
static inline float o_floor(float x) { return x != x ? quietf(x) : floorf(x); }
static inline double o_floor(double x) { return x != x ? quietd(x) : floor(x); }
static inline float o_sqrt(float x) { return x != x ? quietf(x) : (x < 0 ? bitsf(F32_DEFAULT_NAN) : sqrtf(x)); }
static inline double o_sqrt(double x) { return x != x ? quietd(x) : (x < 0 ? bitsd(F64_DEFAULT_NAN) : sqrt(x)); }

// ---------------------------------------------------------------------------
// Float "kinds" for the generic float algorithms: f32, f64 and half::f16,
// whose arithmetic is to_f32 -> f32 op -> from_f32 (half crate).
// ---------------------------------------------------------------------------
struct H16 { uint16_t b; };

struct OpsF32 {
    typedef float T;
    static T add(T x, T y) { return fadd(x, y); }
    static T sub(T x, T y) { return fsub(x, y); }
    static T mul(T x, T y) { return fmul(x, y); }
    static T div(T x, T y) { return fdiv(x, y); }
    static T rem(T x, T y) { return o_fmod(x, y); }
    static T floor_(T x) { return o_floor(x); }
    static bool isnan_(T x) { return x != x; }
    static bool isinf_(T x) { return std::isinf(x); }
    static bool isfin(T x) { return std::isfinite(x); }
    static bool iszero(T x) { return x == 0; }
    static bool neg(T x) { return std::signbit(x); }
    static bool eq(T x, T y) { return x == y; }
    static bool gt(T x, T y) { return x > y; }
    static bool lt(T x, T y) { return x < y; }
    static T one() { return 1.0f; }
    static T half() { return 0.5f; }
    static T nan() { return bitsf(0x7FC00000u); }      // f32::NAN
    static T negone() { return -1.0f; }
    static T copysign0(T s) { return std::signbit(s) ? -0.0f : 0.0f; }
};
struct OpsF64 {
    typedef double T;
    static T add(T x, T y) { return fadd(x, y); }
    static T sub(T x, T y) { return fsub(x, y); }
    static T mul(T x, T y) { return fmul(x, y); }
    static T div(T x, T y) { return fdiv(x, y); }
    static T rem(T x, T y) { return o_fmod(x, y); }
    static T floor_(T x) { return o_floor(x); }
    static bool isnan_(T x) { return x != x; }
    static bool isinf_(T x) { return std::isinf(x); }
    static bool isfin(T x) { return std::isfinite(x); }
    static bool iszero(T x) { return x == 0; }
    static bool neg(T x) { return std::signbit(x); }
    static bool eq(T x, T y) { return x == y; }
    static bool gt(T x, T y) { return x > y; }
    static bool lt(T x, T y) { return x < y; }
    static T one() { return 1.0; }
    static T half() { return 0.5; }
    static T nan() { return bitsd(0x7FF8000000000000ull); }  // f64::NAN
    static T negone() { return -1.0; }
    static T copysign0(T s) { return std::signbit(s) ? -0.0 : 0.0; }
};
struct OpsF16 {
    typedef uint16_t T;
    static T add(T x, T y) { return f2h(fadd(h2f(x), h2f(y))); }
    static T sub(T x, T y) { return f2h(fsub(h2f(x), h2f(y))); }
    static T mul(T x, T y) { return f2h(fmul(h2f(x), h2f(y))); }
    static T div(T x, T y) { return f2h(fdiv(h2f(x), h2f(y))); }
    static T rem(T x, T y) { return f2h(o_fmod(h2f(x), h2f(y))); }
    static T floor_(T x) { return f2h(o_floor(h2f(x))); }
    static bool isnan_(T x) { return (x & 0x7C00) == 0x7C00 && (x & 0x3FF); }
    static bool isinf_(T x) { return (x & 0x7FFF) == 0x7C00; }
    static bool isfin(T x) { return (x & 0x7C00) != 0x7C00; }
    static bool iszero(T x) { return (x & 0x7FFF) == 0; }
    static bool neg(T x) { return (x & 0x8000) != 0; }
    static bool eq(T x, T y) { return h2f(x) == h2f(y); }
    static bool gt(T x, T y) { return h2f(x) > h2f(y); }
    static bool lt(T x, T y) { return h2f(x) < h2f(y); }
    static T one() { return 0x3C00; }
    static T half() { return 0x3800; }
    static T nan() { return 0x7E00; }                        // half::f16::NAN
    static T negone() { return 0xBC00; }
    static T copysign0(T s) { return (uint16_t)(s & 0x8000); }
};

// float_same FloorDivide (ufunc.rs:2493-2572): numpy's npy_divmod order.
template <class O> static typename O::T float_floor_divide(typename O::T x, typename O::T y) {
    typedef typename O::T T;
    if (O::isinf_(x) && O::isfin(y) && !O::iszero(y)) return O::nan();
    if (O::isinf_(y) && O::isfin(x) && !O::iszero(x) && O::neg(x) != O::neg(y)) return O::negone();
    if (O::isfin(x) && O::isfin(y) && !O::iszero(y)) {
        T raw_r = O::rem(x, y);
        T div = O::div(O::sub(x, raw_r), y);
        if (!O::iszero(raw_r)) {
            if (O::neg(raw_r) != O::neg(y)) div = O::sub(div, O::one());
        }
        if (!O::iszero(div)) {
            T fl = O::floor_(div);
            return O::gt(O::sub(div, fl), O::half()) ? O::add(fl, O::one()) : fl;
        }
        return O::copysign0(O::div(x, y));
    }
    return O::floor_(O::div(x, y));
}

// float_max / float_min (ufunc.rs:2402-2436): NaN operand returned as is,
// +0 wins a signed-zero tie for max, -0 for min.
template <class F> static F float_max(F x, F y) {
    if (x != x) return x;
    if (y != y) return y;
    if (x == y) return std::signbit(x) ? y : x;
    return x > y ? x : y;
}
template <class F> static F float_min(F x, F y) {
    if (x != x) return x;
    if (y != y) return y;
    if (x == y) return std::signbit(x) ? x : y;
    return x < y ? x : y;
}
// float_same_f16 Maximum/Minimum (ufunc.rs:2448-2458): first operand on ties.
static uint16_t h_max(uint16_t x, uint16_t y) {
    if (OpsF16::isnan_(x)) return x;
    if (OpsF16::isnan_(y)) return y;
    float a = h2f(x), b = h2f(y);
    if (a == b) return x;
    return a > b ? x : y;
}
static uint16_t h_min(uint16_t x, uint16_t y) {
    if (OpsF16::isnan_(x)) return x;
    if (OpsF16::isnan_(y)) return y;
    float a = h2f(x), b = h2f(y);
    if (a == b) return x;
    return a < b ? x : y;
}

// float_remainder_f / _f32 (ufunc.rs:4015-4034)
template <class F> static F float_remainder(F x, F y) {
    F r = o_fmod(x, y);
    if (r == 0) return std::copysign((F)0, y);
    if ((r < 0) != (y < 0)) return fadd(r, y);
    return r;
}

// ---------------------------------------------------------------------------
// Integer ops (ufunc.rs:2200-2320, 4036-4128)
// ---------------------------------------------------------------------------
template <class I> static I w_add(I x, I y) { typedef typename std::make_unsigned<I>::type U; return (I)((U)x + (U)y); }
template <class I> static I w_sub(I x, I y) { typedef typename std::make_unsigned<I>::type U; return (I)((U)x - (U)y); }
template <class I> static I w_mul(I x, I y) {
    typedef typename std::make_unsigned<I>::type U;
    if (sizeof(I) < sizeof(int)) return (I)((unsigned)(U)x * (unsigned)(U)y);
    return (I)((U)x * (U)y);
}
template <class I> static I w_div(I x, I y) {  // wrapping_div: MIN / -1 = MIN
    if (std::is_signed<I>::value && y == (I)-1) return w_sub<I>((I)0, x);
    return (I)(x / y);
}
template <class I> static I w_rem(I x, I y) {  // wrapping_rem: MIN % -1 = 0
    if (std::is_signed<I>::value && y == (I)-1) return 0;
    return (I)(x % y);
}
template <class I> static I floor_div(I x, I y) {
    if (y == 0) return 0;
    if (!std::is_signed<I>::value) return (I)(x / y);
    I q = w_div(x, y), r = w_rem(x, y);
    if (r != 0 && ((r < 0) != (y < 0))) return w_sub<I>(q, (I)1);
    return q;
}
template <class I> static I int_remainder(I x, I y) {
    if (y == 0) return 0;
    if (!std::is_signed<I>::value) return (I)(x % y);
    I r = w_rem(x, y);
    if (r != 0 && ((r < 0) != (y < 0))) return w_add(r, y);
    return r;
}
template <class I> static I int_fmod(I x, I y) { return y == 0 ? (I)0 : w_rem(x, y); }
template <class I> static I shl_np(I x, I amt) {
    const int B = (int)sizeof(I) * 8;
    if ((std::is_signed<I>::value && amt < 0) || amt >= (I)B) return 0;
    typedef typename std::make_unsigned<I>::type U;
    return (I)(U)((U)x << (int)amt);
}
template <class I> static I shr_np(I x, I amt) {
    const int B = (int)sizeof(I) * 8;
    if ((std::is_signed<I>::value && amt < 0) || amt >= (I)B) return (std::is_signed<I>::value && x < 0) ? (I)-1 : (I)0;
    return (I)(x >> (int)amt);
}

template <class I> static I int_same(int op, I x, I y) {
    switch (op) {
        case OP_ADD: return w_add(x, y);
        case OP_SUBTRACT: return w_sub(x, y);
        case OP_MULTIPLY: return w_mul(x, y);
        case OP_MAXIMUM: return x > y ? x : y;   // Ord::max returns the second on ties; equal ints are identical
        case OP_MINIMUM: return x < y ? x : y;
        case OP_BITWISE_AND: return x & y;
        case OP_BITWISE_OR: return x | y;
        case OP_BITWISE_XOR: return x ^ y;
        case OP_FLOOR_DIVIDE: return floor_div(x, y);
        case OP_LEFT_SHIFT: return shl_np(x, y);
        case OP_RIGHT_SHIFT: return shr_np(x, y);
        case OP_REMAINDER: return int_remainder(x, y);
        case OP_FMOD: return int_fmod(x, y);
    }
    return 0;
}
static bool bool_same(int op, bool x, bool y) {
    switch (op) {
        case OP_ADD: case OP_MAXIMUM: case OP_LOGICAL_OR: case OP_BITWISE_OR: return x || y;
        case OP_MULTIPLY: case OP_MINIMUM: case OP_LOGICAL_AND: case OP_BITWISE_AND: return x && y;
        case OP_LOGICAL_XOR: case OP_BITWISE_XOR: return x != y;
    }
    return false;
}
template <class T> static bool cmp_same(int op, T x, T y) {
    switch (op) {
        case OP_GREATER: return x > y;
        case OP_GREATER_EQUAL: return x >= y;
        case OP_LESS: return x < y;
        case OP_LESS_EQUAL: return x <= y;
        case OP_EQUAL: return x == y;
        case OP_NOT_EQUAL: return x != y;
    }
    return false;
}
template <class F> static F float_same(int op, F x, F y) {
    switch (op) {
        case OP_ADD: return fadd(x, y);
        case OP_SUBTRACT: return fsub(x, y);
        case OP_MULTIPLY: return fmul(x, y);
        case OP_DIVIDE: return fdiv(x, y);
        case OP_MAXIMUM: return float_max(x, y);
        case OP_MINIMUM: return float_min(x, y);
        case OP_FLOOR_DIVIDE:
            return sizeof(F) == 4 ? (F)float_floor_divide<OpsF32>((float)x, (float)y)
                                  : (F)float_floor_divide<OpsF64>((double)x, (double)y);
        case OP_REMAINDER: return float_remainder(x, y);
        case OP_FMOD: return o_fmod(x, y);
    }
    return 0;
}
static uint16_t half_same(int op, uint16_t x, uint16_t y) {
    switch (op) {
        case OP_ADD: return OpsF16::add(x, y);
        case OP_SUBTRACT: return OpsF16::sub(x, y);
        case OP_MULTIPLY: return OpsF16::mul(x, y);
        case OP_DIVIDE: return OpsF16::div(x, y);
        case OP_MAXIMUM: return h_max(x, y);
        case OP_MINIMUM: return h_min(x, y);
        case OP_FLOOR_DIVIDE: return float_floor_divide<OpsF16>(x, y);
        // math_binary_op F16 arm (ufunc.rs:5893-5915): f32 op, then from_f32
        case OP_REMAINDER: return f2h(float_remainder(h2f(x), h2f(y)));
        case OP_FMOD: return f2h(o_fmod(h2f(x), h2f(y)));
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Element access with runtime dtype, and the reference's casts
// (ionp-core/src/buffer.rs:64-330).
// ---------------------------------------------------------------------------
// A value held as its exact source dtype.
struct Val {
    int d;
    union { uint8_t b; int64_t i; uint64_t u; uint16_t h; float f; double g; };
};

static Val load(const OrArr* a, int64_t off) {
    Val v; v.d = a->dtype; v.u = 0;
    const char* base = (const char*)a->data;
    int64_t e = a->offset + off;
    switch (a->dtype) {
        case D_BOOL: v.b = ((const uint8_t*)base)[e] ? 1 : 0; break;
        case D_I8: v.i = ((const int8_t*)base)[e]; break;
        case D_I16: v.i = ((const int16_t*)base)[e]; break;
        case D_I32: v.i = ((const int32_t*)base)[e]; break;
        case D_I64: v.i = ((const int64_t*)base)[e]; break;
        case D_U8: v.u = ((const uint8_t*)base)[e]; break;
        case D_U16: v.u = ((const uint16_t*)base)[e]; break;
        case D_U32: v.u = ((const uint32_t*)base)[e]; break;
        case D_U64: v.u = ((const uint64_t*)base)[e]; break;
        case D_F16: v.h = ((const uint16_t*)base)[e]; break;
        case D_F32: v.f = ((const float*)base)[e]; break;
        case D_F64: v.g = ((const double*)base)[e]; break;
    }
    return v;
}

// Rust `f as iN` / `f as uN`: saturating, NaN -> 0.
template <class I> static I sat_from_double(double x) {
    if (x != x) return 0;
    const double lo = (double)std::numeric_limits<I>::min();
    const double hi = (double)std::numeric_limits<I>::max();
    if (x <= lo) return std::numeric_limits<I>::min();
    if (x >= hi) return std::numeric_limits<I>::max();
    return (I)x;  // in range: truncation toward zero
}
// float -> narrow int: (x as i32) as iN (buffer.rs:92-100)
template <class I> static I narrow_from_double(double x) { return (I)(uint32_t)sat_from_double<int32_t>(x); }

static double as_double_for_int_cast(const Val& v) {  // float source as f64 (exact)
    if (v.d == D_F32) return (double)v.f;
    if (v.d == D_F64) return v.g;
    return (double)h2f(v.h);
}

// cast_to(dst) of one element: returns the bits in `out` (itemsize bytes).
static void cast_store(const Val& v, int dst, void* out) {
    Kind k = kind_of(v.d);
    if (k == K_BOOL || k == K_INT || k == K_UINT) {
        bool is_u = (k == K_UINT);
        int64_t si = (k == K_BOOL) ? (int64_t)v.b : (k == K_INT ? v.i : (int64_t)v.u);
        uint64_t ui = (k == K_BOOL) ? (uint64_t)v.b : (k == K_INT ? (uint64_t)v.i : v.u);
        switch (dst) {
            case D_BOOL: *(uint8_t*)out = (ui != 0); return;
            case D_I8: *(int8_t*)out = (int8_t)ui; return;
            case D_I16: *(int16_t*)out = (int16_t)ui; return;
            case D_I32: *(int32_t*)out = (int32_t)ui; return;
            case D_I64: *(int64_t*)out = (int64_t)ui; return;
            case D_U8: *(uint8_t*)out = (uint8_t)ui; return;
            case D_U16: *(uint16_t*)out = (uint16_t)ui; return;
            case D_U32: *(uint32_t*)out = (uint32_t)ui; return;
            case D_U64: *(uint64_t*)out = ui; return;
            case D_F16: {
                double d = is_u ? (double)ui : (double)si;
                if (k == K_BOOL) { *(uint16_t*)out = v.b ? 0x3C00 : 0; return; }
                *(uint16_t*)out = d2h(d); return;
            }
            case D_F32: *(float*)out = is_u ? (float)ui : (float)si; return;
            case D_F64: *(double*)out = is_u ? (double)ui : (double)si; return;
        }
        return;
    }
    // float sources
    if (v.d == D_F16) {
        float f = h2f(v.h);
        switch (dst) {
            case D_BOOL: *(uint8_t*)out = (v.h & 0x7FFF) != 0; return;
            case D_I8: *(int8_t*)out = narrow_from_double<int8_t>(f); return;
            case D_I16: *(int16_t*)out = narrow_from_double<int16_t>(f); return;
            case D_I32: *(int32_t*)out = sat_from_double<int32_t>(f); return;
            case D_I64: *(int64_t*)out = sat_from_double<int64_t>(f); return;
            case D_U8: *(uint8_t*)out = narrow_from_double<uint8_t>(f); return;
            case D_U16: *(uint16_t*)out = narrow_from_double<uint16_t>(f); return;
            case D_U32: *(uint32_t*)out = sat_from_double<uint32_t>(f); return;
            case D_U64: *(uint64_t*)out = sat_from_double<uint64_t>(f); return;
            case D_F16: *(uint16_t*)out = v.h; return;
            case D_F32: *(float*)out = f; return;
            case D_F64: *(double*)out = f2d(f); return;
        }
        return;
    }
    double x = as_double_for_int_cast(v);
    bool nz = (v.d == D_F32) ? (v.f != 0) : (v.g != 0);
    switch (dst) {
        case D_BOOL: *(uint8_t*)out = nz; return;
        case D_I8: *(int8_t*)out = narrow_from_double<int8_t>(x); return;
        case D_I16: *(int16_t*)out = narrow_from_double<int16_t>(x); return;
        case D_I32: *(int32_t*)out = sat_from_double<int32_t>(x); return;
        case D_I64: *(int64_t*)out = sat_from_double<int64_t>(x); return;
        case D_U8: *(uint8_t*)out = narrow_from_double<uint8_t>(x); return;
        case D_U16: *(uint16_t*)out = narrow_from_double<uint16_t>(x); return;
        case D_U32: *(uint32_t*)out = sat_from_double<uint32_t>(x); return;
        case D_U64: *(uint64_t*)out = sat_from_double<uint64_t>(x); return;
        case D_F16: *(uint16_t*)out = (v.d == D_F32) ? d2h(f2d(v.f)) : d2h(v.g); return;
        case D_F32: *(float*)out = (v.d == D_F32) ? v.f : d2f(v.g); return;
        case D_F64: *(double*)out = (v.d == D_F32) ? f2d(v.f) : v.g; return;
    }
}

// A C-contiguous host buffer of one dtype (the result of `cast_to`).
struct Buf {
    int d;
    std::vector<int64_t> shape, strides;
    std::vector<uint8_t> bytes;
    int64_t size() const { int64_t n = 1; for (auto s : shape) n *= s; return n; }
};

static std::vector<int64_t> c_strides(const std::vector<int64_t>& shape) {
    std::vector<int64_t> st(shape.size());
    int64_t acc = 1;
    for (int i = (int)shape.size() - 1; i >= 0; --i) { st[i] = acc; acc *= std::max<int64_t>(shape[i], 1); }
    return st;
}

// NdIter (shape.rs:317-390): C-order odometer yielding element offsets.
template <class Fn> static void nd_iter(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, Fn fn) {
    int nd = (int)shape.size();
    for (int i = 0; i < nd; ++i) if (shape[i] == 0) return;
    std::vector<int64_t> idx(nd, 0);
    int64_t off = 0;
    while (true) {
        fn(off);
        int ax = nd - 1;
        while (ax >= 0) {
            idx[ax]++;
            off += strides[ax];
            if (idx[ax] < shape[ax]) break;
            off -= strides[ax] * shape[ax];
            idx[ax] = 0;
            ax--;
        }
        if (ax < 0) return;
    }
}

static std::vector<int64_t> shape_of(const OrArr* a) { return std::vector<int64_t>(a->shape, a->shape + a->ndim); }
static std::vector<int64_t> strides_of(const OrArr* a) { return std::vector<int64_t>(a->strides, a->strides + a->ndim); }

// cast_to (array.rs:393): C-contiguous copy in the target dtype.
static Buf cast_to(const OrArr* a, int dst) {
    Buf b; b.d = dst; b.shape = shape_of(a); b.strides = c_strides(b.shape);
    int64_t n = b.size();
    int is = itemsize(dst);
    b.bytes.resize((size_t)(n * is) + 8);
    int64_t k = 0;
    nd_iter(b.shape, strides_of(a), [&](int64_t off) {
        Val v = load(a, off);
        cast_store(v, dst, b.bytes.data() + k * is);
        k++;
    });
    return b;
}

static OrArr view_of(const Buf& b) {
    OrArr a; memset(&a, 0, sizeof(a));
    a.dtype = b.d; a.ndim = (int)b.shape.size();
    for (int i = 0; i < a.ndim; ++i) { a.shape[i] = b.shape[i]; a.strides[i] = b.strides[i]; }
    a.offset = 0; a.data = (void*)b.bytes.data();
    return a;
}

// broadcast_shapes (shape.rs:54-72)
static int broadcast_shapes(const std::vector<int64_t>& a, const std::vector<int64_t>& b, std::vector<int64_t>& out) {
    size_t nd = std::max(a.size(), b.size());
    out.assign(nd, 0);
    for (size_t i = 0; i < nd; ++i) {
        int64_t da = i < nd - a.size() ? 1 : a[i - (nd - a.size())];
        int64_t db = i < nd - b.size() ? 1 : b[i - (nd - b.size())];
        if (da == db) out[i] = da;
        else if (da == 1) out[i] = db;
        else if (db == 1) out[i] = da;
        else return ST_BROADCAST;
    }
    return ST_OK;
}
// broadcast_strides_to (shape.rs:113-160): 0 stride on broadcast axes.
static std::vector<int64_t> bstrides(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, const std::vector<int64_t>& target) {
    size_t nd = target.size(), pad = nd - shape.size();
    std::vector<int64_t> out(nd, 0);
    for (size_t i = pad; i < nd; ++i) out[i] = (shape[i - pad] == 1 && target[i] != 1) ? 0 : strides[i - pad];
    return out;
}

template <class T> static T& at(Buf& b, int64_t e) { return ((T*)b.bytes.data())[e]; }
template <class T> static const T& atc(const Buf& b, int64_t e) { return ((const T*)b.bytes.data())[e]; }

// binary_elementwise (ufunc.rs:3539-3564) over two buffers of the same dtype.
template <class T, class TO, class Fn>
static void bin_loop(const Buf& a, const Buf& b, const std::vector<int64_t>& oshape, TO* out, Fn fn) {
    auto sa = bstrides(a.shape, a.strides, oshape), sb = bstrides(b.shape, b.strides, oshape);
    std::vector<int64_t> offa, offb;
    int64_t n = 1; for (auto s : oshape) n *= s;
    offa.reserve(n); offb.reserve(n);
    nd_iter(oshape, sa, [&](int64_t o) { offa.push_back(o); });
    nd_iter(oshape, sb, [&](int64_t o) { offb.push_back(o); });
    const T* pa = (const T*)a.bytes.data();
    const T* pb = (const T*)b.bytes.data();
    for (size_t i = 0; i < offa.size(); ++i) out[i] = fn(pa[offa[i]], pb[offb[i]]);
}

// ---------------------------------------------------------------------------
// FPE detectors (ionp-core/src/fpe.rs:173-398). Operands are flattened in
// C order and paired as `x[i % len_x]` exactly like the reference.
// ---------------------------------------------------------------------------
enum { FPE_DIVIDE = 1, FPE_OVER = 2, FPE_UNDER = 4, FPE_INVALID = 8 };

static std::vector<double> to_f64_lossy(const OrArr* a) {
    std::vector<double> v;
    nd_iter(shape_of(a), strides_of(a), [&](int64_t off) {
        Val x = load(a, off);
        double d = 0;
        switch (kind_of(x.d)) {
            case K_BOOL: d = x.b ? 1.0 : 0.0; break;
            case K_INT: d = (double)x.i; break;
            case K_UINT: d = (double)x.u; break;
            case K_FLOAT: d = x.d == D_F16 ? h2d(x.h) : (x.d == D_F32 ? (double)x.f : x.g); break;
        }
        v.push_back(d);
    });
    return v;
}
static int64_t numel(const OrArr* a) { int64_t n = 1; for (int i = 0; i < a->ndim; ++i) n *= a->shape[i]; return n; }

static int detect_divide_family(const OrArr* a, const OrArr* b, bool out_is_floating) {
    if (numel(a) == 0 || numel(b) == 0) return 0;
    auto av = to_f64_lossy(a), bv = to_f64_lossy(b);
    size_t n = std::max(av.size(), bv.size());
    bool saw_divide = false;
    for (size_t i = 0; i < n; ++i) {
        double x = av[av.size() == 1 ? 0 : i % av.size()];
        double y = bv[bv.size() == 1 ? 0 : i % bv.size()];
        if (y == 0.0) {
            if (x == 0.0 && out_is_floating) return FPE_INVALID;
            saw_divide = true;
        }
    }
    return saw_divide ? FPE_DIVIDE : 0;
}
static int detect_remainder(const OrArr* a, const OrArr* b, bool out_is_floating) {
    if (out_is_floating) return 0;
    if (numel(a) == 0 || numel(b) == 0) return 0;
    auto av = to_f64_lossy(a), bv = to_f64_lossy(b);
    size_t n = std::max(av.size(), bv.size());
    for (size_t i = 0; i < n; ++i) {
        double y = bv[bv.size() == 1 ? 0 : i % bv.size()];
        if (y == 0.0) return FPE_DIVIDE;
    }
    return 0;
}
static int detect_multiply(const OrArr* a, const OrArr* b, const OrArr* out) {
    if (numel(a) == 0 || numel(b) == 0 || numel(out) == 0) return 0;
    auto av = to_f64_lossy(a), bv = to_f64_lossy(b);
    size_t olen = (size_t)std::max<int64_t>(numel(out), 1);
    size_t n = std::max(std::max(av.size(), bv.size()), olen);
    // out_is_infinite / out_finite_and_zero_or_subnormal (fpe.rs:320-345)
    std::vector<uint8_t> oinf, ozero;
    nd_iter(shape_of(out), strides_of(out), [&](int64_t off) {
        Val v = load(out, off);
        bool inf = false, tiny = false;
        if (v.d == D_F16) {
            uint16_t h = v.h; int e = (h >> 10) & 0x1F;
            inf = (h & 0x7FFF) == 0x7C00; tiny = (e == 0);
        } else if (v.d == D_F32) {
            inf = std::isinf(v.f); tiny = std::isfinite(v.f) && (v.f == 0 || !std::isnormal(v.f));
        } else if (v.d == D_F64) {
            inf = std::isinf(v.g); tiny = std::isfinite(v.g) && (v.g == 0 || !std::isnormal(v.g));
        }
        oinf.push_back(inf); ozero.push_back(tiny);
    });
    bool over = false, under = false;
    for (size_t i = 0; i < n; ++i) {
        double x = av[av.size() == 1 ? 0 : i % av.size()];
        double y = bv[bv.size() == 1 ? 0 : i % bv.size()];
        if (!std::isfinite(x) || !std::isfinite(y) || x == 0.0 || y == 0.0) continue;
        size_t oi = olen == 1 ? 0 : i % olen;
        if (oinf[oi]) over = true;
        else if (ozero[oi]) under = true;
    }
    return over ? FPE_OVER : under ? FPE_UNDER : 0;
}

// ---------------------------------------------------------------------------
// Reductions (ufunc.rs:6349-7825)
// ---------------------------------------------------------------------------
static const int PW_BLOCKSIZE = 128;

// tree_combine (ufunc.rs:6371-6378)
template <class T, class Add> static T tree_combine(const T* r, int n, Add add) {
    if (n == 1) return r[0];
    int mid = n / 2;
    return add(tree_combine(r, mid, add), tree_combine(r + mid, n - mid, add));
}
// pairwise_sum (ufunc.rs:6416-6448)
template <class T, class Get, class Add> static T pairwise_sum(Get get, int64_t base, int64_t n, Add add, int width) {
    int64_t block = PW_BLOCKSIZE / 8 * width;
    if (n < width) {
        T res = get(base);
        for (int64_t i = 1; i < n; ++i) res = add(res, get(base + i));
        return res;
    } else if (n <= block) {
        T r[8];
        for (int j = 0; j < width; ++j) r[j] = get(base + j);
        int64_t i = width;
        while (i < n - (n % width)) {
            for (int j = 0; j < width; ++j) r[j] = add(r[j], get(base + i + j));
            i += width;
        }
        T res = tree_combine(r, width, add);
        while (i < n) { res = add(res, get(base + i)); ++i; }
        return res;
    } else {
        int64_t n2 = n / 2;
        n2 -= n2 % width;
        return add(pairwise_sum<T>(get, base, n2, add, width), pairwise_sum<T>(get, base + n2, n - n2, add, width));
    }
}

// axes_by_memory_order (ufunc.rs:6463-6467): stable sort by |stride| desc.
static std::vector<int> axes_by_memory_order(const std::vector<int64_t>& strides, std::vector<int> axes) {
    std::stable_sort(axes.begin(), axes.end(), [&](int a, int b) { return std::llabs(strides[a]) > std::llabs(strides[b]); });
    return axes;
}
// coalesce_runs (ufunc.rs:6481-6502): innermost-first (size, stride) runs.
static std::vector<std::pair<int64_t, int64_t>> coalesce_runs(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides) {
    std::vector<std::pair<int64_t, int64_t>> runs;
    for (int i = (int)shape.size() - 1; i >= 0; --i) {
        if (shape[i] <= 1) continue;
        if (!runs.empty() && strides[i] == runs.back().second * runs.back().first) runs.back().first *= shape[i];
        else runs.push_back({shape[i], strides[i]});
    }
    return runs;
}
// pairwise_group (ufunc.rs:6504-6544)
template <class T, class Get, class Add>
static T pairwise_group(Get get, int64_t base, const std::vector<std::pair<int64_t, int64_t>>& runs, Add add, int width) {
    if (runs.empty()) return get(base);
    int64_t isz = runs[0].first, ist = runs[0].second;
    auto inner = [&](int64_t b) {
        return pairwise_sum<T>([&](int64_t i) { return get(b + ist * i); }, 0, isz, add, width);
    };
    if (runs.size() == 1) return inner(base);
    std::vector<int64_t> oshape, ostr;
    for (size_t r = 1; r < runs.size(); ++r) { oshape.push_back(runs[r].first); ostr.push_back(runs[r].second); }
    bool first = true; T acc{};
    nd_iter(oshape, ostr, [&](int64_t o) {
        T v = inner(base + o);
        if (first) { acc = v; first = false; } else acc = add(acc, v);
    });
    return acc;
}

struct RedPlan {
    std::vector<int> keep_axes, wide_axes, narrow_axes;
    std::vector<int64_t> keep_shape, keep_strides, narrow_shape, narrow_strides;
    std::vector<int64_t> wide_shape_il, wide_strides_il;   // wide axes, innermost last
    std::vector<std::pair<int64_t, int64_t>> wide_runs;
};
static bool contains(const std::vector<int>& v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); }

// The wide/narrow classification shared by ufunc.rs:6679-6700, 6893-6913,
// 7254-7275 and 7445-7466.
static RedPlan make_plan(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, const std::vector<int>& red) {
    RedPlan p;
    int nd = (int)shape.size();
    for (int a = 0; a < nd; ++a) if (!contains(red, a)) { p.keep_axes.push_back(a); p.keep_shape.push_back(shape[a]); p.keep_strides.push_back(strides[a]); }
    std::vector<int> by_stride;
    for (int a = 0; a < nd; ++a) if (shape[a] > 1) by_stride.push_back(a);
    std::stable_sort(by_stride.begin(), by_stride.end(), [&](int a, int b) { return std::llabs(strides[a]) < std::llabs(strides[b]); });
    for (int a : by_stride) { if (contains(red, a)) p.wide_axes.push_back(a); else break; }
    for (int i = (int)p.wide_axes.size() - 1; i >= 0; --i) { p.wide_shape_il.push_back(shape[p.wide_axes[i]]); p.wide_strides_il.push_back(strides[p.wide_axes[i]]); }
    p.wide_runs = coalesce_runs(p.wide_shape_il, p.wide_strides_il);
    std::vector<int> nar;
    for (int a : red) if (!contains(p.wide_axes, a)) nar.push_back(a);
    p.narrow_axes = axes_by_memory_order(strides, nar);
    for (int a : p.narrow_axes) { p.narrow_shape.push_back(shape[a]); p.narrow_strides.push_back(strides[a]); }
    return p;
}

// Identities: int_identity (2322), bool_identity (2371), f*_identity (6131-6150).
static bool identity_of(int op, int d, uint8_t* out /*8 bytes*/) {
    memset(out, 0, 8);
    Kind k = kind_of(d);
    if (k == K_BOOL) {
        if (op == OP_ADD || op == OP_LOGICAL_OR || op == OP_BITWISE_OR || op == OP_LOGICAL_XOR || op == OP_BITWISE_XOR) { out[0] = 0; return true; }
        if (op == OP_MULTIPLY || op == OP_LOGICAL_AND || op == OP_BITWISE_AND) { out[0] = 1; return true; }
        return false;
    }
    if (k == K_INT || k == K_UINT) {
        int is = itemsize(d);
        if (op == OP_ADD || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) return true;
        if (op == OP_MULTIPLY) { out[0] = 1; return true; }
        if (op == OP_BITWISE_AND) { memset(out, 0xFF, is); return true; }
        return false;
    }
    if (op == OP_ADD) return true;
    if (op == OP_MULTIPLY) {
        if (d == D_F16) { uint16_t one = 0x3C00; memcpy(out, &one, 2); }
        else if (d == D_F32) { float one = 1.0f; memcpy(out, &one, 4); }
        else { double one = 1.0; memcpy(out, &one, 8); }
        return true;
    }
    return false;
}

// The per-dtype fold (int_same/bool_fold/float_same/float_same_f16) as a
// functor on raw values.
template <class T> struct Fold;
template <> struct Fold<uint8_t> {  // bool
    int op; bool operator()(uint8_t x, uint8_t y) const {
        if (is_compare(op)) return cmp_same<bool>(op, x != 0, y != 0);
        return bool_same(op, x != 0, y != 0);
    }
};
template <class T> struct Fold { int op; T operator()(T x, T y) const { return int_same<T>(op, x, y); } };
template <> struct Fold<float> { int op; float operator()(float x, float y) const { return float_same<float>(op, x, y); } };
template <> struct Fold<double> { int op; double operator()(double x, double y) const { return float_same<double>(op, x, y); } };
struct FoldH { int op; uint16_t operator()(uint16_t x, uint16_t y) const { return half_same(op, x, y); } };

// reduce_axis_pairwise_narrow_wide (ufunc.rs:6658-6806) for f32/f64 Add.
template <class T, class F>
static void reduce_pairwise(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, int64_t offset,
                            const T* buf, const std::vector<int>& red, F add, T seed, T* out) {
    RedPlan p = make_plan(shape, strides, red);
    auto get = [&](int64_t o) { return buf[o]; };
    auto compute_wide = [&](int64_t wb) -> T {
        if (p.wide_axes.empty()) return get(wb);
        return pairwise_group<T>(get, wb, p.wide_runs, add, 8);
    };
    auto compute_one = [&](int64_t base) -> T {
        if (p.narrow_axes.empty()) return add(seed, compute_wide(base));
        T acc = seed;
        nd_iter(p.narrow_shape, p.narrow_strides, [&](int64_t o) { acc = add(acc, compute_wide(base + o)); });
        return acc;
    };
    int64_t k = 0;
    if (p.keep_axes.empty()) { out[0] = compute_one(offset); return; }
    nd_iter(p.keep_shape, p.keep_strides, [&](int64_t ko) { out[k++] = compute_one(offset + ko); });
}

// reduce_axis_f16_narrow_wide (ufunc.rs:6868-7089)
static int reduce_f16(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, int64_t offset,
                      const uint16_t* buf, const std::vector<int>& red, int op, bool has_init, uint16_t init, uint16_t* out) {
    RedPlan p = make_plan(shape, strides, red);
    auto get32 = [&](int64_t o) { return h2f(buf[o]); };
    auto add32 = [](float x, float y) { return fadd(x, y); };
    auto op32 = [&](float x, float y) { return float_same<float>(op, x, y); };
    auto compute_wide = [&](int64_t wb) -> float {
        if (p.wide_axes.empty()) return get32(wb);
        if (op == OP_ADD) return pairwise_group<float>(get32, wb, p.wide_runs, add32, 8);
        bool first = true; float acc = 0;
        nd_iter(p.wide_shape_il, p.wide_strides_il, [&](int64_t o) {
            if (first) { acc = get32(wb + o); first = false; } else acc = op32(acc, get32(wb + o));
        });
        return acc;
    };
    auto compute_wide_seeded = [&](int64_t wb, float s) -> float {
        if (p.wide_axes.empty()) return op32(s, get32(wb));
        float acc = s;
        nd_iter(p.wide_shape_il, p.wide_strides_il, [&](int64_t o) { acc = op32(acc, get32(wb + o)); });
        return acc;
    };
    bool has_seed = has_init; uint16_t seed = init;
    if (!has_seed) {
        if (op == OP_ADD) { has_seed = true; seed = 0; }
        else if (op == OP_MULTIPLY) { has_seed = true; seed = 0x3C00; }
    }
    auto compute_one = [&](int64_t base) -> uint16_t {
        if (p.narrow_axes.empty()) {
            if (has_seed && op != OP_ADD) return f2h(compute_wide_seeded(base, h2f(seed)));
            if (has_seed) return half_same(op, seed, f2h(compute_wide(base)));
            return f2h(compute_wide(base));
        }
        bool have = has_seed; uint16_t acc = seed;
        nd_iter(p.narrow_shape, p.narrow_strides, [&](int64_t o) {
            uint16_t part = f2h(compute_wide(base + o));
            if (!have) { acc = part; have = true; } else acc = half_same(op, acc, part);
        });
        return acc;
    };
    int64_t k = 0;
    if (p.keep_axes.empty()) { out[0] = compute_one(offset); return ST_OK; }
    nd_iter(p.keep_shape, p.keep_strides, [&](int64_t ko) { out[k++] = compute_one(offset + ko); });
    return ST_OK;
}

// sequential_group (6546) / sequential_group_ordered (6583) under
// reduce_axis_generic (7091-7150).
template <class T, class F>
static void reduce_sequential(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, int64_t offset,
                              const T* buf, const std::vector<int>& red, F fold, bool has_seed, T seed, bool ordered, T* out) {
    std::vector<int> keep;
    std::vector<int64_t> ks, kst;
    for (int a = 0; a < (int)shape.size(); ++a) if (!contains(red, a)) { keep.push_back(a); ks.push_back(shape[a]); kst.push_back(strides[a]); }
    std::vector<int> rax = red;
    if (ordered) rax = axes_by_memory_order(strides, red);
    std::vector<int64_t> rs, rst;
    for (int a : rax) { rs.push_back(shape[a]); rst.push_back(strides[a]); }
    auto compute_one = [&](int64_t base) -> T {
        bool have = has_seed; T acc = seed;
        nd_iter(rs, rst, [&](int64_t o) {
            T v = buf[base + o];
            if (!have) { acc = v; have = true; } else acc = fold(acc, v);
        });
        return acc;
    };
    int64_t k = 0;
    if (keep.empty()) { out[0] = compute_one(offset); return; }
    nd_iter(ks, kst, [&](int64_t ko) { out[k++] = compute_one(offset + ko); });
}

// reduce_axis_masked (ufunc.rs:7213-7412)
template <class T, class F>
static void reduce_masked(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, int64_t offset, const T* buf,
                          const std::vector<int64_t>& mstrides, int64_t moff, const uint8_t* mbuf,
                          const std::vector<int>& red, F fold, bool pairwise, T seed, T* out) {
    int nd = (int)shape.size();
    std::vector<int> keep;
    std::vector<int64_t> ks, kst, kmst;
    for (int a = 0; a < nd; ++a) if (!contains(red, a)) { keep.push_back(a); ks.push_back(shape[a]); kst.push_back(strides[a]); kmst.push_back(mstrides[a]); }
    int64_t k = 0;
    if (pairwise) {
        RedPlan p = make_plan(shape, strides, red);
        std::vector<int64_t> nmst, wsh, wst, wmst;
        for (int a : p.narrow_axes) nmst.push_back(mstrides[a]);
        for (int i = (int)p.wide_axes.size() - 1; i >= 0; --i) { int a = p.wide_axes[i]; wsh.push_back(shape[a]); wst.push_back(strides[a]); wmst.push_back(mstrides[a]); }
        auto cwm = [&](int64_t wb, int64_t mwb, T acc_in) -> T {
            if (p.wide_axes.empty()) return mbuf[mwb] ? fold(acc_in, buf[wb]) : acc_in;
            std::vector<int64_t> offs, moffs;
            nd_iter(wsh, wst, [&](int64_t o) { offs.push_back(wb + o); });
            nd_iter(wsh, wmst, [&](int64_t o) { moffs.push_back(mwb + o); });
            T acc = acc_in;
            std::vector<int64_t> run;
            auto flush = [&]() {
                if (run.empty()) return;
                T r = pairwise_sum<T>([&](int64_t i) { return buf[run[i]]; }, 0, (int64_t)run.size(), fold, 8);
                acc = fold(acc, r);
                run.clear();
            };
            for (size_t i = 0; i < offs.size(); ++i) { if (mbuf[moffs[i]]) run.push_back(offs[i]); else flush(); }
            flush();
            return acc;
        };
        auto one = [&](int64_t base, int64_t mbase) -> T {
            if (p.narrow_axes.empty()) return cwm(base, mbase, seed);
            std::vector<int64_t> no, nmo;
            nd_iter(p.narrow_shape, p.narrow_strides, [&](int64_t o) { no.push_back(o); });
            nd_iter(p.narrow_shape, nmst, [&](int64_t o) { nmo.push_back(o); });
            T acc = seed;
            for (size_t i = 0; i < no.size(); ++i) acc = cwm(base + no[i], mbase + nmo[i], acc);
            return acc;
        };
        if (keep.empty()) { out[0] = one(offset, moff); return; }
        std::vector<int64_t> ko, kmo;
        nd_iter(ks, kst, [&](int64_t o) { ko.push_back(o); });
        nd_iter(ks, kmst, [&](int64_t o) { kmo.push_back(o); });
        for (size_t i = 0; i < ko.size(); ++i) out[k++] = one(offset + ko[i], moff + kmo[i]);
        return;
    }
    std::vector<int> ord = axes_by_memory_order(strides, red);
    std::vector<int64_t> rs, rst, rmst;
    for (int a : ord) { rs.push_back(shape[a]); rst.push_back(strides[a]); rmst.push_back(mstrides[a]); }
    auto fold_one = [&](int64_t base, int64_t mbase) -> T {
        std::vector<int64_t> o1, o2;
        nd_iter(rs, rst, [&](int64_t o) { o1.push_back(o); });
        nd_iter(rs, rmst, [&](int64_t o) { o2.push_back(o); });
        T acc = seed;
        for (size_t i = 0; i < o1.size(); ++i) if (mbuf[mbase + o2[i]]) acc = fold(acc, buf[base + o1[i]]);
        return acc;
    };
    if (keep.empty()) { out[0] = fold_one(offset, moff); return; }
    std::vector<int64_t> ko, kmo;
    nd_iter(ks, kst, [&](int64_t o) { ko.push_back(o); });
    nd_iter(ks, kmst, [&](int64_t o) { kmo.push_back(o); });
    for (size_t i = 0; i < ko.size(); ++i) out[k++] = fold_one(offset + ko[i], moff + kmo[i]);
}

// reduce_axis_masked_f16_widen (ufunc.rs:7414-7548)
static void reduce_masked_f16(const std::vector<int64_t>& shape, const std::vector<int64_t>& strides, int64_t offset, const uint16_t* buf,
                              const std::vector<int64_t>& mstrides, int64_t moff, const uint8_t* mbuf,
                              const std::vector<int>& red, int op, uint16_t seed, uint16_t* out) {
    int nd = (int)shape.size();
    std::vector<int64_t> ks, kst, kmst;
    std::vector<int> keep;
    for (int a = 0; a < nd; ++a) if (!contains(red, a)) { keep.push_back(a); ks.push_back(shape[a]); kst.push_back(strides[a]); kmst.push_back(mstrides[a]); }
    float seed32 = h2f(seed);
    RedPlan p = make_plan(shape, strides, red);
    std::vector<int64_t> nmst, wsh, wst, wmst;
    for (int a : p.narrow_axes) nmst.push_back(mstrides[a]);
    for (int i = (int)p.wide_axes.size() - 1; i >= 0; --i) { int a = p.wide_axes[i]; wsh.push_back(shape[a]); wst.push_back(strides[a]); wmst.push_back(mstrides[a]); }
    auto op32 = [&](float x, float y) { return float_same<float>(op, x, y); };
    auto get32 = [&](int64_t o) { return h2f(buf[o]); };
    auto cwm = [&](int64_t wb, int64_t mwb, float acc_in) -> float {
        if (p.wide_axes.empty()) return mbuf[mwb] ? h2f(f2h(op32(acc_in, get32(wb)))) : acc_in;
        std::vector<int64_t> offs, moffs;
        nd_iter(wsh, wst, [&](int64_t o) { offs.push_back(wb + o); });
        nd_iter(wsh, wmst, [&](int64_t o) { moffs.push_back(mwb + o); });
        float acc = acc_in;
        std::vector<int64_t> run;
        auto flush = [&]() {
            if (run.empty()) return;
            float combined;
            if (op == OP_ADD) {
                float r = pairwise_sum<float>([&](int64_t i) { return get32(run[i]); }, 0, (int64_t)run.size(), op32, 8);
                combined = op32(acc, r);
            } else if (op == OP_MULTIPLY) {
                float r = get32(run[0]);
                for (size_t i = 1; i < run.size(); ++i) r = op32(r, get32(run[i]));
                combined = op32(acc, r);
            } else {
                float a = acc;
                for (size_t i = 0; i < run.size(); ++i) a = op32(a, get32(run[i]));
                combined = a;
            }
            acc = h2f(f2h(combined));
            run.clear();
        };
        for (size_t i = 0; i < offs.size(); ++i) { if (mbuf[moffs[i]]) run.push_back(offs[i]); else flush(); }
        flush();
        return acc;
    };
    auto one = [&](int64_t base, int64_t mbase) -> uint16_t {
        if (p.narrow_axes.empty()) return f2h(cwm(base, mbase, seed32));
        std::vector<int64_t> no, nmo;
        nd_iter(p.narrow_shape, p.narrow_strides, [&](int64_t o) { no.push_back(o); });
        nd_iter(p.narrow_shape, nmst, [&](int64_t o) { nmo.push_back(o); });
        float acc = seed32;
        for (size_t i = 0; i < no.size(); ++i) acc = cwm(base + no[i], mbase + nmo[i], acc);
        return f2h(acc);
    };
    int64_t k = 0;
    if (keep.empty()) { out[0] = one(offset, moff); return; }
    std::vector<int64_t> ko, kmo;
    nd_iter(ks, kst, [&](int64_t o) { ko.push_back(o); });
    nd_iter(ks, kmst, [&](int64_t o) { kmo.push_back(o); });
    for (size_t i = 0; i < ko.size(); ++i) out[k++] = one(offset + ko[i], moff + kmo[i]);
}

// reduce_family_compute_dtype (ufunc.rs:2080-2168) + reduce_compute_dtype (2041-2078)
static int reduce_compute_dtype(int op, int in, int* out) {
    Kind k = kind_of(in);
    if (is_logical(op)) { *out = D_BOOL; return ST_OK; }
    if (is_bitwise(op)) { if (k == K_FLOAT) return ST_TYPE; *out = in; return ST_OK; }
    if (is_shift(op)) { if (k == K_FLOAT) return ST_TYPE; *out = in == D_BOOL ? D_I8 : in; return ST_OK; }
    if (op == OP_SUBTRACT && in == D_BOOL) return ST_TYPE;
    if (op == OP_FLOOR_DIVIDE && in == D_BOOL) { *out = D_I8; return ST_OK; }
    if (op == OP_DIVIDE && k != K_FLOAT) { *out = D_F64; return ST_OK; }
    if (op == OP_ADD || op == OP_MULTIPLY) {
        if (in == D_BOOL) { *out = D_I64; return ST_OK; }
        if (k == K_INT) { *out = D_I64; return ST_OK; }
        if (k == K_UINT) { *out = D_U64; return ST_OK; }
    }
    *out = in;
    return ST_OK;
}

template <class T, class F>
static int reduce_typed(int op, const OrArr* src, const std::vector<int>& red, int cd, F fold, bool pairwise, bool ordered,
                        const uint8_t* initial, const OrArr* mask, void* out) {
    std::vector<int64_t> shape = shape_of(src), strides = strides_of(src);
    const T* buf = (const T*)src->data;
    int64_t offset = src->offset;
    uint8_t idb[8];
    bool has_id = identity_of(op, cd, idb);
    bool has_seed = initial != nullptr || has_id;
    T seed{};
    if (initial) memcpy(&seed, initial, sizeof(T)); else if (has_id) memcpy(&seed, idb, sizeof(T));
    int64_t group = 1; for (int a : red) group *= shape[a];
    std::vector<int64_t> keep_shape; for (int a = 0; a < (int)shape.size(); ++a) if (!contains(red, a)) keep_shape.push_back(shape[a]);
    int64_t osz = 1; for (auto s : keep_shape) osz *= s;
    if (mask) {
        if (!has_seed) return ST_VALUE;
        std::vector<int64_t> mst = bstrides(shape_of(mask), strides_of(mask), shape);
        reduce_masked<T>(shape, strides, offset, buf, mst, mask->offset, (const uint8_t*)mask->data, red, fold, pairwise, seed, (T*)out);
        return ST_OK;
    }
    if (group == 0) {
        if (!has_seed) return ST_VALUE;
        for (int64_t i = 0; i < std::max<int64_t>(osz, 1); ++i) ((T*)out)[i] = seed;
        return ST_OK;
    }
    if (pairwise) { reduce_pairwise<T>(shape, strides, offset, buf, red, fold, seed, (T*)out); return ST_OK; }
    reduce_sequential<T>(shape, strides, offset, buf, red, fold, has_seed, seed, ordered, (T*)out);
    return ST_OK;
}

}  // namespace

// ===========================================================================
// C ABI of the oracle
// ===========================================================================
extern "C" {

int oracle_promote(int a, int b) { return promote(a, b); }

// Result dtype of a binary/unary call, or a negative status.
int oracle_binary_out_dtype(int op, int a, int b) {
    int out = -1, st;
    if (op == OP_REMAINDER || op == OP_FMOD) st = math_binary_out_dtype(op, a, b, &out);
    else st = binary_out_dtype(op, a, b, &out);
    return st == ST_OK ? out : -st;
}
int oracle_unary_out_dtype(int op, int a) {
    int out = -1, st = unary_out_dtype(op, a, &out);
    return st == ST_OK ? out : -st;
}
int oracle_reduce_compute_dtype(int op, int a) {
    if (is_compare(op) && a != D_BOOL) return -ST_NO_LOOP;
    int out = -1, st = reduce_compute_dtype(op, a, &out);
    return st == ST_OK ? out : -st;
}

// Element-wise cast of `a` into `out` (same shape, out's dtype/strides).
int oracle_cast(const OrArr* a, OrArr* out) {
    std::vector<int64_t> shape = shape_of(a);
    std::vector<int64_t> ooff;
    nd_iter(shape, strides_of(out), [&](int64_t o) { ooff.push_back(o); });
    size_t k = 0;
    int is = itemsize(out->dtype);
    nd_iter(shape, strides_of(a), [&](int64_t off) {
        Val v = load(a, off);
        cast_store(v, out->dtype, (char*)out->data + (out->offset + ooff[k++]) * is);
    });
    return ST_OK;
}

// binary_op / math_binary_op: result written C-contiguous into out->data
// (out dtype and broadcast shape as resolved by oracle_binary_out_dtype).
// *fpe receives the fpe_check_after_call category (lib.rs:9077-9138).
int oracle_binary(int op, const OrArr* a, const OrArr* b, OrArr* out, int* fpe) {
    int od = oracle_binary_out_dtype(op, a->dtype, b->dtype);
    if (od < 0) return -od;
    std::vector<int64_t> oshape;
    int st = broadcast_shapes(shape_of(a), shape_of(b), oshape);
    if (st != ST_OK) return st;
    int cd = is_compare(op) ? promote(a->dtype, b->dtype) : (is_logical(op) ? D_BOOL : od);
    Buf ca = cast_to(a, cd), cb = cast_to(b, cd);
    void* o = out->data;
    if (is_compare(op)) {
        uint8_t* po = (uint8_t*)o;
        switch (cd) {
            case D_BOOL: bin_loop<uint8_t>(ca, cb, oshape, po, [&](uint8_t x, uint8_t y) { return (uint8_t)cmp_same<bool>(op, x != 0, y != 0); }); break;
            case D_I8: bin_loop<int8_t>(ca, cb, oshape, po, [&](int8_t x, int8_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_I16: bin_loop<int16_t>(ca, cb, oshape, po, [&](int16_t x, int16_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_I32: bin_loop<int32_t>(ca, cb, oshape, po, [&](int32_t x, int32_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_I64: bin_loop<int64_t>(ca, cb, oshape, po, [&](int64_t x, int64_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_U8: bin_loop<uint8_t>(ca, cb, oshape, po, [&](uint8_t x, uint8_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_U16: bin_loop<uint16_t>(ca, cb, oshape, po, [&](uint16_t x, uint16_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_U32: bin_loop<uint32_t>(ca, cb, oshape, po, [&](uint32_t x, uint32_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_U64: bin_loop<uint64_t>(ca, cb, oshape, po, [&](uint64_t x, uint64_t y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_F16: bin_loop<uint16_t>(ca, cb, oshape, po, [&](uint16_t x, uint16_t y) { return (uint8_t)cmp_same(op, h2f(x), h2f(y)); }); break;
            case D_F32: bin_loop<float>(ca, cb, oshape, po, [&](float x, float y) { return (uint8_t)cmp_same(op, x, y); }); break;
            case D_F64: bin_loop<double>(ca, cb, oshape, po, [&](double x, double y) { return (uint8_t)cmp_same(op, x, y); }); break;
        }
    } else {
        switch (cd) {
            case D_BOOL: bin_loop<uint8_t>(ca, cb, oshape, (uint8_t*)o, [&](uint8_t x, uint8_t y) { return (uint8_t)bool_same(op, x != 0, y != 0); }); break;
            case D_I8: bin_loop<int8_t>(ca, cb, oshape, (int8_t*)o, [&](int8_t x, int8_t y) { return int_same(op, x, y); }); break;
            case D_I16: bin_loop<int16_t>(ca, cb, oshape, (int16_t*)o, [&](int16_t x, int16_t y) { return int_same(op, x, y); }); break;
            case D_I32: bin_loop<int32_t>(ca, cb, oshape, (int32_t*)o, [&](int32_t x, int32_t y) { return int_same(op, x, y); }); break;
            case D_I64: bin_loop<int64_t>(ca, cb, oshape, (int64_t*)o, [&](int64_t x, int64_t y) { return int_same(op, x, y); }); break;
            case D_U8: bin_loop<uint8_t>(ca, cb, oshape, (uint8_t*)o, [&](uint8_t x, uint8_t y) { return int_same(op, x, y); }); break;
            case D_U16: bin_loop<uint16_t>(ca, cb, oshape, (uint16_t*)o, [&](uint16_t x, uint16_t y) { return int_same(op, x, y); }); break;
            case D_U32: bin_loop<uint32_t>(ca, cb, oshape, (uint32_t*)o, [&](uint32_t x, uint32_t y) { return int_same(op, x, y); }); break;
            case D_U64: bin_loop<uint64_t>(ca, cb, oshape, (uint64_t*)o, [&](uint64_t x, uint64_t y) { return int_same(op, x, y); }); break;
            case D_F16: bin_loop<uint16_t>(ca, cb, oshape, (uint16_t*)o, [&](uint16_t x, uint16_t y) { return half_same(op, x, y); }); break;
            case D_F32: bin_loop<float>(ca, cb, oshape, (float*)o, [&](float x, float y) { return float_same<float>(op, x, y); }); break;
            case D_F64: bin_loop<double>(ca, cb, oshape, (double*)o, [&](double x, double y) { return float_same<double>(op, x, y); }); break;
        }
    }
    if (fpe) {
        *fpe = 0;
        bool ofl = kind_of(od) == K_FLOAT;
        if (op == OP_DIVIDE || op == OP_FLOOR_DIVIDE) *fpe = detect_divide_family(a, b, ofl);
        else if (op == OP_REMAINDER || op == OP_FMOD) *fpe = detect_remainder(a, b, ofl);
        else if (op == OP_MULTIPLY) {
            OrArr ov = *out;
            ov.dtype = od; ov.ndim = (int)oshape.size(); ov.offset = 0;
            auto cs = c_strides(oshape);
            for (int i = 0; i < ov.ndim; ++i) { ov.shape[i] = oshape[i]; ov.strides[i] = cs[i]; }
            *fpe = detect_multiply(a, b, &ov);
        }
    }
    return ST_OK;
}

// unary_op / math_unary_op (ufunc.rs:3824-3975, 4606-4895): C-contiguous out.
int oracle_unary(int op, const OrArr* a, OrArr* out, int* fpe) {
    int od = oracle_unary_out_dtype(op, a->dtype);
    if (od < 0) return -od;
    int cd = (op == OP_LOGICAL_NOT) ? D_BOOL : od;
    Buf c = cast_to(a, cd);
    int64_t n = c.size();
    void* o = out->data;
    for (int64_t i = 0; i < n; ++i) {
        switch (op) {
            case OP_LOGICAL_NOT: ((uint8_t*)o)[i] = !atc<uint8_t>(c, i); break;
            case OP_NEGATIVE: case OP_ABSOLUTE: case OP_INVERT: {
                bool neg = op == OP_NEGATIVE, ab = op == OP_ABSOLUTE;
                switch (cd) {
                    case D_BOOL: ((uint8_t*)o)[i] = ab ? atc<uint8_t>(c, i) : !atc<uint8_t>(c, i); break;
                    case D_I8: { int8_t x = atc<int8_t>(c, i); ((int8_t*)o)[i] = neg ? w_sub<int8_t>(0, x) : ab ? (x < 0 ? w_sub<int8_t>(0, x) : x) : (int8_t)~x; } break;
                    case D_I16: { int16_t x = atc<int16_t>(c, i); ((int16_t*)o)[i] = neg ? w_sub<int16_t>(0, x) : ab ? (x < 0 ? w_sub<int16_t>(0, x) : x) : (int16_t)~x; } break;
                    case D_I32: { int32_t x = atc<int32_t>(c, i); ((int32_t*)o)[i] = neg ? w_sub<int32_t>(0, x) : ab ? (x < 0 ? w_sub<int32_t>(0, x) : x) : (int32_t)~x; } break;
                    case D_I64: { int64_t x = atc<int64_t>(c, i); ((int64_t*)o)[i] = neg ? w_sub<int64_t>(0, x) : ab ? (x < 0 ? w_sub<int64_t>(0, x) : x) : (int64_t)~x; } break;
                    case D_U8: { uint8_t x = atc<uint8_t>(c, i); ((uint8_t*)o)[i] = neg ? (uint8_t)(0u - x) : ab ? x : (uint8_t)~x; } break;
                    case D_U16: { uint16_t x = atc<uint16_t>(c, i); ((uint16_t*)o)[i] = neg ? (uint16_t)(0u - x) : ab ? x : (uint16_t)~x; } break;
                    case D_U32: { uint32_t x = atc<uint32_t>(c, i); ((uint32_t*)o)[i] = neg ? (uint32_t)(0u - x) : ab ? x : (uint32_t)~x; } break;
                    case D_U64: { uint64_t x = atc<uint64_t>(c, i); ((uint64_t*)o)[i] = neg ? (uint64_t)(0ull - x) : ab ? x : (uint64_t)~x; } break;
                    case D_F16: { uint16_t x = atc<uint16_t>(c, i); ((uint16_t*)o)[i] = neg ? (uint16_t)(x ^ 0x8000) : (uint16_t)(x & 0x7FFF); } break;
                    case D_F32: { uint32_t x = fbits(atc<float>(c, i)); ((uint32_t*)o)[i] = neg ? (x ^ 0x80000000u) : (x & 0x7FFFFFFFu); } break;
                    case D_F64: { uint64_t x = dbits(atc<double>(c, i)); ((uint64_t*)o)[i] = neg ? (x ^ 0x8000000000000000ull) : (x & 0x7FFFFFFFFFFFFFFFull); } break;
                }
            } break;
            case OP_SQRT: case OP_EXP: case OP_LOG: case OP_SIN: case OP_COS: {
                auto f32 = [&](float x) -> float {
                    switch (op) {
                        case OP_SQRT: return o_sqrt(x);
                        case OP_EXP: return expf(x);
                        case OP_LOG: return logf(x);
                        case OP_COS: return cosf(x);
                        default: return sinf(x);
                    }
                };
                auto f64 = [&](double x) -> double {
                    switch (op) {
                        case OP_SQRT: return o_sqrt(x);
                        case OP_EXP: return exp(x);
                        case OP_LOG: return log(x);
                        case OP_COS: return cos(x);
                        default: return sin(x);
                    }
                };
                if (cd == D_F16) ((uint16_t*)o)[i] = f2h(f32(h2f(atc<uint16_t>(c, i))));
                else if (cd == D_F32) ((float*)o)[i] = f32(atc<float>(c, i));
                else ((double*)o)[i] = f64(atc<double>(c, i));
            } break;
        }
    }
    if (fpe) {
        *fpe = 0;
        if (op == OP_SQRT || op == OP_LOG) {
            auto v = to_f64_lossy(a);
            bool neg = false, zero = false;
            for (double x : v) { if (x < 0.0) neg = true; if (x == 0.0) zero = true; }
            if (neg) *fpe = FPE_INVALID;
            else if (op == OP_LOG && zero) *fpe = FPE_DIVIDE;
        }
    }
    return ST_OK;
}

// reduce_axis (ufunc.rs:7634-7825). `axes` sorted and normalized; `cd` the
// compute dtype (from oracle_reduce_compute_dtype or a dtype= override);
// `initial` a 0-d array or NULL; `mask` a where= array already broadcastable
// to a's shape (any dtype; it is cast to bool) or NULL. Output: C order over
// the kept axes (the natural result before relayout_for_reduction).
int oracle_reduce(int op, const OrArr* a, int naxes, const int32_t* axes, int cd,
                  const OrArr* initial, const OrArr* mask, OrArr* out) {
    if (is_compare(op) && a->dtype != D_BOOL) return ST_NO_LOOP;
    if (naxes > 1 && (op == OP_SUBTRACT || op == OP_DIVIDE || op == OP_FLOOR_DIVIDE || is_shift(op))) return ST_VALUE;
    std::vector<int> red(axes, axes + naxes);
    // a is cast (C-contiguous copy) only when its dtype differs (7708-7712)
    Buf cast;
    OrArr src = *a;
    if (a->dtype != cd) { cast = cast_to(a, cd); src = view_of(cast); }
    uint8_t init[8] = {0};
    const uint8_t* initp = nullptr;
    if (initial) {
        OrArr iv; memset(&iv, 0, sizeof(iv)); iv.dtype = cd; iv.ndim = 0; iv.data = init;
        oracle_cast(initial, &iv);
        initp = init;
    }
    Buf mcast;
    OrArr mview;
    const OrArr* mp = nullptr;
    if (mask) { mcast = cast_to(mask, D_BOOL); mview = view_of(mcast); mp = &mview; }
    bool pairwise = (op == OP_ADD) && kind_of(cd) == K_FLOAT;
    bool ordered = (op == OP_MULTIPLY) && kind_of(cd) == K_FLOAT;
    void* o = out->data;
    switch (cd) {
        case D_BOOL: return reduce_typed<uint8_t>(op, &src, red, cd, Fold<uint8_t>{op}, false, false, initp, mp, o);
        case D_I8: return reduce_typed<int8_t>(op, &src, red, cd, Fold<int8_t>{op}, false, false, initp, mp, o);
        case D_I16: return reduce_typed<int16_t>(op, &src, red, cd, Fold<int16_t>{op}, false, false, initp, mp, o);
        case D_I32: return reduce_typed<int32_t>(op, &src, red, cd, Fold<int32_t>{op}, false, false, initp, mp, o);
        case D_I64: return reduce_typed<int64_t>(op, &src, red, cd, Fold<int64_t>{op}, false, false, initp, mp, o);
        case D_U8: return reduce_typed<uint8_t>(op, &src, red, cd, [op](uint8_t x, uint8_t y) { return int_same<uint8_t>(op, x, y); }, false, false, initp, mp, o);
        case D_U16: return reduce_typed<uint16_t>(op, &src, red, cd, Fold<uint16_t>{op}, false, false, initp, mp, o);
        case D_U32: return reduce_typed<uint32_t>(op, &src, red, cd, Fold<uint32_t>{op}, false, false, initp, mp, o);
        case D_U64: return reduce_typed<uint64_t>(op, &src, red, cd, Fold<uint64_t>{op}, false, false, initp, mp, o);
        case D_F32: return reduce_typed<float>(op, &src, red, cd, Fold<float>{op}, pairwise, ordered, initp, mp, o);
        case D_F64: return reduce_typed<double>(op, &src, red, cd, Fold<double>{op}, pairwise, ordered, initp, mp, o);
        case D_F16: {
            if (op == OP_ADD || op == OP_MULTIPLY || op == OP_SUBTRACT || op == OP_DIVIDE) {
                std::vector<int64_t> shape = shape_of(&src), strides = strides_of(&src);
                uint16_t init16 = 0; memcpy(&init16, init, 2);
                if (mp) {
                    bool has = initp != nullptr;
                    uint16_t seed = init16;
                    if (!has) {
                        if (op == OP_ADD) { has = true; seed = 0; }
                        else if (op == OP_MULTIPLY) { has = true; seed = 0x3C00; }
                    }
                    if (!has) return ST_VALUE;
                    std::vector<int64_t> mst = bstrides(shape_of(mp), strides_of(mp), shape);
                    reduce_masked_f16(shape, strides, src.offset, (const uint16_t*)src.data, mst, mp->offset, (const uint8_t*)mp->data, red, op, seed, (uint16_t*)o);
                    return ST_OK;
                }
                int64_t group = 1; for (int x : red) group *= shape[x];
                if (group == 0) {
                    bool has = initp != nullptr; uint16_t v = init16;
                    if (!has) { if (op == OP_ADD) { has = true; v = 0; } else if (op == OP_MULTIPLY) { has = true; v = 0x3C00; } }
                    if (!has) return ST_VALUE;
                    int64_t osz = 1; for (int x = 0; x < (int)shape.size(); ++x) if (!contains(red, x)) osz *= shape[x];
                    for (int64_t i = 0; i < std::max<int64_t>(osz, 1); ++i) ((uint16_t*)o)[i] = v;
                    return ST_OK;
                }
                return reduce_f16(shape, strides, src.offset, (const uint16_t*)src.data, red, op, initp != nullptr, init16, (uint16_t*)o);
            }
            return reduce_typed<uint16_t>(op, &src, red, cd, FoldH{op}, false, false, initp, mp, o);
        }
    }
    return ST_UNSUPPORTED;
}

// argext (ufunc.rs:8131-8206) over one axis; out int64 C order over kept axes.
int oracle_argext(int is_max, const OrArr* a, int axis, OrArr* out) {
    std::vector<int64_t> shape = shape_of(a), strides = strides_of(a);
    std::vector<int64_t> rs, rst, ks, kst;
    if (shape.empty()) { rs.push_back(1); rst.push_back(0); }
    for (int x = 0; x < (int)shape.size(); ++x) {
        if (x == axis) { rs.push_back(shape[x]); rst.push_back(strides[x]); }
        else { ks.push_back(shape[x]); kst.push_back(strides[x]); }
    }
    int64_t group = 1; for (auto s : rs) group *= s;
    if (group == 0) return ST_VALUE;
    int64_t* po = (int64_t*)out->data;
    Kind k = kind_of(a->dtype);
    auto better = [&](const Val& v, const Val& b) -> bool {
        if (k == K_FLOAT) {
            double x = v.d == D_F16 ? h2d(v.h) : v.d == D_F32 ? (double)v.f : v.g;
            double y = b.d == D_F16 ? h2d(b.h) : b.d == D_F32 ? (double)b.f : b.g;
            bool c = is_max ? (x > y) : (x < y);
            return c || (x != x && !(y != y));
        }
        if (k == K_BOOL) return is_max ? (v.b > b.b) : (v.b < b.b);
        if (k == K_INT) return is_max ? (v.i > b.i) : (v.i < b.i);
        return is_max ? (v.u > b.u) : (v.u < b.u);
    };
    auto seq = [&](int64_t base) -> int64_t {
        bool first = true; Val best; int64_t bi = 0, i = 0;
        nd_iter(rs, rst, [&](int64_t o) {
            Val v = load(a, base + o);
            if (first) { best = v; first = false; }
            else if (better(v, best)) { best = v; bi = i; }
            i++;
        });
        return bi;
    };
    int64_t kk = 0;
    if (ks.empty()) { po[0] = seq(0); return ST_OK; }
    nd_iter(ks, kst, [&](int64_t ko) { po[kk++] = seq(ko); });
    return ST_OK;
}

// Pairwise sum of a contiguous f32/f64 vector, used by the timed CPU
// baseline; identical fold to reduce over a 1-D array's only axis.
double oracle_pairwise_f64(const double* x, int64_t n) {
    return pairwise_sum<double>([&](int64_t i) { return x[i]; }, 0, n, [](double p, double q) { return fadd(p, q); }, 8);
}

}  // extern "C"
