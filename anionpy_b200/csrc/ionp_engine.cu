// Host engine of the B200 ufunc path: error reporting, dtype and layout
// rules, the caching device allocator, element-wise planning (dim merging,
// vector-path selection, FPE detector placement) and the element-wise
// C-ABI entry points.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include "ionp_internal.h"
#include <nvtx3/nvToolsExt.h>
#include "ionp_host.h"
#include "ionp_scalar.cuh"

namespace ionp {

// ===========================================================================
// errors (ionp-core/src/error.rs:8-100 message shapes)
// ===========================================================================
static thread_local std::string g_last_error;

int32_t set_err(int32_t status, const std::string& msg) {
    g_last_error = msg;
    return status;
}
int32_t cuda_err(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return IONP_OK;
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return set_err(e == cudaErrorMemoryAllocation ? IONP_ERR_OOM : IONP_ERR_CUDA, m);
}
// numpy's bespoke shape formatter: "(3,)" / "(4,5)" (error.rs:59-69)
std::string fmt_shape(const int64_t* shape, int nd) {
    std::ostringstream s;
    s << "(";
    for (int i = 0; i < nd; ++i) {
        if (i) s << ",";
        s << shape[i];
    }
    if (nd == 1) s << ",";
    s << ")";
    return s.str();
}
const char* op_name(int op) {
    switch (op) {
        case OP_ADD: return "add"; case OP_SUBTRACT: return "subtract"; case OP_MULTIPLY: return "multiply";
        case OP_DIVIDE: return "divide"; case OP_MAXIMUM: return "maximum"; case OP_MINIMUM: return "minimum";
        case OP_GREATER: return "greater"; case OP_GREATER_EQUAL: return "greater_equal"; case OP_LESS: return "less";
        case OP_LESS_EQUAL: return "less_equal"; case OP_EQUAL: return "equal"; case OP_NOT_EQUAL: return "not_equal";
        case OP_LOGICAL_AND: return "logical_and"; case OP_LOGICAL_OR: return "logical_or"; case OP_LOGICAL_XOR: return "logical_xor";
        case OP_BITWISE_AND: return "bitwise_and"; case OP_BITWISE_OR: return "bitwise_or"; case OP_BITWISE_XOR: return "bitwise_xor";
        case OP_FLOOR_DIVIDE: return "floor_divide"; case OP_LEFT_SHIFT: return "left_shift"; case OP_RIGHT_SHIFT: return "right_shift";
        case OP_REMAINDER: return "remainder"; case OP_FMOD: return "fmod";
        case OP_NEGATIVE: return "negative"; case OP_ABSOLUTE: return "absolute"; case OP_INVERT: return "invert";
        case OP_LOGICAL_NOT: return "logical_not"; case OP_SQRT: return "sqrt"; case OP_EXP: return "exp";
        case OP_LOG: return "log"; case OP_SIN: return "sin"; case OP_COS: return "cos";
    }
    return "?";
}

// ===========================================================================
// dtype rules (ionp-core/src/dtype.rs:297-845, ufunc.rs:1101-2168)
// ===========================================================================
bool dt_valid(int d) { return d >= 0 && d < DT_COUNT; }
int dt_bytes(int d) { return dt_size(d); }
const char* dt_name(int d) {
    static const char* n[] = {"bool", "int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64", "float16", "float32", "float64"};
    return dt_valid(d) ? n[d] : "?";
}
enum Kind { KB, KI, KU, KF };
static Kind kind(int d) { return d == DT_BOOL ? KB : dt_is_sint(d) ? KI : dt_is_uint(d) ? KU : KF; }
static int bits(int d) { return d == DT_BOOL ? 8 : dt_size(d) * 8; }
static int sint_of(int b) { return b == 8 ? DT_I8 : b == 16 ? DT_I16 : b == 32 ? DT_I32 : DT_I64; }
static int uint_of(int b) { return b == 8 ? DT_U8 : b == 16 ? DT_U16 : b == 32 ? DT_U32 : DT_U64; }
static int float_of(int b) { return b <= 16 ? DT_F16 : b == 32 ? DT_F32 : DT_F64; }
static int float_bits_for_int(int b) { return b == 8 ? 16 : b == 16 ? 32 : 64; }

// promote_dtype: numpy's promote_types table for two array dtypes
int promote(int a, int b) {
    if (a == b) return a;
    Kind ka = kind(a), kb = kind(b);
    if (ka == KB) return b;
    if (kb == KB) return a;
    if (ka == KI && kb == KI) return sint_of(std::max(bits(a), bits(b)));
    if (ka == KU && kb == KU) return uint_of(std::max(bits(a), bits(b)));
    if ((ka == KI && kb == KU) || (ka == KU && kb == KI)) {
        int sb = ka == KI ? bits(a) : bits(b), ub = ka == KU ? bits(a) : bits(b);
        if (ub < sb) return sint_of(sb);
        return ub == 64 ? DT_F64 : sint_of(ub * 2);
    }
    if (ka == KF && kb == KF) return float_of(std::max(bits(a), bits(b)));
    if (kb == KF) return float_of(std::max(float_bits_for_int(bits(a)), bits(b)));
    return float_of(std::max(bits(a), float_bits_for_int(bits(b))));
}

static std::string no_safe_loop(int op) {
    return std::string("ufunc '") + op_name(op) +
           "' not supported for the input types, and the inputs could not be safely coerced to any supported "
           "types according to the casting rule ''safe''";
}

int32_t binary_loop(int op, int a, int b, int* cd, int* rd) {
    if (!dt_valid(a) || !dt_valid(b)) return set_err(IONP_ERR_UNSUPPORTED, "unsupported dtype");
    int p = promote(a, b);
    Kind k = kind(p);
    if (op_is_compare(op)) { *cd = p; *rd = DT_BOOL; return IONP_OK; }
    if (op_is_logical(op)) { *cd = DT_BOOL; *rd = DT_BOOL; return IONP_OK; }
    if (op == OP_REMAINDER || op == OP_FMOD) {  // math_binary_out_dtype, non-float-promoting
        *cd = *rd = (p == DT_BOOL) ? DT_I8 : p;
        return IONP_OK;
    }
    if (op == OP_BITWISE_AND || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) {
        if (k == KF) return set_err(IONP_ERR_TYPE, no_safe_loop(op));
        *cd = *rd = p;
        return IONP_OK;
    }
    if (op == OP_LEFT_SHIFT || op == OP_RIGHT_SHIFT) {
        if (k == KF) return set_err(IONP_ERR_TYPE, no_safe_loop(op));
        *cd = *rd = (p == DT_BOOL) ? DT_I8 : p;
        return IONP_OK;
    }
    if (op == OP_SUBTRACT && p == DT_BOOL)
        return set_err(IONP_ERR_TYPE,
                       "numpy boolean subtract, the `-` operator, is not supported, use the bitwise_xor, the `^` "
                       "operator, or the logical_xor function instead.");
    if (op == OP_DIVIDE) { *cd = *rd = (k == KF) ? p : DT_F64; return IONP_OK; }
    if (op == OP_FLOOR_DIVIDE) { *cd = *rd = (p == DT_BOOL) ? DT_I8 : p; return IONP_OK; }
    if (op == OP_ADD || op == OP_MULTIPLY || op == OP_MAXIMUM || op == OP_MINIMUM || op == OP_SUBTRACT) {
        *cd = *rd = p;
        return IONP_OK;
    }
    return set_err(IONP_ERR_UNSUPPORTED, std::string("op ") + std::to_string(op) + " is not a binary ufunc of this engine");
}

int32_t unary_loop(int op, int a, int* cd, int* rd) {
    if (!dt_valid(a)) return set_err(IONP_ERR_UNSUPPORTED, "unsupported dtype");
    switch (op) {
        case OP_LOGICAL_NOT: *cd = DT_BOOL; *rd = DT_BOOL; return IONP_OK;
        case OP_NEGATIVE:
            if (a == DT_BOOL)
                return set_err(IONP_ERR_TYPE,
                               "The numpy boolean negative, the `-` operator, is not supported, use the `~` operator "
                               "or the logical_not function instead.");
            *cd = *rd = a;
            return IONP_OK;
        case OP_INVERT:
            if (kind(a) == KF) return set_err(IONP_ERR_TYPE, no_safe_loop(op));
            *cd = *rd = a;
            return IONP_OK;
        case OP_ABSOLUTE: *cd = *rd = a; return IONP_OK;
        case OP_SQRT: case OP_EXP: case OP_LOG: case OP_SIN: case OP_COS:
            // math_unary_out_dtype float tiers (ufunc.rs:1705-1712)
            if (a == DT_BOOL || a == DT_I8 || a == DT_U8) *cd = DT_F16;
            else if (a == DT_I16 || a == DT_U16) *cd = DT_F32;
            else if (kind(a) != KF) *cd = DT_F64;
            else *cd = a;
            *rd = *cd;
            return IONP_OK;
    }
    return set_err(IONP_ERR_UNSUPPORTED, std::string("op ") + std::to_string(op) + " is not a unary ufunc of this engine");
}

// reduce_family_compute_dtype (ufunc.rs:2080) + reduce_compute_dtype (2041)
int32_t reduce_cd(int op, int a, int* cd) {
    if (!dt_valid(a)) return set_err(IONP_ERR_UNSUPPORTED, "unsupported dtype");
    Kind k = kind(a);
    if (op_is_compare(op)) {
        if (a != DT_BOOL) return set_err(IONP_ERR_NO_LOOP, std::string("ufunc '") + op_name(op) + "' did not contain a loop with signature matching types");
        *cd = DT_BOOL;
        return IONP_OK;
    }
    if (op_is_logical(op)) { *cd = DT_BOOL; return IONP_OK; }
    if (op == OP_BITWISE_AND || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) {
        if (k == KF) return set_err(IONP_ERR_TYPE, no_safe_loop(op));
        *cd = a;
        return IONP_OK;
    }
    if (op == OP_LEFT_SHIFT || op == OP_RIGHT_SHIFT) {
        if (k == KF) return set_err(IONP_ERR_TYPE, no_safe_loop(op));
        *cd = a == DT_BOOL ? DT_I8 : a;
        return IONP_OK;
    }
    if (op == OP_SUBTRACT && a == DT_BOOL)
        return set_err(IONP_ERR_TYPE,
                       "numpy boolean subtract, the `-` operator, is not supported, use the bitwise_xor, the `^` "
                       "operator, or the logical_xor function instead.");
    if (op == OP_FLOOR_DIVIDE && a == DT_BOOL) { *cd = DT_I8; return IONP_OK; }
    if (op == OP_DIVIDE && k != KF) { *cd = DT_F64; return IONP_OK; }
    if (op == OP_ADD || op == OP_MULTIPLY) {
        if (a == DT_BOOL || k == KI) { *cd = DT_I64; return IONP_OK; }
        if (k == KU) { *cd = DT_U64; return IONP_OK; }
    }
    if (op == OP_ADD || op == OP_MULTIPLY || op == OP_MAXIMUM || op == OP_MINIMUM || op == OP_SUBTRACT ||
        op == OP_DIVIDE || op == OP_FLOOR_DIVIDE) {
        *cd = a;
        return IONP_OK;
    }
    return set_err(IONP_ERR_UNSUPPORTED, std::string("op ") + op_name(op) + " has no reduce in this engine");
}

// can_cast (dtype.rs:823): safe = promote(from, to) == to; same_kind adds
// downcasts within a kind and into a higher kind (never int -> uint, never
// anything -> bool).
bool can_cast(int from, int to, int rule) {
    switch (rule) {
        case IONP_CAST_NO: case IONP_CAST_EQUIV: return from == to;
        case IONP_CAST_UNSAFE: return true;
    }
    bool safe = promote(from, to) == to;
    if (rule == IONP_CAST_SAFE) return safe;
    if (safe) return true;
    Kind kf = kind(from), kt = kind(to);
    switch (kt) {
        case KB: return false;
        case KI: case KU: return (kf == KB || kf == KI || kf == KU) && !(kf == KI && kt == KU);
        case KF: return true;
    }
    return false;
}

// ---- host copy of one scalar cast (initial= values) ------------------------
static double h_h2d(uint16_t h) {
    uint32_t sign = (h & 0x8000u) ? 1 : 0, e = (h >> 10) & 0x1F, m = h & 0x3FF;
    double v;
    if (e == 0x1F) return m ? std::nan("") : (sign ? -INFINITY : INFINITY);
    if (e == 0) v = std::ldexp((double)m, -24);
    else v = std::ldexp((double)(m | 0x400), (int)e - 25);
    return sign ? -v : v;
}
static uint16_t h_d2h(double d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    uint32_t sign = (uint32_t)((b >> 48) & 0x8000u);
    uint32_t ex = (uint32_t)((b >> 52) & 0x7FF);
    uint64_t man = b & 0xFFFFFFFFFFFFFull;
    if (ex == 0x7FF) return (uint16_t)(man == 0 ? (sign | 0x7C00u) : (sign | 0x7E00u | (uint32_t)((man >> 42) & 0x3FFu)));
    if (ex == 0) return (uint16_t)sign;
    int e = (int)ex - 1023;
    if (e > 15) return (uint16_t)(sign | 0x7C00u);
    uint64_t m = man | (1ull << 52);
    if (e >= -14) {
        uint64_t q = m >> 42, rem = m & ((1ull << 42) - 1), half = 1ull << 41;
        if (rem > half || (rem == half && (q & 1))) q++;
        uint32_t he = (uint32_t)(e + 15);
        if (q == 2048) { q = 1024; he++; }
        if (he >= 31) return (uint16_t)(sign | 0x7C00u);
        return (uint16_t)(sign | (he << 10) | (uint32_t)(q & 0x3FFu));
    }
    int shift = 28 - e;
    if (shift > 60) return (uint16_t)sign;
    uint64_t q = m >> shift, rem = m & ((1ull << shift) - 1), half = 1ull << (shift - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    return (uint16_t)(sign | (uint32_t)q);
}
template <class I> static I h_sat(double x) {
    if (x != x) return 0;
    double lo = (double)std::numeric_limits<I>::min(), hi = (double)std::numeric_limits<I>::max();
    if (x <= lo) return std::numeric_limits<I>::min();
    if (x >= hi) return std::numeric_limits<I>::max();
    return (I)x;
}
void host_cast_scalar(const void* src, int sd, void* dst, int dd) {
    // read source as one of: bool/int64/uint64/double(float kinds)
    Kind k = kind(sd);
    int64_t si = 0; uint64_t ui = 0; double fv = 0; bool nz = false; uint16_t hb = 0; float ff = 0; double df = 0;
    switch (sd) {
        case DT_BOOL: ui = *(const uint8_t*)src ? 1 : 0; si = (int64_t)ui; break;
        case DT_I8: si = *(const int8_t*)src; ui = (uint64_t)si; break;
        case DT_I16: si = *(const int16_t*)src; ui = (uint64_t)si; break;
        case DT_I32: si = *(const int32_t*)src; ui = (uint64_t)si; break;
        case DT_I64: si = *(const int64_t*)src; ui = (uint64_t)si; break;
        case DT_U8: ui = *(const uint8_t*)src; si = (int64_t)ui; break;
        case DT_U16: ui = *(const uint16_t*)src; si = (int64_t)ui; break;
        case DT_U32: ui = *(const uint32_t*)src; si = (int64_t)ui; break;
        case DT_U64: ui = *(const uint64_t*)src; si = (int64_t)ui; break;
        case DT_F16: hb = *(const uint16_t*)src; fv = h_h2d(hb); nz = (hb & 0x7FFF) != 0; break;
        case DT_F32: ff = *(const float*)src; fv = ff; nz = ff != 0; break;
        case DT_F64: df = *(const double*)src; fv = df; nz = df != 0; break;
    }
    if (k != KF) {
        bool u = k == KU;
        switch (dd) {
            case DT_BOOL: *(uint8_t*)dst = ui != 0; return;
            case DT_I8: *(int8_t*)dst = (int8_t)ui; return;
            case DT_I16: *(int16_t*)dst = (int16_t)ui; return;
            case DT_I32: *(int32_t*)dst = (int32_t)ui; return;
            case DT_I64: *(int64_t*)dst = (int64_t)ui; return;
            case DT_U8: *(uint8_t*)dst = (uint8_t)ui; return;
            case DT_U16: *(uint16_t*)dst = (uint16_t)ui; return;
            case DT_U32: *(uint32_t*)dst = (uint32_t)ui; return;
            case DT_U64: *(uint64_t*)dst = ui; return;
            case DT_F16: *(uint16_t*)dst = sd == DT_BOOL ? (ui ? 0x3C00 : 0) : h_d2h(u ? (double)ui : (double)si); return;
            case DT_F32: *(float*)dst = u ? (float)ui : (float)si; return;
            case DT_F64: *(double*)dst = u ? (double)ui : (double)si; return;
        }
        return;
    }
    switch (dd) {
        case DT_BOOL: *(uint8_t*)dst = nz; return;
        case DT_I8: *(int8_t*)dst = (int8_t)(uint32_t)h_sat<int32_t>(fv); return;
        case DT_I16: *(int16_t*)dst = (int16_t)(uint32_t)h_sat<int32_t>(fv); return;
        case DT_I32: *(int32_t*)dst = h_sat<int32_t>(fv); return;
        case DT_I64: *(int64_t*)dst = h_sat<int64_t>(fv); return;
        case DT_U8: *(uint8_t*)dst = (uint8_t)(uint32_t)h_sat<int32_t>(fv); return;
        case DT_U16: *(uint16_t*)dst = (uint16_t)(uint32_t)h_sat<int32_t>(fv); return;
        case DT_U32: *(uint32_t*)dst = h_sat<uint32_t>(fv); return;
        case DT_U64: *(uint64_t*)dst = h_sat<uint64_t>(fv); return;
        case DT_F16: *(uint16_t*)dst = sd == DT_F16 ? hb : h_d2h(fv); return;
        case DT_F32: *(float*)dst = sd == DT_F32 ? ff : (float)fv; return;
        case DT_F64: *(double*)dst = fv; return;
    }
}

// ===========================================================================
// arrays
// ===========================================================================
int32_t check_arr(const IonpArr* a, const char* what) {
    if (!a) return set_err(IONP_ERR_INVALID, std::string(what) + " is NULL");
    if (a->ndim < 0 || a->ndim > IONP_MAX_DIMS) return set_err(IONP_ERR_INVALID, std::string(what) + ": ndim out of range");
    if (!dt_valid(a->dtype)) return set_err(IONP_ERR_UNSUPPORTED, std::string(what) + ": dtype not supported by this engine (complex/string)");
    int64_t total = 1;
    for (int i = 0; i < a->ndim; ++i) {
        if (a->shape[i] < 0) return set_err(IONP_ERR_INVALID, std::string(what) + ": negative extent");
        if (a->shape[i] > 0 && total > ((int64_t)1 << 62) / a->shape[i])
            return set_err(IONP_ERR_INVALID, std::string(what) + ": more than 2^62 elements");
        total *= a->shape[i];
    }
    if (total > 0 && a->data == nullptr) return set_err(IONP_ERR_INVALID, std::string(what) + ": NULL data");
    return IONP_OK;
}

bool bcast_strides(const IonpArr* a, int nd, const int64_t* shape, int64_t* out) {
    if (a->ndim > nd) return false;
    int pad = nd - a->ndim;
    for (int i = 0; i < nd; ++i) {
        if (i < pad) { out[i] = 0; continue; }
        int64_t s = a->shape[i - pad];
        if (s == shape[i]) out[i] = (s == 1) ? 0 : a->strides[i - pad];
        else if (s == 1) out[i] = 0;
        else return false;
    }
    return true;
}

static bool bshape2(const IonpArr* a, const IonpArr* b, int* nd, int64_t* out) {
    int n = std::max(a->ndim, b->ndim);
    for (int i = 0; i < n; ++i) {
        int ia = i - (n - a->ndim), ib = i - (n - b->ndim);
        int64_t da = ia < 0 ? 1 : a->shape[ia], db = ib < 0 ? 1 : b->shape[ib];
        if (da == db) out[i] = da;
        else if (da == 1) out[i] = db;
        else if (db == 1) out[i] = da;
        else return false;
    }
    *nd = n;
    return true;
}

// ===========================================================================
// caching device allocator
// ===========================================================================
namespace {
struct Block {
    void* p;
    size_t size;
    cudaStream_t stream;
    cudaEvent_t ev;  // recorded at free time on `stream`
};
// Caching device allocator: one pool per device (its own lock, free list
// and counters). A freed block is cached with an event recorded on the
// freeing stream; a later allocation from another stream waits for that
// event before reuse. On a failed cudaMalloc the device's cached blocks
// are released and the allocation retried once.
struct DevicePool {
    std::mutex mu;
    std::multimap<size_t, Block> free_;   // by size
    uint64_t in_use = 0, cached = 0, peak = 0, mallocs = 0;
};
struct Allocator {
    static constexpr int MAXDEV = 64;
    DevicePool pools[MAXDEV];
    std::mutex used_mu;
    std::map<void*, std::pair<int, Block>> used_;   // pointer -> (device, block)

    static size_t round(size_t b) {
        if (b == 0) b = 1;
        if (b <= (1u << 20)) return (b + 511) & ~(size_t)511;
        return (b + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
    }
    static int32_t current_device(int* dev) {
        if (cudaGetDevice(dev) != cudaSuccess) return cuda_err(cudaGetLastError(), "cudaGetDevice");
        if (*dev < 0 || *dev >= MAXDEV) return set_err(IONP_ERR_INVALID, "device ordinal out of the allocator's range");
        return IONP_OK;
    }
    int32_t alloc(void** out, size_t bytes, cudaStream_t s) {
        int dev;
        int32_t st = current_device(&dev);
        if (st) return st;
        const size_t sz = round(bytes);
        DevicePool& P = pools[dev];
        Block got{nullptr, 0, s, nullptr};
        {
            std::lock_guard<std::mutex> g(P.mu);
            auto it = P.free_.lower_bound(sz);
            if (it != P.free_.end() && it->first <= sz + sz / 8) {
                got = it->second;
                if (got.stream != s && got.ev) cudaStreamWaitEvent(s, got.ev, 0);
                P.free_.erase(it);
                P.cached -= got.size;
                got.stream = s;
                P.in_use += got.size;
                P.peak = std::max(P.peak, P.in_use);
            }
        }
        if (!got.p) {
            void* p = nullptr;
            cudaError_t e = cudaMalloc(&p, sz);
            if (e != cudaSuccess) {
                cudaGetLastError();
                trim_device(dev);
                e = cudaMalloc(&p, sz);
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    return set_err(IONP_ERR_OOM, "device allocation of " + std::to_string(sz) + " bytes failed: " + cudaGetErrorString(e));
                }
            }
            got = Block{p, sz, s, nullptr};
            std::lock_guard<std::mutex> g(P.mu);
            P.mallocs++;
            P.in_use += sz;
            P.peak = std::max(P.peak, P.in_use);
        }
        {
            std::lock_guard<std::mutex> g(used_mu);
            used_[got.p] = {dev, got};
        }
        *out = got.p;
        return IONP_OK;
    }
    int32_t release(void* p, cudaStream_t s) {
        if (!p) return IONP_OK;
        int dev;
        Block b;
        {
            std::lock_guard<std::mutex> g(used_mu);
            auto it = used_.find(p);
            if (it == used_.end()) return set_err(IONP_ERR_INVALID, "ionp_free: pointer not from ionp_alloc");
            dev = it->second.first;
            b = it->second.second;
            used_.erase(it);
        }
        int cur = dev;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);   // the event lives on the block's device
        if (!b.ev) cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming);
        b.stream = s;
        cudaEventRecord(b.ev, s);
        if (cur != dev) cudaSetDevice(cur);
        DevicePool& P = pools[dev];
        std::lock_guard<std::mutex> g(P.mu);
        P.in_use -= b.size;
        P.free_.insert({b.size, b});
        P.cached += b.size;
        return IONP_OK;
    }
    void trim_device(int dev) {
        DevicePool& P = pools[dev];
        std::lock_guard<std::mutex> g(P.mu);
        int cur = dev;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);
        for (auto& kv : P.free_) {
            if (kv.second.ev) { cudaEventSynchronize(kv.second.ev); cudaEventDestroy(kv.second.ev); }
            cudaFree(kv.second.p);
        }
        if (cur != dev) cudaSetDevice(cur);
        P.free_.clear();
        P.cached = 0;
    }
    void trim_all() {
        for (int d = 0; d < MAXDEV; ++d) {
            bool any;
            {
                std::lock_guard<std::mutex> g(pools[d].mu);
                any = !pools[d].free_.empty();
            }
            if (any) trim_device(d);
        }
    }
};
Allocator& allocator() {
    static Allocator* a = new Allocator();  // lives until exit; never torn down under a live context
    return *a;
}
std::atomic<uint64_t> g_launches{0};
}  // namespace

void count_launch(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }

static bool nvtx_enabled() {
    static const bool on = [] {
        const char* e = getenv("IONP_NVTX");
        return e && e[0] == '1';
    }();
    return on;
}
NvtxRange::NvtxRange(const char* name) : on(nvtx_enabled()) {
    if (on) nvtxRangePushA(name);
}
NvtxRange::~NvtxRange() {
    if (on) nvtxRangePop();
}

int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return 148; }
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = 148;  // a B200's count, for planning only
    }
    cache[dev].store(n, std::memory_order_relaxed);
    return n;
}

void* scratch_alloc(size_t bytes, cudaStream_t s) {
    void* p = nullptr;
    if (allocator().alloc(&p, bytes, s) != IONP_OK) return nullptr;
    return p;
}
void scratch_free(void* p, cudaStream_t s) { allocator().release(p, s); }

static std::mutex g_err_mu;
static uint32_t* g_err_word[256] = {nullptr};

uint32_t* async_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return nullptr;
    std::lock_guard<std::mutex> g(g_err_mu);
    if (!g_err_word[dev]) {
        void* p = nullptr;
        if (cudaMalloc(&p, 256) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        if (cudaMemset(p, 0, 256) != cudaSuccess) { cudaFree(p); cudaGetLastError(); return nullptr; }
        g_err_word[dev] = (uint32_t*)p;
    }
    return g_err_word[dev];
}

int32_t check_async_error() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return IONP_OK;
    uint32_t* w;
    {
        std::lock_guard<std::mutex> g(g_err_mu);
        w = g_err_word[dev];
    }
    if (!w) return IONP_OK;
    uint32_t v = 0;
    if (cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return cuda_err(cudaGetLastError(), "error word read");
    if (!v) return IONP_OK;
    cudaMemset(w, 0, sizeof(uint32_t));
    return set_err(IONP_ERR_TIMEOUT, "a kernel's bounded wait for a bulk copy gave up; its results are incomplete");
}

static thread_local uint32_t* t_pinned_flag = nullptr;

int32_t FlagWord::open(cudaStream_t st) {
    s = st;
    d = (uint32_t*)scratch_alloc(256, s);
    if (!d) return IONP_ERR_OOM;
    return cuda_err(cudaMemsetAsync(d, 0, sizeof(uint32_t), s), "fpe flag reset");
}
int32_t FlagWord::read(uint32_t* host) {
    if (!t_pinned_flag) {
        if (cudaMallocHost(&t_pinned_flag, 64) != cudaSuccess) return cuda_err(cudaGetLastError(), "pinned flag");
    }
    int32_t st = cuda_err(cudaMemcpyAsync(t_pinned_flag, d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "fpe flag read");
    if (st) return st;
    st = cuda_err(cudaStreamSynchronize(s), "fpe flag sync");
    if (st) return st;
    *host = *t_pinned_flag;
    return IONP_OK;
}
int32_t FlagWord::read_async(uint32_t* host) {
    return cuda_err(cudaMemcpyAsync(host, d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "fpe flag copy");
}
FlagWord::~FlagWord() {
    if (d) scratch_free(d, s);
}

// ===========================================================================
// element-wise planning
// ===========================================================================
// Drop unit dims, order by |output stride| (outermost first), and merge
// neighbours whose strides chain for every operand.
MergeOut merge_dims(const MergeIn& in) {
    MergeOut r;
    int idx[IONP_MAX_DIMS];
    int n = 0;
    for (int i = 0; i < in.nd; ++i)
        if (in.shape[i] != 1) idx[n++] = i;
    std::stable_sort(idx, idx + n, [&](int x, int y) { return std::llabs(in.st[0][x]) > std::llabs(in.st[0][y]); });
    r.nd = 0;
    for (int k = 0; k < n; ++k) {
        int i = idx[k];
        if (r.nd > 0) {
            int j = r.nd - 1;
            bool ok = true;
            // dim i becomes the new inner dim; outer (j) merges if st_j == st_i * shape_i
            for (int o = 0; o < in.nops; ++o)
                if (r.st[o][j] != in.st[o][i] * in.shape[i]) { ok = false; break; }
            if (ok) {
                r.shape[j] *= in.shape[i];
                for (int o = 0; o < in.nops; ++o) r.st[o][j] = in.st[o][i];
                continue;
            }
        }
        r.shape[r.nd] = in.shape[i];
        for (int o = 0; o < in.nops; ++o) r.st[o][r.nd] = in.st[o][i];
        r.nd++;
    }
    if (r.nd == 0) {
        r.nd = 1;
        r.shape[0] = 1;
        for (int o = 0; o < in.nops; ++o) r.st[o][0] = 0;
    }
    return r;
}

namespace {

// Whether the reference's flat `x[i % len_x]` pairing (fpe.rs) equals true
// broadcasting for operand `a` against the broadcast shape: a's shape must be
// a trailing slice of it (after leading ones).
bool trailing_aligned(const IonpArr* a, int nd, const int64_t* shape) {
    int pad = nd - a->ndim;
    int k = 0;
    while (k < a->ndim && a->shape[k] == 1) ++k;
    for (int i = k; i < a->ndim; ++i)
        if (a->shape[i] != shape[i + pad]) return false;
    return true;
}

bool ranges_overlap(const IonpArr* x, const IonpArr* y) {
    if (numel(x) == 0 || numel(y) == 0) return false;
    auto range = [](const IonpArr* a, int64_t* lo, int64_t* hi) {
        int64_t l = a->offset, h = a->offset;
        for (int i = 0; i < a->ndim; ++i) {
            int64_t e = (a->shape[i] - 1) * a->strides[i];
            if (e < 0) l += e; else h += e;
        }
        int b = dt_bytes(a->dtype);
        *lo = (int64_t)(uintptr_t)a->data + l * b;
        *hi = (int64_t)(uintptr_t)a->data + (h + 1) * b;
    };
    int64_t l1, h1, l2, h2;
    range(x, &l1, &h1);
    range(y, &l2, &h2);
    return l1 < h2 && l2 < h1;
}
// In-place is safe when the operand is read at exactly the element each
// thread writes.
bool same_layout(const IonpArr* o, const IonpArr* x, const int64_t* xb) {
    if (o->data != x->data || dt_bytes(o->dtype) != dt_bytes(x->dtype) || o->offset != x->offset) return false;
    for (int i = 0; i < o->ndim; ++i)
        if (o->shape[i] != 1 && xb[i] != o->strides[i]) return false;
    return true;
}

int32_t launch_ew(bool binary, int op, int cd, int rd, const IonpArr* a, const IonpArr* b, IonpArr* out,
                  const IonpArr* where, uint32_t* dflags, bool fpe_inkernel, cudaStream_t s) {
    const int nd = out->ndim;
    MergeIn mi;
    mi.nd = nd;
    mi.nops = 4;
    for (int i = 0; i < nd; ++i) { mi.shape[i] = out->shape[i]; mi.st[0][i] = out->strides[i]; }
    if (!bcast_strides(a, nd, out->shape, mi.st[1]))
        return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(a->shape, a->ndim) + " " + fmt_shape(out->shape, nd) + " ");
    if (binary) {
        if (!bcast_strides(b, nd, out->shape, mi.st[2]))
            return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(b->shape, b->ndim) + " " + fmt_shape(out->shape, nd) + " ");
    } else {
        for (int i = 0; i < nd; ++i) mi.st[2][i] = 0;
    }
    if (where) {
        if (!bcast_strides(where, nd, out->shape, mi.st[3]))
            return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(where->shape, where->ndim) + " " + fmt_shape(out->shape, nd) + " ");
    } else {
        for (int i = 0; i < nd; ++i) mi.st[3][i] = 0;
    }
    MergeOut mo = merge_dims(mi);
    int64_t n = numel(out);
    if (n == 0) return IONP_OK;

    auto make_desc = [&](int dims, const int64_t* shape, const int64_t (*st)[IONP_MAX_DIMS], int64_t off_o, int64_t off_a,
                         int64_t off_b, int64_t off_m) {
        EwDesc d;
        memset(&d, 0, sizeof(d));
        d.nd = dims;
        d.n = 1;
        for (int i = 0; i < dims; ++i) {
            d.shape[i] = shape[i];
            d.n *= shape[i];
            d.so[i] = st[0][i];
            d.a.st[i] = st[1][i];
            d.b.st[i] = st[2][i];
            d.m.st[i] = st[3][i];
        }
        d.o = (char*)elem_ptr(out) + off_o * dt_bytes(out->dtype);
        d.odt = out->dtype;
        d.a.p = elem_ptr(a) + off_a * dt_bytes(a->dtype);
        d.a.dt = a->dtype;
        if (binary) { d.b.p = elem_ptr(b) + off_b * dt_bytes(b->dtype); d.b.dt = b->dtype; }
        else { d.b.p = d.a.p; d.b.dt = a->dtype; }
        if (where) { d.m.p = elem_ptr(where) + off_m; d.m.dt = DT_BOOL; }
        return d;
    };

    if (mo.nd <= EW_MAXD) {
        const int64_t(*st)[IONP_MAX_DIMS] = mo.st;
        EwDesc d = make_desc(mo.nd, mo.shape, st, 0, 0, 0, 0);
        ContigInfo ci{false, false, false};
        if (mo.nd == 1 && !where && mo.st[0][0] == 1 && a->dtype == cd && (!binary || b->dtype == cd) && out->dtype == rd) {
            bool a_ok = mo.st[1][0] == 1 || mo.st[1][0] == 0;
            bool b_ok = !binary || mo.st[2][0] == 1 || mo.st[2][0] == 0;
            bool al = ((uintptr_t)d.o % 16 == 0) && (mo.st[1][0] == 0 || (uintptr_t)d.a.p % 16 == 0) &&
                      (!binary || mo.st[2][0] == 0 || (uintptr_t)d.b.p % 16 == 0);
            if (a_ok && b_ok && al) {
                ci.ok = true;
                ci.a_scalar = mo.st[1][0] == 0;
                ci.b_scalar = binary && mo.st[2][0] == 0;
            }
        }
        uint32_t* f = fpe_inkernel ? dflags : nullptr;
        cudaError_t e = binary ? launch_binary(op, cd, d, ci, f, s) : launch_unary(op, cd, d, ci, f, s);
        return cuda_err(e, binary ? "binary launch" : "unary launch");
    }
    // more than 4 merged dims: one launch per index of the leading dims
    int lead = mo.nd - EW_MAXD;
    int64_t nlead = 1;
    for (int i = 0; i < lead; ++i) nlead *= mo.shape[i];
    int64_t tail_st[4][IONP_MAX_DIMS];
    for (int o = 0; o < 4; ++o)
        for (int i = 0; i < EW_MAXD; ++i) tail_st[o][i] = mo.st[o][lead + i];
    for (int64_t q = 0; q < nlead; ++q) {
        int64_t rem = q, off[4] = {0, 0, 0, 0};
        for (int i = lead - 1; i >= 0; --i) {
            int64_t id = rem % mo.shape[i];
            rem /= mo.shape[i];
            for (int o = 0; o < 4; ++o) off[o] += id * mo.st[o][i];
        }
        EwDesc d = make_desc(EW_MAXD, mo.shape + lead, tail_st, off[0], off[1], off[2], off[3]);
        ContigInfo ci{false, false, false};
        uint32_t* f = fpe_inkernel ? dflags : nullptr;
        cudaError_t e = binary ? launch_binary(op, cd, d, ci, f, s) : launch_unary(op, cd, d, ci, f, s);
        if (e != cudaSuccess) return cuda_err(e, "element-wise launch");
    }
    return IONP_OK;
}

}  // namespace
}  // namespace ionp

using namespace ionp;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int32_t ionp_last_error_message(char* buf, size_t len) {
    if (!buf || len == 0) return IONP_ERR_INVALID;
    size_t n = std::min(len - 1, g_last_error.size());
    memcpy(buf, g_last_error.data(), n);
    buf[n] = 0;
    return IONP_OK;
}
uint64_t ionp_launch_count(void) { return g_launches.load(); }

int32_t ionp_promote(int32_t a, int32_t b, int32_t* out) {
    if (!dt_valid(a) || !dt_valid(b) || !out) return set_err(IONP_ERR_INVALID, "bad dtype");
    *out = promote(a, b);
    return IONP_OK;
}
int32_t ionp_binary_out_dtype(int32_t op, int32_t a, int32_t b, int32_t* out) {
    int cd, rd;
    int32_t st = binary_loop(op, a, b, &cd, &rd);
    if (st == IONP_OK && out) *out = rd;
    return st;
}
int32_t ionp_unary_out_dtype(int32_t op, int32_t a, int32_t* out) {
    int cd, rd;
    int32_t st = unary_loop(op, a, &cd, &rd);
    if (st == IONP_OK && out) *out = rd;
    return st;
}
int32_t ionp_reduce_compute_dtype(int32_t op, int32_t a, int32_t* out) {
    int cd;
    int32_t st = reduce_cd(op, a, &cd);
    if (st == IONP_OK && out) *out = cd;
    return st;
}
int32_t ionp_can_cast(int32_t from, int32_t to, int32_t rule, int32_t* out) {
    if (!dt_valid(from) || !dt_valid(to) || !out) return set_err(IONP_ERR_INVALID, "bad dtype");
    *out = can_cast(from, to, rule) ? 1 : 0;
    return IONP_OK;
}

int32_t ionp_alloc(void** ptr, size_t bytes, IonpStream stream) {
    if (!ptr) return set_err(IONP_ERR_INVALID, "ionp_alloc: NULL out pointer");
    return allocator().alloc(ptr, bytes, (cudaStream_t)stream);
}
int32_t ionp_free(void* ptr, IonpStream stream) { return allocator().release(ptr, (cudaStream_t)stream); }
int32_t ionp_alloc_stats(uint64_t* s) {
    if (!s) return set_err(IONP_ERR_INVALID, "ionp_alloc_stats: NULL stats pointer");
    int dev;
    int32_t st = Allocator::current_device(&dev);
    if (st) return st;
    DevicePool& P = allocator().pools[dev];
    std::lock_guard<std::mutex> g(P.mu);
    s[0] = P.in_use; s[1] = P.cached; s[2] = P.peak; s[3] = P.mallocs;
    return IONP_OK;
}
int32_t ionp_alloc_trim(void) {
    allocator().trim_all();
    return IONP_OK;
}

static int32_t binary_call(int32_t op, const IonpArr* a, const IonpArr* b, IonpArr* out, const IonpArr* where,
                           uint32_t* fpe, bool nowait, IonpStream stream) {
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(b, "b")) || (st = check_arr(out, "out"))) return st;
    if (where && (st = check_arr(where, "where"))) return st;
    if (where && where->dtype != DT_BOOL) return set_err(IONP_ERR_TYPE, "where= mask must be boolean");
    cudaStream_t s = (cudaStream_t)stream;
    int cd, rd;
    // the dtype loop is resolved before shapes are checked (ufunc.rs:3636-3640)
    if ((st = binary_loop(op, a->dtype, b->dtype, &cd, &rd))) return st;
    int bnd;
    int64_t bsh[IONP_MAX_DIMS];
    if (!bshape2(a, b, &bnd, bsh))
        return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(a->shape, a->ndim) + " " + fmt_shape(b->shape, b->ndim) + " ");
    {
        // out must hold the broadcast result (it may broadcast it up)
        IonpArr tmp;
        tmp.ndim = bnd;
        for (int i = 0; i < bnd; ++i) tmp.shape[i] = bsh[i];
        int64_t dummy[IONP_MAX_DIMS];
        if (!bcast_strides(&tmp, out->ndim, out->shape, dummy))
            return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(bsh, bnd) + " " + fmt_shape(out->shape, out->ndim) + " ");
    }
    // FPE detector placement (fpe_check_after_call, lib.rs:9077-9138)
    int fkind = 0;
    if (op == OP_DIVIDE || op == OP_FLOOR_DIVIDE) fkind = 1;
    else if ((op == OP_REMAINDER || op == OP_FMOD) && !dt_is_float(rd)) fkind = 2;
    else if (op == OP_MULTIPLY && dt_is_float(rd)) fkind = 3;
    bool want = fpe && fkind;
    bool aligned = trailing_aligned(a, bnd, bsh) && trailing_aligned(b, bnd, bsh) && out->ndim == bnd;
    // overlap: compute into a temporary when out aliases an input differently
    bool tmp_needed = false;
    int64_t ab[IONP_MAX_DIMS], bb[IONP_MAX_DIMS];
    bcast_strides(a, out->ndim, out->shape, ab);
    bcast_strides(b, out->ndim, out->shape, bb);
    if (ranges_overlap(out, a) && !same_layout(out, a, ab)) tmp_needed = true;
    if (ranges_overlap(out, b) && !same_layout(out, b, bb)) tmp_needed = true;
    if (where && ranges_overlap(out, where)) tmp_needed = true;
    if (want && fkind == 3 && !aligned) tmp_needed = true;  // the quirk detector reads the computed result
    FlagWord fw;
    if (want && (st = fw.open(s))) return st;
    if (fpe) *fpe = 0;
    if (!tmp_needed) {
        if ((st = launch_ew(true, op, cd, rd, a, b, out, where, fw.d, want && aligned, s))) return st;
    } else {
        // full computed result in the loop result dtype, C order, then write_out
        IonpArr t;
        memset(&t, 0, sizeof(t));
        t.dtype = rd;
        t.ndim = bnd;
        int64_t acc = 1;
        for (int i = bnd - 1; i >= 0; --i) { t.shape[i] = bsh[i]; t.strides[i] = acc; acc *= std::max<int64_t>(bsh[i], 1); }
        t.data = scratch_alloc((size_t)std::max<int64_t>(acc, 1) * dt_bytes(rd), s);
        if (!t.data) return IONP_ERR_OOM;
        st = launch_ew(true, op, cd, rd, a, b, &t, nullptr, fw.d, want && aligned, s);
        if (!st && want && !aligned) {
            FpeQuirkDesc q;
            memset(&q, 0, sizeof(q));
            q.kind = fkind;
            q.out_is_float = dt_is_float(rd);
            q.la = numel(a); q.lb = numel(b); q.lo = numel(&t);
            q.n = std::max(q.la, q.lb);
            if (fkind == 3) q.n = std::max(q.n, q.lo);
            q.a = elem_ptr(a); q.da = a->dtype; q.nda = a->ndim;
            q.b = elem_ptr(b); q.dbt = b->dtype; q.ndb = b->ndim;
            q.o = t.data; q.dout = rd; q.ndo = t.ndim;
            for (int i = 0; i < a->ndim; ++i) { q.sha[i] = a->shape[i]; q.sta[i] = a->strides[i]; }
            for (int i = 0; i < b->ndim; ++i) { q.shb[i] = b->shape[i]; q.stb[i] = b->strides[i]; }
            for (int i = 0; i < t.ndim; ++i) { q.sho[i] = t.shape[i]; q.sto[i] = t.strides[i]; }
            if (q.la && q.lb) st = cuda_err(launch_fpe_quirk(q, fw.d, s), "fpe detector");
        }
        if (!st) {
            // write_out: cast into out with the optional mask
            st = cast_impl(&t, out, where, s);
        }
        scratch_free(t.data, s);
        if (st) return st;
    }
    if (want && !tmp_needed && !aligned) {
        // the computed values are not needed by the divide/remainder detectors
        FpeQuirkDesc q;
        memset(&q, 0, sizeof(q));
        q.kind = fkind;
        q.out_is_float = dt_is_float(rd);
        q.la = numel(a); q.lb = numel(b); q.lo = numel(out);
        q.n = std::max(q.la, q.lb);
        q.a = elem_ptr(a); q.da = a->dtype; q.nda = a->ndim;
        q.b = elem_ptr(b); q.dbt = b->dtype; q.ndb = b->ndim;
        for (int i = 0; i < a->ndim; ++i) { q.sha[i] = a->shape[i]; q.sta[i] = a->strides[i]; }
        for (int i = 0; i < b->ndim; ++i) { q.shb[i] = b->shape[i]; q.stb[i] = b->strides[i]; }
        if (q.la && q.lb && (st = cuda_err(launch_fpe_quirk(q, fw.d, s), "fpe detector"))) return st;
    }
    if (want) {
        if (numel(a) == 0 || numel(b) == 0) return IONP_OK;
        return fw.deliver(fpe, nowait);
    }
    return IONP_OK;
}

int32_t ionp_binary(int32_t op, const IonpArr* a, const IonpArr* b, IonpArr* out, const IonpArr* where, uint32_t* fpe,
                    IonpStream stream) {
    NvtxRange nvtx_("ionp_binary");
    return binary_call(op, a, b, out, where, fpe, false, stream);
}
int32_t ionp_binary_nowait(int32_t op, const IonpArr* a, const IonpArr* b, IonpArr* out, const IonpArr* where,
                           uint32_t* fpe, IonpStream stream) {
    NvtxRange nvtx_("ionp_binary_nowait");
    return binary_call(op, a, b, out, where, fpe, true, stream);
}

static int32_t unary_call(int32_t op, const IonpArr* a, IonpArr* out, const IonpArr* where, uint32_t* fpe, bool nowait,
                          IonpStream stream) {
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    if (where && (st = check_arr(where, "where"))) return st;
    if (where && where->dtype != DT_BOOL) return set_err(IONP_ERR_TYPE, "where= mask must be boolean");
    cudaStream_t s = (cudaStream_t)stream;
    int cd, rd;
    if ((st = unary_loop(op, a->dtype, &cd, &rd))) return st;
    int64_t ab[IONP_MAX_DIMS];
    if (!bcast_strides(a, out->ndim, out->shape, ab))
        return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(a->shape, a->ndim) + " " + fmt_shape(out->shape, out->ndim) + " ");
    if ((ranges_overlap(out, a) && !same_layout(out, a, ab)) || (where && ranges_overlap(out, where)))
        return set_err(IONP_ERR_UNSUPPORTED, "out= overlapping the input with a different layout is not supported");
    bool want = fpe && (op == OP_SQRT || op == OP_LOG);
    FlagWord fw;
    if (want && (st = fw.open(s))) return st;
    if (fpe) *fpe = 0;
    if ((st = launch_ew(false, op, cd, rd, a, nullptr, out, where, fw.d, want, s))) return st;
    if (want) return fw.deliver(fpe, nowait);
    return IONP_OK;
}

int32_t ionp_unary(int32_t op, const IonpArr* a, IonpArr* out, const IonpArr* where, uint32_t* fpe, IonpStream stream) {
    NvtxRange nvtx_("ionp_unary");
    return unary_call(op, a, out, where, fpe, false, stream);
}
int32_t ionp_unary_nowait(int32_t op, const IonpArr* a, IonpArr* out, const IonpArr* where, uint32_t* fpe,
                          IonpStream stream) {
    NvtxRange nvtx_("ionp_unary_nowait");
    return unary_call(op, a, out, where, fpe, true, stream);
}

int32_t ionp_cast(const IonpArr* a, IonpArr* out, IonpStream stream) {
    NvtxRange nvtx_("ionp_cast");
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    return cast_impl(a, out, nullptr, (cudaStream_t)stream);
}

// ndarray.astype (ionp-py/src/lib.rs:5960-6003): detect_cast_overflow
// (fpe.rs:398) on the source, then the cast. Only a float source cast to an
// integer destination is checked; its bounds are the destination's range as
// float64 (i64::MAX as f64 is 2^63, so 2^63 itself is not flagged).
int32_t ionp_astype(const IonpArr* a, IonpArr* out, uint32_t* fpe, IonpStream stream) {
    NvtxRange nvtx_("ionp_astype");
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (fpe) *fpe = 0;
    const bool to_int = !dt_is_float(out->dtype) && out->dtype != DT_BOOL;
    if (fpe && dt_is_float(a->dtype) && to_int && numel(a) > 0) {
        double lo, hi;
        switch (out->dtype) {
            case DT_I8: lo = -128.0; hi = 127.0; break;
            case DT_I16: lo = -32768.0; hi = 32767.0; break;
            case DT_I32: lo = -2147483648.0; hi = 2147483647.0; break;
            case DT_I64: lo = -9223372036854775808.0; hi = 9223372036854775808.0; break;
            case DT_U8: lo = 0.0; hi = 255.0; break;
            case DT_U16: lo = 0.0; hi = 65535.0; break;
            case DT_U32: lo = 0.0; hi = 4294967295.0; break;
            default: lo = 0.0; hi = 18446744073709551616.0; break;
        }
        MergeIn mi;
        memset(&mi, 0, sizeof(mi));
        mi.nd = a->ndim;
        mi.nops = 1;
        for (int i = 0; i < a->ndim; ++i) { mi.shape[i] = a->shape[i]; mi.st[0][i] = a->strides[i]; }
        MergeOut mo = merge_dims(mi);
        FlagWord fw;
        if ((st = fw.open(s))) return st;
        const int lead = mo.nd > EW_MAXD ? mo.nd - EW_MAXD : 0;
        int64_t nlead = 1;
        for (int i = 0; i < lead; ++i) nlead *= mo.shape[i];
        for (int64_t q = 0; q < nlead; ++q) {
            int64_t rem = q, oa = 0;
            for (int i = lead - 1; i >= 0; --i) {
                oa += (rem % mo.shape[i]) * mo.st[0][i];
                rem /= mo.shape[i];
            }
            EwDesc d;
            memset(&d, 0, sizeof(d));
            d.nd = mo.nd - lead;
            d.n = 1;
            for (int i = 0; i < d.nd; ++i) {
                d.shape[i] = mo.shape[lead + i];
                d.n *= d.shape[i];
                d.a.st[i] = mo.st[0][lead + i];
            }
            if (d.nd == 0) { d.nd = 1; d.shape[0] = 1; d.n = 1; }
            d.a.p = elem_ptr(a) + oa * dt_bytes(a->dtype);
            d.a.dt = a->dtype;
            if ((st = cuda_err(launch_cast_check(d, lo, hi, fw.d, s), "cast overflow detector"))) return st;
        }
        if ((st = fw.read(fpe))) return st;
    }
    return cast_impl(a, out, nullptr, s);
}

}  // extern "C"

namespace ionp {
int32_t cast_impl(const IonpArr* a, IonpArr* out, const IonpArr* where, cudaStream_t s) {
    int32_t st;
    const int nd = out->ndim;
    MergeIn mi;
    mi.nd = nd;
    mi.nops = 3;
    for (int i = 0; i < nd; ++i) { mi.shape[i] = out->shape[i]; mi.st[0][i] = out->strides[i]; mi.st[2][i] = 0; }
    if (!bcast_strides(a, nd, out->shape, mi.st[1]))
        return set_err(IONP_ERR_BROADCAST, "could not broadcast input array from shape " + fmt_shape(a->shape, a->ndim) + " into shape " + fmt_shape(out->shape, nd));
    if (where && !bcast_strides(where, nd, out->shape, mi.st[2]))
        return set_err(IONP_ERR_BROADCAST, "could not broadcast where mask from shape " + fmt_shape(where->shape, where->ndim) + " into shape " + fmt_shape(out->shape, nd));
    if (numel(out) == 0) return IONP_OK;
    MergeOut mo = merge_dims(mi);
    int lead = mo.nd > EW_MAXD ? mo.nd - EW_MAXD : 0;
    int64_t nlead = 1;
    for (int i = 0; i < lead; ++i) nlead *= mo.shape[i];
    for (int64_t q = 0; q < nlead; ++q) {
        int64_t rem = q, oo = 0, oa = 0, om = 0;
        for (int i = lead - 1; i >= 0; --i) {
            int64_t id = rem % mo.shape[i];
            rem /= mo.shape[i];
            oo += id * mo.st[0][i];
            oa += id * mo.st[1][i];
            om += id * mo.st[2][i];
        }
        EwDesc d;
        memset(&d, 0, sizeof(d));
        d.nd = mo.nd - lead;
        d.n = 1;
        for (int i = 0; i < d.nd; ++i) {
            d.shape[i] = mo.shape[lead + i];
            d.n *= d.shape[i];
            d.so[i] = mo.st[0][lead + i];
            d.a.st[i] = mo.st[1][lead + i];
            d.m.st[i] = mo.st[2][lead + i];
        }
        d.o = (char*)elem_ptr(out) + oo * dt_bytes(out->dtype);
        d.odt = out->dtype;
        d.a.p = elem_ptr(a) + oa * dt_bytes(a->dtype);
        d.a.dt = a->dtype;
        if (where) { d.m.p = elem_ptr(where) + om; d.m.dt = DT_BOOL; }
        if ((st = cuda_err(launch_cast(d, s), "cast launch"))) return st;
    }
    return IONP_OK;
}
}  // namespace ionp

extern "C" {

// order='K' result strides (lib.rs:1290-1330; array.rs:1153-1222)
int32_t ionp_order_k_strides(int32_t nops, const IonpArr* const* ops, int32_t ndim, const int64_t* shape, int64_t* out) {
    if (ndim < 0 || ndim > IONP_MAX_DIMS || !out) return set_err(IONP_ERR_INVALID, "bad arguments");
    auto is_contig = [](const IonpArr* a, bool f) {
        if (numel(a) == 0) return true;
        int64_t expect = 1;
        for (int k = 0; k < a->ndim; ++k) {
            int i = f ? k : a->ndim - 1 - k;
            if (a->shape[i] == 1) continue;
            if (a->strides[i] != expect) return false;
            expect *= a->shape[i];
        }
        return true;
    };
    std::vector<int> perm(ndim);
    for (int i = 0; i < ndim; ++i) perm[i] = i;
    bool allc = true, allf = true;
    for (int k = 0; k < nops; ++k) { allc = allc && is_contig(ops[k], false); allf = allf && is_contig(ops[k], true); }
    if (!allc && allf) std::reverse(perm.begin(), perm.end());
    else if (!allc) {
        // multi_sorted_stride_perm: insertion sort where an axis moves before
        // another only if some operand, first decisive, says its stride is larger
        for (int i0 = 1; i0 < ndim; ++i0) {
            int ax0 = perm[i0], ipos = i0;
            for (int i1 = i0 - 1; i1 >= 0; --i1) {
                int ax1 = perm[i1];
                bool ambig = true, swap = false;
                for (int k = 0; k < nops; ++k) {
                    const IonpArr* o = ops[k];
                    int off = ndim - o->ndim;
                    if (ax0 < off || ax1 < off) continue;
                    if (o->shape[ax0 - off] == 1 || o->shape[ax1 - off] == 1) continue;
                    int64_t s0 = std::llabs(o->strides[ax0 - off]), s1 = std::llabs(o->strides[ax1 - off]);
                    if (s0 <= s1) swap = false;
                    else if (ambig) swap = true;
                    ambig = false;
                }
                if (!ambig) {
                    if (swap) ipos = i1;
                    else break;
                }
            }
            for (int k = i0; k > ipos; --k) perm[k] = perm[k - 1];
            perm[ipos] = ax0;
        }
    }
    int64_t acc = 1, total = 1;
    for (int i = 0; i < ndim; ++i) total *= shape[i];
    for (int i = ndim - 1; i >= 0; --i) {
        out[perm[i]] = acc;
        acc *= std::max<int64_t>(shape[perm[i]], 1);
    }
    if (total == 0)
        for (int i = 0; i < ndim; ++i) out[i] = 0;
    return IONP_OK;
}

// relayout_for_reduction / reduce_output_layout (array.rs:845-930)
int32_t ionp_reduce_layout(const IonpArr* a, const int32_t* axes, int32_t naxes, int32_t keepdims, int32_t* out_ndim,
                           int64_t* out_shape, int64_t* out_strides) {
    if (!a || !out_ndim || !out_shape || !out_strides) return set_err(IONP_ERR_INVALID, "bad arguments");
    int nd = a->ndim;
    bool red[IONP_MAX_DIMS] = {false};
    for (int k = 0; k < naxes; ++k) red[axes[k]] = true;
    std::vector<int> full(nd);
    for (int i = 0; i < nd; ++i) full[i] = i;
    std::stable_sort(full.begin(), full.end(), [&](int x, int y) { return std::llabs(a->strides[x]) > std::llabs(a->strides[y]); });
    if (!keepdims) {
        std::vector<int> retained;
        for (int i = 0; i < nd; ++i) if (!red[i]) retained.push_back(i);
        int r = (int)retained.size();
        std::vector<int> local_of(nd, -1);
        for (int i = 0; i < r; ++i) local_of[retained[i]] = i;
        std::vector<int> lperm;
        for (int ax : full) if (local_of[ax] >= 0) lperm.push_back(local_of[ax]);
        int64_t total = 1;
        for (int i = 0; i < r; ++i) { out_shape[i] = a->shape[retained[i]]; total *= out_shape[i]; }
        int64_t acc = 1;
        for (int i = r - 1; i >= 0; --i) { out_strides[lperm[i]] = acc; acc *= std::max<int64_t>(out_shape[lperm[i]], 1); }
        if (total == 0) for (int i = 0; i < r; ++i) out_strides[i] = 0;
        *out_ndim = r;
        return IONP_OK;
    }
    int64_t total = 1;
    for (int i = 0; i < nd; ++i) { out_shape[i] = red[i] ? 1 : a->shape[i]; total *= out_shape[i]; }
    int64_t acc = 1;
    for (int i = nd - 1; i >= 0; --i) { out_strides[full[i]] = acc; acc *= std::max<int64_t>(out_shape[full[i]], 1); }
    if (total == 0) for (int i = 0; i < nd; ++i) out_strides[i] = 0;
    *out_ndim = nd;
    return IONP_OK;
}

}  // extern "C"

// ===========================================================================
// runtime helpers
// ===========================================================================
extern "C" {

int32_t ionp_memcpy(void* dst, const void* src, size_t bytes, int32_t kind, IonpStream stream) {
    if (bytes == 0) return IONP_OK;
    cudaMemcpyKind k = kind == IONP_H2D ? cudaMemcpyHostToDevice : kind == IONP_D2H ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    return cuda_err(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream), "memcpy");
}
int32_t ionp_stream_create(IonpStream* stream) {
    cudaStream_t s;
    int32_t st = cuda_err(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream create");
    if (!st) *stream = (IonpStream)s;
    return st;
}
int32_t ionp_stream_destroy(IonpStream stream) { return cuda_err(cudaStreamDestroy((cudaStream_t)stream), "stream destroy"); }
int32_t ionp_stream_synchronize(IonpStream stream) {
    int32_t st = cuda_err(cudaStreamSynchronize((cudaStream_t)stream), "stream synchronize");
    return st ? st : check_async_error();
}
int32_t ionp_device_synchronize(void) {
    int32_t st = cuda_err(cudaDeviceSynchronize(), "device synchronize");
    return st ? st : check_async_error();
}
int32_t ionp_host_alloc(void** ptr, size_t bytes) { return cuda_err(cudaMallocHost(ptr, bytes ? bytes : 1), "pinned alloc"); }
int32_t ionp_host_free(void* ptr) { return cuda_err(cudaFreeHost(ptr), "pinned free"); }
int32_t ionp_event_create(void** ev) {
    cudaEvent_t e;
    int32_t st = cuda_err(cudaEventCreate(&e), "event create");
    if (!st) *ev = (void*)e;
    return st;
}
int32_t ionp_event_destroy(void* ev) { return cuda_err(cudaEventDestroy((cudaEvent_t)ev), "event destroy"); }
int32_t ionp_event_record(void* ev, IonpStream stream) { return cuda_err(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream), "event record"); }
int32_t ionp_event_elapsed_ms(void* a, void* b, float* ms) {
    int32_t st = cuda_err(cudaEventSynchronize((cudaEvent_t)b), "event sync");
    if (st) return st;
    return cuda_err(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b), "event elapsed");
}
int32_t ionp_set_device(int32_t device) { return cuda_err(cudaSetDevice(device), "set device"); }
int32_t ionp_device_info(int32_t* count, int32_t* sm_count, char* name, size_t len) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); n = 0; }
    if (count) *count = n;
    if (n == 0) return IONP_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); dev = 0; }
    cudaDeviceProp p;
    int32_t st = cuda_err(cudaGetDeviceProperties(&p, dev), "device properties");
    if (st) return st;
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (name && len) { strncpy(name, p.name, len - 1); name[len - 1] = 0; }
    return IONP_OK;
}

}  // extern "C"
