// Which (op, compute dtype) pairs each reduction kernel is instantiated for.
#pragma once
#include "ionp_reduce.cuh"

namespace ionp {

// Ops whose fold may be re-bracketed without changing a single bit (given
// left-to-right operand order is kept): integer/bool add and multiply
// (wrapping), max/min (first NaN / tie rules are associative), bitwise and
// logical ops, and equal/not_equal on bool (xnor/xor).
__host__ __device__ constexpr bool red_assoc(int op, int cd) {
    return ((op == OP_ADD || op == OP_MULTIPLY) && !dt_is_float(cd)) || op == OP_MAXIMUM || op == OP_MINIMUM ||
           ((op == OP_BITWISE_AND || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) && !dt_is_float(cd)) ||
           (op_is_logical(op) && cd == DT_BOOL) || ((op == OP_EQUAL || op == OP_NOT_EQUAL) && cd == DT_BOOL);
}
// Row (tree) kernel: associative ops plus the float pairwise add.
__host__ __device__ constexpr bool red_row_valid(int op, int cd) { return red_assoc(op, cd) || (op == OP_ADD && dt_is_float(cd)); }
// Any op/dtype pair that has a reduce loop in the reference.
__host__ __device__ constexpr bool red_any_valid(int op, int cd) {
    if (op_is_compare(op)) return cd == DT_BOOL;
    if (op_is_logical(op)) return cd == DT_BOOL;
    if (op == OP_ADD || op == OP_MULTIPLY || op == OP_MAXIMUM || op == OP_MINIMUM) return true;
    if (op == OP_SUBTRACT) return cd != DT_BOOL;
    if (op == OP_DIVIDE) return dt_is_float(cd);
    if (op == OP_BITWISE_AND || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) return !dt_is_float(cd);
    if (op == OP_LEFT_SHIFT || op == OP_RIGHT_SHIFT) return dt_is_sint(cd) || dt_is_uint(cd);
    if (op == OP_FLOOR_DIVIDE) return cd != DT_BOOL;
    return false;
}

#define IONP_RED_OPS(X)                                                                                        \
    X(OP_ADD) X(OP_SUBTRACT) X(OP_MULTIPLY) X(OP_DIVIDE) X(OP_MAXIMUM) X(OP_MINIMUM) X(OP_GREATER)           \
    X(OP_GREATER_EQUAL) X(OP_LESS) X(OP_LESS_EQUAL) X(OP_EQUAL) X(OP_NOT_EQUAL) X(OP_LOGICAL_AND)              \
    X(OP_LOGICAL_OR) X(OP_LOGICAL_XOR) X(OP_BITWISE_AND) X(OP_BITWISE_OR) X(OP_BITWISE_XOR) X(OP_FLOOR_DIVIDE) \
    X(OP_LEFT_SHIFT) X(OP_RIGHT_SHIFT)

#define IONP_DTS(X) X(DT_BOOL) X(DT_I8) X(DT_I16) X(DT_I32) X(DT_I64) X(DT_U8) X(DT_U16) X(DT_U32) X(DT_U64) X(DT_F16) X(DT_F32) X(DT_F64)

}  // namespace ionp
