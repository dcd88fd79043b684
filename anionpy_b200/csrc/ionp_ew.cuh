// Element-wise kernels (ufunc __call__ hot path).
//
//  k_bin_contig / k_un_contig : operands contiguous (or 0-d broadcast) in the
//      loop dtype, 16-byte aligned: 128-bit vector loads/stores, unrolled so
//      each thread keeps several independent loads in flight, streaming cache
//      hints (data is touched once).
//  k_bin_nd / k_un_nd : up to 4 merged dims with arbitrary element strides
//      (broadcast axes have stride 0), cast-on-load from any operand dtype,
//      cast-on-store to the out= dtype, optional where= mask. Long inner rows
//      are walked in coalesced row tiles; short rows use a flat index.
// The per-element arithmetic is BinOp/UnOp from ionp_scalar.cuh / ionp_math.cuh.
#pragma once
#include "ionp_scalar.cuh"
#include "ionp_math.cuh"
#include "ionp_internal.h"

namespace ionp {

constexpr int EW_THREADS = 256;

__device__ __forceinline__ void flush_flags(uint32_t bits, uint32_t* flags) {
    bits = __reduce_or_sync(0xffffffffu, bits);
    if (bits && (threadIdx.x & 31) == 0) atomicOr(flags, bits);
}

template <class T> struct Vec16 {
    static constexpr int N = 16 / (int)sizeof(T);
    T v[N];
};
template <class T> __device__ __forceinline__ Vec16<T> ldv(const T* p, int64_t i) {
    Vec16<T> r;
    uint4 u = __ldcs(reinterpret_cast<const uint4*>(p) + i);
    memcpy(&r, &u, 16);
    return r;
}
// store N results of type R (N*sizeof(R) bytes, naturally aligned)
template <class R, int N> __device__ __forceinline__ void stv(R* p, int64_t i, const R (&r)[N]) {
    constexpr int B = N * (int)sizeof(R);
    if constexpr (B == 16) { uint4 u; memcpy(&u, r, 16); __stcs(reinterpret_cast<uint4*>(p) + i, u); }
    else if constexpr (B == 8) { uint2 u; memcpy(&u, r, 8); __stcs(reinterpret_cast<uint2*>(p) + i, u); }
    else if constexpr (B == 4) { unsigned u; memcpy(&u, r, 4); __stcs(reinterpret_cast<unsigned*>(p) + i, u); }
    else if constexpr (B == 2) { unsigned short u; memcpy(&u, r, 2); reinterpret_cast<unsigned short*>(p)[i] = u; }
    else { for (int k = 0; k < N; ++k) p[i * N + k] = r[k]; }
}

// ---------------------------------------------------------------------------
// binary
// ---------------------------------------------------------------------------
// 32-bit integer division ops: their loads are issued a group ahead (measured
// 10 % faster for int32 floor_divide; the same prefetch made the float and
// 64-bit division family 7-50 % slower, so they keep the plain loop)
__host__ __device__ constexpr bool ew_prefetch_op(int op, int cd) {
    return (op == OP_FLOOR_DIVIDE || op == OP_REMAINDER || op == OP_FMOD) && (cd == DT_I32 || cd == DT_U32);
}

// N results of one vector of pairs. Ops with a branch-free fast path
// (BinOp::FAST) evaluate the whole vector that way and redo it with apply()
// and the FPE detector only when some pair lies outside the fast path, whose
// pairs raise no FPE flag; the others apply() and detect per pair. Used by
// the transposed tile kernel k_bin_trv1, where gathering a vector's pairs
// before the arithmetic measured 4-10 % faster on the int32 / int64 /
// float32 division family (float64 division keeps its per-pair loop there:
// 5-10 % slower this way).
template <int OP, int CD, bool FPE, int N>
__device__ __forceinline__ void bin_vec(const typename DT<CD>::T (&x)[N], const typename DT<CD>::T (&y)[N],
                                        typename BinOp<OP, CD>::R (&r)[N], uint32_t& bits) {
    typedef BinOp<OP, CD> Op;
    if constexpr (Op::FAST) {
        bool ok = true;
#pragma unroll
        for (int k = 0; k < N; ++k) ok &= Op::fast(x[k], y[k], &r[k]);
        if (ok) return;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        r[k] = Op::apply(x[k], y[k]);
        if constexpr (FPE) bits |= fpe_bits<OP, CD>(x[k], y[k], r[k]);
    }
}

template <int OP, int CD, bool FPE>
__device__ __forceinline__ void bin_contig_body(const typename DT<CD>::T* __restrict__ a, const typename DT<CD>::T* __restrict__ b,
                                                typename BinOp<OP, CD>::R* __restrict__ o, int64_t n, int a_sc, int b_sc,
                                                uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef typename BinOp<OP, CD>::R R;
    constexpr int N = Vec16<T>::N;
    constexpr int U = 2;  // vectors per thread per iteration
    uint32_t bits = 0;
    const T a0 = a[0], b0 = b[0];
    const int64_t nvec = n / N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    auto load = [&](Vec16<T> (&xa)[U], Vec16<T> (&xb)[U], int64_t w) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!a_sc) xa[u] = ldv(a, w + u * stride); else for (int k = 0; k < N; ++k) xa[u].v[k] = a0;
            if (!b_sc) xb[u] = ldv(b, w + u * stride); else for (int k = 0; k < N; ++k) xb[u].v[k] = b0;
        }
    };
    auto compute = [&](const Vec16<T> (&xa)[U], const Vec16<T> (&xb)[U], int64_t w) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            R r[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
                r[k] = BinOp<OP, CD>::apply(xa[u].v[k], xb[u].v[k]);
                if constexpr (FPE) bits |= fpe_bits<OP, CD>(xa[u].v[k], xb[u].v[k], r[k]);
            }
            stv<R, N>(o, w + u * stride, r);
        }
    };
    if constexpr (ew_prefetch_op(OP, CD)) {
        // the next group's vectors are loaded before this group is
        // computed, so loads stay in flight through the math
        Vec16<T> xa[U], xb[U], na[U], nb[U];
        if (v + (U - 1) * stride < nvec) {
            load(xa, xb, v);
            for (;;) {
                const int64_t vn = v + U * stride;
                const bool more = vn + (U - 1) * stride < nvec;
                if (more) load(na, nb, vn);
                compute(xa, xb, v);
                v = vn;
                if (!more) break;
#pragma unroll
                for (int u = 0; u < U; ++u) { xa[u] = na[u]; xb[u] = nb[u]; }
            }
        }
    } else {
        for (; v + (U - 1) * stride < nvec; v += U * stride) {
            Vec16<T> xa[U], xb[U];
            load(xa, xb, v);
            compute(xa, xb, v);
        }
    }
    for (; v < nvec; v += stride) {
        Vec16<T> xa, xb;
        if (!a_sc) xa = ldv(a, v); else for (int k = 0; k < N; ++k) xa.v[k] = a0;
        if (!b_sc) xb = ldv(b, v); else for (int k = 0; k < N; ++k) xb.v[k] = b0;
        R r[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r[k] = BinOp<OP, CD>::apply(xa.v[k], xb.v[k]);
            if constexpr (FPE) bits |= fpe_bits<OP, CD>(xa.v[k], xb.v[k], r[k]);
        }
        stv<R, N>(o, v, r);
    }
    // tail
    for (int64_t i = nvec * N + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T x = a_sc ? a0 : a[i], y = b_sc ? b0 : b[i];
        R r = BinOp<OP, CD>::apply(x, y);
        if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r);
        o[i] = r;
    }
    if constexpr (FPE) flush_flags(bits, flags);
}
template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_bin_contig(const typename DT<CD>::T* __restrict__ a, const typename DT<CD>::T* __restrict__ b,
             typename BinOp<OP, CD>::R* __restrict__ o, int64_t n, int a_sc, int b_sc, uint32_t* flags) {
    bin_contig_body<OP, CD, FPE>(a, b, o, n, a_sc, b_sc, flags);
}
// the same with three resident CTAs, for float64 floor_divide (80 registers,
// 90 unbounded): measured 13 % faster, where the same bound made float64
// remainder 14 % slower
template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS, 3)
k_bin_contig3(const typename DT<CD>::T* __restrict__ a, const typename DT<CD>::T* __restrict__ b,
              typename BinOp<OP, CD>::R* __restrict__ o, int64_t n, int a_sc, int b_sc, uint32_t* flags) {
    bin_contig_body<OP, CD, FPE>(a, b, o, n, a_sc, b_sc, flags);
}

// Offsets of flat index i over the merged dims (C order, last dim fastest).
struct Offs { int64_t a, b, o, m; };
__device__ __forceinline__ Offs unravel(const EwDesc& d, int64_t i, int nd_from_end) {
    Offs r = {0, 0, 0, 0};
    for (int k = d.nd - 1 - nd_from_end; k >= 0; --k) {
        int64_t s = d.shape[k];
        int64_t q = i / s;
        int64_t id = i - q * s;
        i = q;
        r.a += id * d.a.st[k]; r.b += id * d.b.st[k]; r.o += id * d.so[k]; r.m += id * d.m.st[k];
    }
    return r;
}

template <int OP, int CD, bool FPE, bool SAME>
__global__ void __launch_bounds__(EW_THREADS)
k_bin_nd(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef BinOp<OP, CD> Op;
    typedef typename Op::R R;
    uint32_t bits = 0;
    const int nd = d.nd;
    const int64_t inner = d.shape[nd - 1];
    const int64_t sa = d.a.st[nd - 1], sb = d.b.st[nd - 1], so = d.so[nd - 1], sm = d.m.st[nd - 1];
    const bool has_m = d.m.p != nullptr;
    auto one = [&](int64_t oa, int64_t ob, int64_t oo, int64_t om) {
        T x, y;
        if constexpr (SAME) { x = ((const T*)d.a.p)[oa]; y = ((const T*)d.b.p)[ob]; }
        else { x = load_cast<CD>(d.a.p, oa, d.a.dt); y = load_cast<CD>(d.b.p, ob, d.b.dt); }
        R r = Op::apply(x, y);
        if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r);
        if (has_m && !((const uint8_t*)d.m.p)[om]) return;
        if constexpr (SAME) ((R*)d.o)[oo] = r;
        else store_cast<Op::OUT_DT>(d.o, oo, d.odt, r);
    };
    if (inner >= 64) {
        constexpr int ILP = 4;
        const int64_t tile = (int64_t)blockDim.x * ILP;
        const int64_t tpr = (inner + tile - 1) / tile;
        const int64_t rows = d.n / inner;
        const int64_t ntiles = rows * tpr;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            int64_t row = t / tpr, cb = t - row * tpr;
            Offs base = unravel(d, row, 1);
            int64_t c0 = cb * tile + threadIdx.x;
#pragma unroll
            for (int u = 0; u < ILP; ++u) {
                int64_t c = c0 + u * blockDim.x;
                if (c < inner) one(base.a + c * sa, base.b + c * sb, base.o + c * so, base.m + c * sm);
            }
        }
    } else {
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
            Offs f = unravel(d, i, 0);
            one(f.a, f.b, f.o, f.m);
        }
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// One merged dim with any element strides, operands and result in the loop
// dtypes, no mask (a step-k slice, a reversed view): U elements of each
// operand loaded per thread before any arithmetic, so 2U loads are in
// flight, and no per-element index unravelling.
// streaming (evict-first) scalar load / store where the type has one
template <class T> __device__ __forceinline__ T ld_cs(const T* p) {
    if constexpr (sizeof(T) >= 4) return __ldcs(p);
    else return *p;
}
template <class T> __device__ __forceinline__ void st_cs(T* p, T v) {
    if constexpr (sizeof(T) >= 4) __stcs(p, v);
    else *p = v;
}

template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_bin_run(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef BinOp<OP, CD> Op;
    typedef typename Op::R R;
    constexpr int U = sizeof(T) >= 8 ? 4 : 8;
    const T* pa = reinterpret_cast<const T*>(d.a.p);
    const T* pb = reinterpret_cast<const T*>(d.b.p);
    R* po = reinterpret_cast<R*>(d.o);
    const int64_t sa = d.a.st[0], sb = d.b.st[0], so = d.so[0], n = d.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    uint32_t bits = 0;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (U - 1) * stride < n; i += U * stride) {
        T x[U], y[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            x[u] = ld_cs(pa + (i + u * stride) * sa);
            y[u] = ld_cs(pb + (i + u * stride) * sb);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const R r = Op::apply(x[u], y[u]);
            if constexpr (FPE) bits |= fpe_bits<OP, CD>(x[u], y[u], r);
            st_cs(po + (i + u * stride) * so, r);
        }
    }
    for (; i < n; i += stride) {
        const T x = pa[i * sa], y = pb[i * sb];
        const R r = Op::apply(x, y);
        if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r);
        po[i * so] = r;
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// Two merged dims whose operands disagree on which dim is contiguous (a
// transposed view against a C-ordered one): 32 x 32 tiles staged through
// shared memory. Each operand is read along its own contiguous dim, the
// output written along its own, so every global access is coalesced.
constexpr int TR_TILE = 32;
template <class T> __device__ __forceinline__ void tr_load(T (*sm)[TR_TILE + 1], const T* p, int64_t s0, int64_t s1,
                                                         int64_t i0, int64_t j0, int64_t R, int64_t C) {
    const int tid = threadIdx.x;
    if (s0 == 1 && s1 != 1) {  // column-contiguous: consecutive threads walk rows
#pragma unroll
        for (int k = 0; k < TR_TILE * TR_TILE / EW_THREADS; ++k) {
            const int r = tid % TR_TILE, c = tid / TR_TILE + k * (EW_THREADS / TR_TILE);
            if (i0 + r < R && j0 + c < C) sm[r][c] = p[(i0 + r) * s0 + (j0 + c) * s1];
        }
    } else {                   // row-contiguous (or broadcast): consecutive threads walk columns
#pragma unroll
        for (int k = 0; k < TR_TILE * TR_TILE / EW_THREADS; ++k) {
            const int c = tid % TR_TILE, r = tid / TR_TILE + k * (EW_THREADS / TR_TILE);
            if (i0 + r < R && j0 + c < C) sm[r][c] = p[(i0 + r) * s0 + (j0 + c) * s1];
        }
    }
}

template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_bin_tr(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef BinOp<OP, CD> Op;
    typedef typename Op::R R;
    __shared__ T sa[TR_TILE][TR_TILE + 1], sb[TR_TILE][TR_TILE + 1];
    uint32_t bits = 0;
    const int64_t R0 = d.shape[0], C0 = d.shape[1];
    const int64_t tr = (R0 + TR_TILE - 1) / TR_TILE, tc = (C0 + TR_TILE - 1) / TR_TILE;
    const T* pa = (const T*)d.a.p;
    const T* pb = (const T*)d.b.p;
    R* po = (R*)d.o;
    const bool ocol = d.so[0] == 1 && d.so[1] != 1;
    const int tid = threadIdx.x;
    for (int64_t t = blockIdx.x; t < tr * tc; t += gridDim.x) {
        const int64_t i0 = (t / tc) * TR_TILE, j0 = (t % tc) * TR_TILE;
        tr_load<T>(sa, pa, d.a.st[0], d.a.st[1], i0, j0, R0, C0);
        tr_load<T>(sb, pb, d.b.st[0], d.b.st[1], i0, j0, R0, C0);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < TR_TILE * TR_TILE / EW_THREADS; ++k) {
            int r, c;
            if (ocol) { r = tid % TR_TILE; c = tid / TR_TILE + k * (EW_THREADS / TR_TILE); }
            else { c = tid % TR_TILE; r = tid / TR_TILE + k * (EW_THREADS / TR_TILE); }
            if (i0 + r < R0 && j0 + c < C0) {
                const T x = sa[r][c], y = sb[r][c];
                const R v = Op::apply(x, y);
                if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, v);
                po[(i0 + r) * d.so[0] + (j0 + c) * d.so[1]] = v;
            }
        }
        __syncthreads();
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// The same two-dim case for whole tiles whose rows are 16-byte aligned:
// TILE x TILE tiles (64 for 4-byte types, 32 for 8-byte ones), every global
// load and store a 16-byte vector along that array's own contiguous dim
// (VW elements), so a warp moves 512 bytes per instruction; each thread has
// all its vectors of both operands in flight before the tile's barrier.
// Shared rows are padded by one element: the column-wise scatter of a
// column-contiguous operand hits each bank at most twice, the row-wise reads
// of the compute phase not at all.
template <class T> struct TrV {
    static constexpr int VW = 16 / (int)sizeof(T);
    static constexpr int TILE = sizeof(T) == 4 ? 64 : 32;
    static constexpr int TPR = TILE / VW;                 // threads per tile row
    static constexpr int PASS = TILE / (EW_THREADS / TPR);
};
template <class T> __device__ __forceinline__ void trv_load(T (*sm)[TrV<T>::TILE + 1], const T* p, int64_t s0,
                                                          int64_t s1, int64_t i0, int64_t j0) {
    typedef TrV<T> V;
    const int tid = threadIdx.x;
    const int lane_v = (tid % V::TPR) * V::VW, line = tid / V::TPR;
    if (s0 == 1) {  // column-contiguous: a vector runs down VW rows of one column
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int c = line + k * (EW_THREADS / V::TPR), r = lane_v;
            const Vec16<T> v = ldv(p + (i0 + r) + (j0 + c) * s1, 0);
#pragma unroll
            for (int e = 0; e < V::VW; ++e) sm[r + e][c] = v.v[e];
        }
    } else {        // row-contiguous: a vector runs along VW columns of one row
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int r = line + k * (EW_THREADS / V::TPR), c = lane_v;
            const Vec16<T> v = ldv(p + (i0 + r) * s0 + (j0 + c), 0);
#pragma unroll
            for (int e = 0; e < V::VW; ++e) sm[r][c + e] = v.v[e];
        }
    }
}

template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_bin_trv(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef BinOp<OP, CD> Op;
    typedef typename Op::R R;
    typedef TrV<T> V;
    static_assert(sizeof(R) == sizeof(T), "the vector path stores results of the operand width");
    __shared__ T sa[V::TILE][V::TILE + 1], sb[V::TILE][V::TILE + 1];
    uint32_t bits = 0;
    const int64_t tr = d.shape[0] / V::TILE, tc = d.shape[1] / V::TILE;
    const T* pa = (const T*)d.a.p;
    const T* pb = (const T*)d.b.p;
    R* po = (R*)d.o;
    const bool ocol = d.so[0] == 1;
    const int tid = threadIdx.x;
    const int lane_v = (tid % V::TPR) * V::VW, line = tid / V::TPR;
    for (int64_t t = blockIdx.x; t < tr * tc; t += gridDim.x) {
        const int64_t i0 = (t / tc) * V::TILE, j0 = (t % tc) * V::TILE;
        trv_load<T>(sa, pa, d.a.st[0], d.a.st[1], i0, j0);
        trv_load<T>(sb, pb, d.b.st[0], d.b.st[1], i0, j0);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int m = line + k * (EW_THREADS / V::TPR);
            R r[V::VW];
#pragma unroll
            for (int e = 0; e < V::VW; ++e) {
                const int rr = ocol ? lane_v + e : m, cc = ocol ? m : lane_v + e;
                const T x = sa[rr][cc], y = sb[rr][cc];
                r[e] = Op::apply(x, y);
                if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r[e]);
            }
            R* dst = ocol ? po + (i0 + lane_v) + (j0 + m) * d.so[1] : po + (i0 + m) * d.so[0] + (j0 + lane_v);
            stv<R, V::VW>(dst, 0, r);
        }
        __syncthreads();
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// Tile kernel for exactly one operand laid out across the output (the other
// follows it): only that operand goes through shared memory; the other is
// read straight into registers at the output's positions; and both
// operands of the next tile are loaded while this tile is computed, so each
// thread keeps one tile of loads in flight through the arithmetic.
// the division family is register-heavy (112 registers for 4-byte types
// unbounded, two resident CTAs): ask for three resident CTAs for 4-byte
// types and four for 8-byte types
template <int OP, int CD> constexpr int trv1_min_ctas() {
    return (OP == OP_FLOOR_DIVIDE || OP == OP_REMAINDER || OP == OP_FMOD)
        ? (sizeof(typename DT<CD>::T) == 8 ? 4 : 3) : 1;
}

template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS, trv1_min_ctas<OP, CD>())
k_bin_trv1(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef BinOp<OP, CD> Op;
    typedef typename Op::R R;
    typedef TrV<T> V;
    static_assert(sizeof(R) == sizeof(T), "the vector path stores results of the operand width");
    __shared__ T st[V::TILE][V::TILE + 1];
    uint32_t bits = 0;
    const int64_t tc = d.shape[1] / V::TILE, nt = (d.shape[0] / V::TILE) * tc;
    const bool ocol = d.so[0] == 1;
    const bool swap = (d.a.st[0] == 1) == ocol;  // a follows the output: b is the one across
    const T* pt = (const T*)(swap ? d.b.p : d.a.p);
    const T* pd = (const T*)(swap ? d.a.p : d.b.p);
    const int64_t t0 = swap ? d.b.st[0] : d.a.st[0], t1 = swap ? d.b.st[1] : d.a.st[1];
    const int64_t q0 = swap ? d.a.st[0] : d.b.st[0], q1 = swap ? d.a.st[1] : d.b.st[1];
    R* po = (R*)d.o;
    const int tid = threadIdx.x;
    const int lane_v = (tid % V::TPR) * V::VW, line = tid / V::TPR;
    constexpr int LSTEP = EW_THREADS / V::TPR;
    // both operands of the next tile are loaded while this one is computed
    Vec16<T> rt[V::PASS], xn[V::PASS];
    auto fetch = [&](int64_t t) {
        const int64_t i0 = (t / tc) * V::TILE, j0 = (t % tc) * V::TILE;
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int w = line + k * LSTEP;
            rt[k] = (t0 == 1) ? ldv(pt + (i0 + lane_v) + (j0 + w) * t1, 0) : ldv(pt + (i0 + w) * t0 + (j0 + lane_v), 0);
            xn[k] = ocol ? ldv(pd + (i0 + lane_v) + (j0 + w) * q1, 0) : ldv(pd + (i0 + w) * q0 + (j0 + lane_v), 0);
        }
    };
    int64_t t = blockIdx.x;
    if (t < nt) fetch(t);
    for (; t < nt; t += gridDim.x) {
        Vec16<T> xd[V::PASS];
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int w = line + k * LSTEP;
            xd[k] = xn[k];
            if (t0 == 1) {
#pragma unroll
                for (int e = 0; e < V::VW; ++e) st[lane_v + e][w] = rt[k].v[e];
            } else {
#pragma unroll
                for (int e = 0; e < V::VW; ++e) st[w][lane_v + e] = rt[k].v[e];
            }
        }
        __syncthreads();
        const int64_t i0 = (t / tc) * V::TILE, j0 = (t % tc) * V::TILE;
        if (t + gridDim.x < nt) fetch(t + gridDim.x);
#pragma unroll
        for (int k = 0; k < V::PASS; ++k) {
            const int m = line + k * LSTEP;
            R r[V::VW];
            if constexpr (sizeof(T) == 8 && Op::FAST) {
                // float64 division: one pair at a time (measured faster
                // here than gathering the vector first)
#pragma unroll
                for (int e = 0; e < V::VW; ++e) {
                    const T vt = ocol ? st[lane_v + e][m] : st[m][lane_v + e];
                    const T vd = xd[k].v[e];
                    const T x = swap ? vd : vt, y = swap ? vt : vd;
                    r[e] = Op::apply(x, y);
                    if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r[e]);
                }
            } else {
                T xs[V::VW], ys[V::VW];
#pragma unroll
                for (int e = 0; e < V::VW; ++e) {
                    const T vt = ocol ? st[lane_v + e][m] : st[m][lane_v + e];
                    const T vd = xd[k].v[e];
                    xs[e] = swap ? vd : vt;
                    ys[e] = swap ? vt : vd;
                }
                bin_vec<OP, CD, FPE, V::VW>(xs, ys, r, bits);
            }
            R* dst = ocol ? po + (i0 + lane_v) + (j0 + m) * d.so[1] : po + (i0 + m) * d.so[0] + (j0 + lane_v);
            stv<R, V::VW>(dst, 0, r);
        }
        __syncthreads();
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// ---------------------------------------------------------------------------
// unary
// ---------------------------------------------------------------------------
template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_un_contig(const typename DT<CD>::T* __restrict__ a, typename UnOp<OP, CD>::R* __restrict__ o, int64_t n, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef typename UnOp<OP, CD>::R R;
    constexpr int N = Vec16<T>::N;
    constexpr int U = 2;
    uint32_t bits = 0;
    const int64_t nvec = n / N;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; v + (U - 1) * stride < nvec; v += U * stride) {
        Vec16<T> xa[U];
#pragma unroll
        for (int u = 0; u < U; ++u) xa[u] = ldv(a, v + u * stride);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            R r[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
                r[k] = UnOp<OP, CD>::apply(xa[u].v[k]);
                if constexpr (FPE) bits |= UnOp<OP, CD>::fpe(xa[u].v[k]);
            }
            stv<R, N>(o, v + u * stride, r);
        }
    }
    for (; v < nvec; v += stride) {
        Vec16<T> xa = ldv(a, v);
        R r[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r[k] = UnOp<OP, CD>::apply(xa.v[k]);
            if constexpr (FPE) bits |= UnOp<OP, CD>::fpe(xa.v[k]);
        }
        stv<R, N>(o, v, r);
    }
    for (int64_t i = nvec * N + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T x = a[i];
        o[i] = UnOp<OP, CD>::apply(x);
        if constexpr (FPE) bits |= UnOp<OP, CD>::fpe(x);
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

template <int OP, int CD, bool FPE>
__global__ void __launch_bounds__(EW_THREADS)
k_un_nd(EwDesc d, uint32_t* flags) {
    typedef typename DT<CD>::T T;
    typedef UnOp<OP, CD> Op;
    typedef typename Op::R R;
    uint32_t bits = 0;
    const int nd = d.nd;
    const int64_t inner = d.shape[nd - 1];
    const int64_t sa = d.a.st[nd - 1], so = d.so[nd - 1], sm = d.m.st[nd - 1];
    const bool has_m = d.m.p != nullptr;
    if (nd == 1 && !has_m && d.a.dt == CD && d.odt == Op::OUT_DT) {
        // one strided run in the loop dtype (a step-k slice): typed loads,
        // U in flight per thread before the arithmetic
        constexpr int U = sizeof(T) >= 8 ? 4 : 8;
        const T* pa = reinterpret_cast<const T*>(d.a.p);
        R* po = reinterpret_cast<R*>(d.o);
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        for (; i + (U - 1) * stride < d.n; i += U * stride) {
            T x[U];
#pragma unroll
            for (int u = 0; u < U; ++u) x[u] = ld_cs(pa + (i + u * stride) * sa);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const R r = Op::apply(x[u]);
                if constexpr (FPE) bits |= Op::fpe(x[u]);
                st_cs(po + (i + u * stride) * so, r);
            }
        }
        for (; i < d.n; i += stride) {
            const T x = pa[i * sa];
            if constexpr (FPE) bits |= Op::fpe(x);
            po[i * so] = Op::apply(x);
        }
        if constexpr (FPE) flush_flags(bits, flags);
        return;
    }
    auto one = [&](int64_t oa, int64_t oo, int64_t om) {
        T x = load_cast<CD>(d.a.p, oa, d.a.dt);
        R r = Op::apply(x);
        if constexpr (FPE) bits |= Op::fpe(x);
        if (has_m && !((const uint8_t*)d.m.p)[om]) return;
        store_cast<Op::OUT_DT>(d.o, oo, d.odt, r);
    };
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
                if (c < inner) one(base.a + c * sa, base.o + c * so, base.m + c * sm);
            }
        }
    } else {
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += stride) {
            Offs f = unravel(d, i, 0);
            one(f.a, f.o, f.m);
        }
    }
    if constexpr (FPE) flush_flags(bits, flags);
}

// Grid size for a grid-stride element-wise launch: enough CTAs to fill all
// 148 SMs at full occupancy, fewer for small problems.
inline int ew_grid(int64_t work_items) {
    int64_t want = (work_items + EW_THREADS - 1) / EW_THREADS;
    int64_t cap = (int64_t)sm_count() * 8;  // 8 resident 256-thread CTAs per SM
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

}  // namespace ionp
