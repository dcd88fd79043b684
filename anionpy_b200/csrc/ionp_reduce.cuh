// Reduction and argmin/argmax kernels (ufunc.reduce / argext hot path).
//
// Fold orders follow the reference exactly (ionp-core/src/ufunc.rs):
//  * float add on the "wide" run (the reduced axes that are the smallest-
//    stride axes of the whole array) is numpy's pairwise sum: recursive
//    halving at n/2 rounded down to a multiple of 8 until a block of <= 128,
//    each block summed by 8 strided accumulators combined as
//    ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), tail added in order
//    (pairwise_sum, ufunc.rs:6416-6448);
//  * "narrow" reduced axes fold sequentially in memory order, seeded with the
//    identity or initial (ufunc.rs:6658-6806);
//  * float16 add/multiply/subtract/divide widen to f32 on the wide run and
//    round to f16 per narrow step (ufunc.rs:6868-7089);
//  * everything else is a sequential fold in ascending-axis C order
//    (sequential_group, ufunc.rs:6546), in memory order for float multiply
//    (sequential_group_ordered, ufunc.rs:6583).
//
// Kernels:
//  k_red_row   : one output per thread group (1, 32 or 256 threads); the
//                group's elements form one strided run. The pairwise tree is
//                rebuilt on the device: each thread locates leaf blocks by
//                descending the split tree from the root, sums each with the
//                8 accumulators (16-byte vector loads on contiguous runs),
//                and parks the result in a shared-memory slot array laid out
//                as a perfect binary tree (a leaf at depth d with path p sits
//                at slot p << (D - d)); the tree is then combined level by
//                level, left operand first. Associative
//                ops (int add, max, bitwise, ...) reuse the same kernel: any
//                order-preserving bracketing gives identical bits for them.
//                Runs longer than one CTA's segment are cut at a fixed tree
//                depth K (every node above K is an interior node), each
//                subtree reduced by its own CTA into scratch, and the top K
//                levels combined by a second launch.
//  k_red_col   : one output per thread, sequential over the reduced offsets
//                (narrow axes, or any op without a pairwise loop); adjacent
//                threads own adjacent outputs so loads coalesce along the
//                kept axis.
//  k_red_gen   : one output per thread, the general wide x narrow nest with
//                several wide runs, for the layouts that need it.
//  k_red_masked: where= reductions (ufunc.rs:7213-7548), one output per thread.
//  k_argext_*  : argmin/argmax with (value, index) pairs, first occurrence on
//                ties and first NaN winning (ufunc.rs:8037-8206).
#pragma once
#include "ionp_scalar.cuh"
#include "ionp_internal.h"

namespace ionp {

constexpr int RD_MAXD = 8;
constexpr int RED_THREADS = 256;
constexpr int PW_BLOCK = 128;

// Reduction launch descriptor (by value).
struct RedDesc {
    const void* a;   // input, first element
    int32_t adt;     // input dtype (cast on load to the compute dtype)
    int32_t cd;      // compute dtype
    int32_t op;
    int64_t nout;    // outputs (product of kept dims)
    int32_t nk;      // kept dims, C order = output order
    int64_t kshape[RD_MAXD], kst[RD_MAXD], kost[RD_MAXD];
    // ROW: the group is one run of `w` elements at stride `ws`.
    int64_t w, ws;
    // COL / GEN: narrow dims in fold order (outermost first)
    int32_t nr;
    int64_t rshape[RD_MAXD], rst[RD_MAXD];
    // GEN: wide runs innermost first (runs[0] pairwise, runs[1..] outer)
    int32_t nw;
    int64_t wshape[RD_MAXD], wst[RD_MAXD];
    int32_t has_seed;
    uint64_t seed;   // bits of the seed in the compute dtype
    void* o;         // output first element
    int32_t odt;
    // split ROW (K > 0): partials scratch, nout x 2^K accumulators
    int32_t K;
    int32_t D;       // slot-tree depth of one segment
    int32_t Dw, Dl;  // wide-row staged kernel: window depth, leaf-slot depth
    void* scratch;
    // a device word a kernel sets when one of its bounded waits gives up
    // (null: none); the library reports it at the next synchronization
    uint32_t* err;
    // masked
    const uint8_t* m;
    int64_t mkst[RD_MAXD], mrst[RD_MAXD], mwst_raw[RD_MAXD];
    int32_t nwr;     // masked: raw (uncoalesced) wide dims, innermost last
    int64_t wrshape[RD_MAXD], wrst[RD_MAXD];
    int32_t pairwise;  // masked: float add family
};

// Loads of the only cast the reduction kernels do on the fly: add/multiply
// widening bool and narrower integers to int64/uint64
// (reduce_compute_dtype, ufunc.rs:2041-2078). Other casts are materialised.
template <int CD> __device__ __forceinline__ typename DT<CD>::T load_int_widen(const void* p, int64_t e, int sdt) {
    typedef typename DT<CD>::T T;
    switch (sdt) {
        case DT_BOOL: return (T)(((const uint8_t*)p)[e] != 0);
        case DT_I8: return (T)((const int8_t*)p)[e];
        case DT_I16: return (T)((const int16_t*)p)[e];
        case DT_I32: return (T)((const int32_t*)p)[e];
        case DT_U8: return (T)((const uint8_t*)p)[e];
        case DT_U16: return (T)((const uint16_t*)p)[e];
        case DT_U32: return (T)((const uint32_t*)p)[e];
        default: return ((const T*)p)[e];
    }
}

// Accumulation policy of the pairwise/tree kernels.
template <int OP, int CD, bool CASTLD = false> struct RPol {
    static constexpr bool F16W = (CD == DT_F16 && OP == OP_ADD);
    // float max/min pick the first NaN (and f16 the first of equal values) in
    // fold order, so their leaves take contiguous chunks per lane; the float
    // pairwise add needs the 8 interleaved accumulators; the integer, bool,
    // bitwise and logical folds are order-free.
    static constexpr bool CHUNK = dt_is_float(CD) && (OP == OP_MAXIMUM || OP == OP_MINIMUM);
    static constexpr int AD = F16W ? DT_F32 : CD;
    typedef typename DT<CD>::T T;
    typedef typename DT<AD>::T A;
    // 8 consecutive elements load as one or two 16-byte vectors: plain 4- and
    // 8-byte element types, and float16 widened to float32 after the load
    static constexpr bool VEC8 = !CASTLD && (F16W || sizeof(T) == 4 || sizeof(T) == 8);
    static __device__ __forceinline__ A fold(A x, A y) { return BinOp<OP, AD>::apply(x, y); }
    static __device__ __forceinline__ A load(const void* p, int64_t e, int sdt) {
        if constexpr (CASTLD) return load_int_widen<CD>(p, e, sdt);
        else if constexpr (F16W) return h2f(((const h16*)p)[e]);
        else return ((const T*)p)[e];
    }
    // the result of one output from its tree total
    static __device__ __forceinline__ T finish(A total, int has_seed, uint64_t seed_bits) {
        if constexpr (F16W) {
            h16 s = (h16)seed_bits;  // add always has a seed (0 or initial)
            return FOps<DT_F16>::add(s, f2h(total));
        } else {
            if (has_seed) {
                T s;
                memcpy(&s, &seed_bits, sizeof(T));
                return BinOp<OP, CD>::apply(s, total);
            }
            return total;
        }
    }
};

// IEEE add without the NaN payload rule: equal to the engine's add whenever
// the result is not NaN.
template <class T> __device__ __forceinline__ T plain_sum(T x, T y) {
    if constexpr (sizeof(T) == 8) return __dadd_rn(x, y);
    else return __fadd_rn(x, y);
}

__host__ __device__ __forceinline__ int64_t pw_split(int64_t len) {
    int64_t n2 = len / 2;
    return n2 - n2 % 8;
}

// Offsets of output index `o` over the kept dims: input and output.
__device__ __forceinline__ void kept_offsets(const RedDesc& d, int64_t o, int64_t* in_off, int64_t* out_off) {
    if (d.nk == 1) {  // o < kshape[0]: no division
        *in_off = o * d.kst[0];
        *out_off = o * d.kost[0];
        return;
    }
    int64_t a = 0, b = 0;
    for (int k = d.nk - 1; k >= 0; --k) {
        int64_t s = d.kshape[k];
        int64_t q = o / s;
        int64_t id = o - q * s;
        o = q;
        a += id * d.kst[k];
        b += id * d.kost[k];
    }
    *in_off = a;
    *out_off = b;
}

// Descend K levels of the split tree of a run of n along `path`.
__device__ __forceinline__ void seg_of(int64_t n, int K, int64_t path, int64_t* off, int64_t* len) {
    int64_t o = 0, l = n;
    for (int k = K - 1; k >= 0; --k) {
        int64_t n2 = pw_split(l);
        if ((path >> k) & 1) { o += n2; l -= n2; } else { l = n2; }
    }
    *off = o;
    *len = l;
}

// Eight consecutive run elements [e, e+8) as accumulator values, loaded as
// 16-byte vectors (the caller checked alignment).
template <class P>
__device__ __forceinline__ void load8_vec(const void* pa, int64_t e, typename P::A (&x)[8]) {
    typedef typename P::T T;
    if constexpr (P::F16W) {
        uint4 u = __ldg(reinterpret_cast<const uint4*>(reinterpret_cast<const h16*>(pa) + e));
        h16 h[8];
        memcpy(h, &u, 16);
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = h2f(h[k]);
    } else if constexpr (sizeof(T) == 4) {
        const uint4* q = reinterpret_cast<const uint4*>(reinterpret_cast<const T*>(pa) + e);
        uint4 u0 = __ldg(q), u1 = __ldg(q + 1);
        memcpy(&x[0], &u0, 16);
        memcpy(&x[4], &u1, 16);
    } else {
        const uint4* q = reinterpret_cast<const uint4*>(reinterpret_cast<const T*>(pa) + e);
        uint4 u0 = __ldg(q), u1 = __ldg(q + 1), u2 = __ldg(q + 2), u3 = __ldg(q + 3);
        memcpy(&x[0], &u0, 16);
        memcpy(&x[2], &u1, 16);
        memcpy(&x[4], &u2, 16);
        memcpy(&x[6], &u3, 16);
    }
}

// One thread sums the leaf block [off, off+len) (len <= 128) of a run with
// pairwise_sum's leaf loop (ufunc.rs:6416-6448): fewer than 8 elements fold
// in order; otherwise 8 interleaved accumulators (r[k] takes elements
// k, k+8, ...), combined ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), then the
// len % 8 tail added in order. Float max/min (P::CHUNK) fold strictly left
// to right, which their first-NaN rule needs. Contiguous runs load 8
// elements per 16-byte vector pair.
template <class P>
__device__ __forceinline__ typename P::A leaf_thread(const void* pa, int adt, int64_t base, int64_t ws, int64_t off,
                                                     int64_t len) {
    typedef typename P::A A;
    typedef typename P::T T;
    const int64_t e0 = base + off * ws;
    if constexpr (P::CHUNK && P::VEC8) {
        // order-sensitive folds on contiguous runs: vector loads, strictly
        // left-to-right fold
        if (len >= 8 && ws == 1 && ((reinterpret_cast<uintptr_t>(pa) + (uint64_t)e0 * sizeof(T)) & 15) == 0) {
            constexpr int GC = sizeof(T) == 8 ? 1 : 2;
            const int64_t lim = len - len % 8;
            A x0[8];
            load8_vec<P>(pa, e0, x0);
            A r = x0[0];
#pragma unroll
            for (int k = 1; k < 8; ++k) r = P::fold(r, x0[k]);
            for (int64_t i = 8; i < lim; i += 8 * GC) {
                A x[GC][8];
#pragma unroll
                for (int g = 0; g < GC; ++g)
                    if (i + 8 * g < lim) load8_vec<P>(pa, e0 + i + 8 * g, x[g]);
#pragma unroll
                for (int g = 0; g < GC; ++g)
                    if (i + 8 * g < lim) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) r = P::fold(r, x[g][k]);
                    }
            }
            for (int64_t i = lim; i < len; ++i) r = P::fold(r, P::load(pa, e0 + i, adt));
            return r;
        }
    }
    if (P::CHUNK || len < 8) {
        A r = P::load(pa, e0, adt);
        int64_t i = 1;
        for (; i + 8 <= len; i += 8) {
            A x[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = P::load(pa, e0 + (i + k) * ws, adt);
#pragma unroll
            for (int k = 0; k < 8; ++k) r = P::fold(r, x[k]);
        }
        for (; i < len; ++i) r = P::fold(r, P::load(pa, e0 + i * ws, adt));
        return r;
    }
    const int64_t lim = len - len % 8;
    A r[8];
    bool vec = false;
    if constexpr (P::VEC8) vec = ws == 1 && ((reinterpret_cast<uintptr_t>(pa) + (uint64_t)e0 * sizeof(T)) & 15) == 0;
    if (vec) {
        if constexpr (P::VEC8) {
            // 64 bytes of loads in flight per chunk: two 8-element groups of
            // 4-byte (or widened 2-byte) elements, one of 8-byte elements
            constexpr int GC = sizeof(T) == 8 ? 1 : 2;
            load8_vec<P>(pa, e0, r);
            for (int64_t i = 8; i < lim; i += 8 * GC) {
                A x[GC][8];
#pragma unroll
                for (int g = 0; g < GC; ++g)
                    if (i + 8 * g < lim) load8_vec<P>(pa, e0 + i + 8 * g, x[g]);
#pragma unroll
                for (int g = 0; g < GC; ++g)
                    if (i + 8 * g < lim) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) r[k] = P::fold(r[k], x[g][k]);
                    }
            }
        }
    } else {
        constexpr int GS = sizeof(A) == 8 ? 1 : 2;
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = P::load(pa, e0 + k * ws, adt);
        for (int64_t i = 8; i < lim; i += 8 * GS) {
            A x[GS][8];
#pragma unroll
            for (int g = 0; g < GS; ++g)
                if (i + 8 * g < lim) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) x[g][k] = P::load(pa, e0 + (i + 8 * g + k) * ws, adt);
                }
#pragma unroll
            for (int g = 0; g < GS; ++g)
                if (i + 8 * g < lim) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) r[k] = P::fold(r[k], x[g][k]);
                }
        }
    }
    A res = P::fold(P::fold(P::fold(r[0], r[1]), P::fold(r[2], r[3])), P::fold(P::fold(r[4], r[5]), P::fold(r[6], r[7])));
    for (int64_t i = lim; i < len; ++i) res = P::fold(res, P::load(pa, e0 + i * ws, adt));
    return res;
}

// Barrier over one TPR-thread group (a CTA-wide barrier when TPR > 32).
template <int TPR> __device__ __forceinline__ void group_sync() {
    if constexpr (TPR > 32) __syncthreads();
    else if constexpr (TPR == 32) __syncwarp();
    else __syncwarp(((1u << TPR) - 1u) << ((threadIdx.x & 31) & ~(unsigned)(TPR - 1)));
}

// One output group of TPR threads reduces the run [seg_off, seg_off+n) of
// output row `base` with the pairwise tree, one leaf per thread: every
// thread takes the leaf blocks that start in its 64-element candidate
// windows (each leaf, 64..128 elements long, starts in exactly one window),
// sums it with leaf_thread and parks it in the perfect-binary-tree slot
// array; the slots are then combined level by level, left operand first.
template <class P, int TPR>
__device__ typename P::A group_tree_t(const void* pa, int adt, int64_t aws, int64_t base, int64_t seg_off, int64_t n,
                                      int D, typename P::A* slots, uint8_t* valid, int t) {
    typedef typename P::A A;
    if (n <= PW_BLOCK) {
        A r{};
        if (t == 0 && n > 0) r = leaf_thread<P>(pa, adt, base, aws, seg_off, n);
        return r;
    }
    const int nslots = 1 << D;
    for (int s = t; s < nslots; s += TPR) valid[s] = 0;
    group_sync<TPR>();
    const int64_t ncand = (n + 63) / 64;
    for (int64_t c = t; c < ncand; c += TPR) {
        const int64_t m = c * 64;
        int64_t off = 0, len = n, path = 0;
        int depth = 0;
        while (len > PW_BLOCK) {
            int64_t n2 = pw_split(len);
            path <<= 1;
            depth++;
            if (m < off + n2) len = n2; else { off += n2; len -= n2; path |= 1; }
        }
        if (off > m - 64) {
            A r = leaf_thread<P>(pa, adt, base, aws, seg_off + off, len);
            int s = (int)(path << (D - depth));
            slots[s] = r;
            valid[s] = 1;
        }
    }
    group_sync<TPR>();
    for (int lvl = D - 1; lvl >= 0; --lvl) {
        const int half = 1 << (D - 1 - lvl), step = half * 2;
        for (int s = t * step; s < nslots; s += TPR * step) {
            if (valid[s + half]) slots[s] = P::fold(slots[s], slots[s + half]);
        }
        group_sync<TPR>();
    }
    return slots[0];
}

// ROW kernel. Tasks = nout x 2^K; each TPR-thread group takes one task.
template <int OP, int CD, int TPR, bool CASTLD>
__global__ void __launch_bounds__(RED_THREADS, 4) k_red_row(RedDesc d) {
    typedef RPol<OP, CD, CASTLD> P;
    typedef typename P::A A;
    typedef typename P::T T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int GROUPS = RED_THREADS / TPR;
    const int g = threadIdx.x / TPR, t = threadIdx.x % TPR;
    const int nslots = TPR >= 32 ? (1 << d.D) : 1;
    A* slots = reinterpret_cast<A*>(smem_raw) + (size_t)g * nslots;
    uint8_t* valid = reinterpret_cast<uint8_t*>(reinterpret_cast<A*>(smem_raw) + (size_t)GROUPS * nslots) + (size_t)g * nslots;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t ntasks = d.nout * nseg;
    // all groups of a CTA iterate the same number of times (TPR > 32 syncs)
    for (int64_t t0 = (int64_t)blockIdx.x * GROUPS; t0 < ntasks; t0 += (int64_t)gridDim.x * GROUPS) {
        int64_t task = t0 + g;
        bool live = task < ntasks;
        int64_t o = live ? task / nseg : 0, sg = live ? task % nseg : 0;
        int64_t in_off, out_off;
        kept_offsets(d, o, &in_off, &out_off);
        int64_t soff, slen;
        seg_of(d.w, d.K, sg, &soff, &slen);
        if (!live) slen = 0;
        A r{};
        if constexpr (TPR == 1) {
            if (slen > 0) r = leaf_thread<P>(d.a, d.adt, in_off, d.ws, soff, slen);
        } else if constexpr (TPR > 32) {
            r = group_tree_t<P, TPR>(d.a, d.adt, d.ws, in_off, soff, slen, d.D, slots, valid, t);
        } else {
            if (slen > 0) r = group_tree_t<P, TPR>(d.a, d.adt, d.ws, in_off, soff, slen, d.D, slots, valid, t);
        }
        if (live && t == 0) {
            if (d.K == 0) store_cast<CD>(d.o, out_off, d.odt, P::finish(r, d.has_seed, d.seed));
            else reinterpret_cast<A*>(d.scratch)[task] = r;
        }
        if constexpr (TPR > 32) __syncthreads();
    }
}

// Top of a split tree: per output, combine its 2^K partials as a perfect
// binary tree (adjacent pairs, left operand first), then seed and store.
// The partials are folded in chunks of 2^KC (each chunk is a perfect
// subtree of the same tree); the 2^(K - KC) chunk results then fold as the
// tree's top levels, so shared memory stays at 2^(K - KC) values plus one per
// warp for any K <= 2 TOP_CHUNK_LOG.
constexpr int TOP_CHUNK_LOG = 11;
__host__ __device__ constexpr int top_chunk_log(int K) { return K < TOP_CHUNK_LOG ? K : TOP_CHUNK_LOG; }
template <class A>
__host__ __device__ constexpr size_t row_top_smem(int K) {
    return (((size_t)1 << (K - top_chunk_log(K))) + RED_THREADS / 32) * sizeof(A);
}
template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS) k_red_row_top(RedDesc d) {
    typedef RPol<OP, CD> P;
    typedef typename P::A A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kc = top_chunk_log(d.K);
    const int csize = 1 << kc, nchunk = 1 << (d.K - kc);
    A* top = reinterpret_cast<A*>(smem_raw);          // nchunk chunk totals
    A* wsum = top + nchunk;                            // RED_THREADS / 32 warp totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nseg = (int64_t)1 << d.K;
    for (int64_t o = blockIdx.x; o < d.nout; o += gridDim.x) {
        for (int c = 0; c < nchunk; ++c) {
            const A* part = reinterpret_cast<const A*>(d.scratch) + o * nseg + (int64_t)c * csize;
            // thread t folds partials [t m, (t + 1) m) in registers (m a power of
            // two), warps fold 32 such blocks by shuffles, then the warp totals
            // fold in one thread: each step joins adjacent perfect subtrees,
            // left operand first, so the whole is the chunk's perfect tree
            const int m = csize > RED_THREADS ? csize / RED_THREADS : 1;
            const int active = csize > RED_THREADS ? RED_THREADS : csize;
            A v{};
            if ((int)threadIdx.x < active) {
                A x[8];
                for (int i = 0; i < m; ++i) x[i] = part[threadIdx.x * m + i];
                for (int h = 1; h < m; h <<= 1)
                    for (int i = 0; i < m; i += 2 * h) x[i] = P::fold(x[i], x[i + h]);
                v = x[0];
            }
            const int wl = active < 32 ? active : 32;  // leaves of each warp's tree
            for (int h = 1; h < wl; h <<= 1) {
                const A ov = __shfl_down_sync(0xffffffffu, v, h);
                if ((lane & (2 * h - 1)) == 0 && lane + h < wl) v = P::fold(v, ov);
            }
            if (lane == 0) wsum[warp] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                const int nw = active / 32 > 1 ? active / 32 : 1;
                for (int h = 1; h < nw; h <<= 1)
                    for (int i = 0; i < nw; i += 2 * h) wsum[i] = P::fold(wsum[i], wsum[i + h]);
                top[c] = wsum[0];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            for (int h = 1; h < nchunk; h <<= 1)
                for (int i = 0; i < nchunk; i += 2 * h) top[i] = P::fold(top[i], top[i + h]);
            int64_t in_off, out_off;
            kept_offsets(d, o, &in_off, &out_off);
            store_cast<CD>(d.o, out_off, d.odt, P::finish(top[0], d.has_seed, d.seed));
        }
        __syncthreads();
    }
}

// Top of a split with at most 32 parts of an order-dependent fold (float
// add): one thread per output folds its 2^K partials as the perfect tree the
// K split levels form, left operand first, all loads independent (the tree
// unrolled at compile time), and applies the seed.
template <class P, int K> struct TopTree {
    static __device__ __forceinline__ typename P::A go(const typename P::A* p) {
        if constexpr (K == 0) return p[0];
        else return P::fold(TopTree<P, K - 1>::go(p), TopTree<P, K - 1>::go(p + (1 << (K - 1))));
    }
};
template <int OP, int CD, int K>
__global__ void __launch_bounds__(RED_THREADS) k_red_row_top_tree(RedDesc d) {
    typedef RPol<OP, CD> P;
    typedef typename P::A A;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += (int64_t)gridDim.x * blockDim.x) {
        const A v = TopTree<P, K>::go(reinterpret_cast<const A*>(d.scratch) + (o << K));
        int64_t in_off, out_off;
        kept_offsets(d, o, &in_off, &out_off);
        store_cast<CD>(d.o, out_off, d.odt, P::finish(v, d.has_seed, d.seed));
    }
}

// Top of a split with few parts of an order-free fold: one thread per
// output folds its 2^K partials left to right (equal to the tree for these
// ops) and applies the seed.
template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS) k_red_row_top_small(RedDesc d) {
    typedef RPol<OP, CD> P;
    typedef typename P::A A;
    const int64_t nseg = (int64_t)1 << d.K;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += (int64_t)gridDim.x * blockDim.x) {
        const A* part = reinterpret_cast<const A*>(d.scratch) + o * nseg;
        A v = part[0];
        for (int64_t s = 1; s < nseg; ++s) v = P::fold(v, part[s]);
        int64_t in_off, out_off;
        kept_offsets(d, o, &in_off, &out_off);
        store_cast<CD>(d.o, out_off, d.odt, P::finish(v, d.has_seed, d.seed));
    }
}

// Signed-integer key of a float's bits, in the order of the values with -0
// below +0 (NaN excluded), and back.
__device__ __forceinline__ int32_t fkey(float v) { const int32_t k = (int32_t)fb(v); return k < 0 ? k ^ 0x7FFFFFFF : k; }
__device__ __forceinline__ int64_t fkey(double v) { const int64_t k = (int64_t)db(v); return k < 0 ? k ^ 0x7FFFFFFFFFFFFFFFll : k; }
__device__ __forceinline__ float fkey_inv(int32_t k) { return bf((uint32_t)(k < 0 ? k ^ 0x7FFFFFFF : k)); }
__device__ __forceinline__ double fkey_inv(int64_t k) { return bd((uint64_t)(k < 0 ? k ^ 0x7FFFFFFFFFFFFFFFll : k)); }

// One batch of a column fold in order: float add sums plainly and replays
// the batch with the engine's NaN rule only when the sum turns NaN (once the
// accumulator is a quiet NaN no later add changes it); float max/min fold a
// NaN-free batch as an integer max/min of order keys.
template <int OP, int CD, int U>
__device__ __forceinline__ void col_fold_batch(typename DT<CD>::T& acc, const typename DT<CD>::T (&x)[U]) {
    typedef typename DT<CD>::T T;
    if constexpr ((OP == OP_MAXIMUM || OP == OP_MINIMUM) && (CD == DT_F32 || CD == DT_F64)) {
        // Without a NaN, float_max / float_min (ufunc.rs:2402-2436) fold to
        // the largest / smallest value with -0 below +0 (their tie rule):
        // an integer max / min of the keys. A batch with a NaN, or a NaN
        // accumulator, folds element by element with the NaN rules.
        bool nan = acc != acc;
#pragma unroll
        for (int u = 0; u < U; ++u) nan |= x[u] != x[u];
        if (!nan) {
            auto k = fkey(acc);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const auto ku = fkey(x[u]);
                k = OP == OP_MAXIMUM ? (ku > k ? ku : k) : (ku < k ? ku : k);
            }
            acc = fkey_inv(k);
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) acc = BinOp<OP, CD>::apply(acc, x[u]);
        }
    } else if constexpr (OP == OP_ADD && (CD == DT_F32 || CD == DT_F64)) {
        if (acc == acc) {
            T r = acc;
#pragma unroll
            for (int u = 0; u < U; ++u) r = plain_sum(r, x[u]);
            if (r != r) {
                r = acc;
#pragma unroll
                for (int u = 0; u < U; ++u) r = BinOp<OP, CD>::apply(r, x[u]);
            }
            acc = r;
        } else {
            acc = BinOp<OP, CD>::apply(acc, x[0]);  // quiets a signaling NaN once
        }
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u) acc = BinOp<OP, CD>::apply(acc, x[u]);
    }
}

// COL kernel: sequential fold per output over the narrow dims (fold order),
// U loads in flight per thread (64 when the outputs are too few for 16 to
// keep HBM busy).
template <int OP, int CD, bool CASTLD, int U = 16>
__global__ void __launch_bounds__(RED_THREADS) k_red_col(RedDesc d) {
    typedef typename DT<CD>::T T;
    typedef RPol<OP, CD, CASTLD> P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t total = 1;
    for (int k = 0; k < d.nr; ++k) total *= d.rshape[k];
    const int64_t rs_in = d.nr > 0 ? d.rst[d.nr - 1] : 0;
    const int64_t rn_in = d.nr > 0 ? d.rshape[d.nr - 1] : 1;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += stride) {
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        bool have = d.has_seed;
        T acc;
        memcpy(&acc, &d.seed, sizeof(T));
        // walk the narrow dims: outer dims by odometer, innermost unrolled
        int64_t idx[RD_MAXD] = {0};
        int64_t outer_off = 0;
        for (int64_t done = 0; done < total; done += rn_in) {
            const int64_t b0 = base + outer_off;
            int64_t j = 0;
            if (!have && rn_in > 0) {
                if constexpr (CASTLD) acc = load_int_widen<CD>(d.a, b0, d.adt);
                else acc = ((const T*)d.a)[b0];
                have = true;
                j = 1;
            }
            for (; j + U <= rn_in; j += U) {
                T x[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if constexpr (CASTLD) x[u] = load_int_widen<CD>(d.a, b0 + (j + u) * rs_in, d.adt);
                    else x[u] = ((const T*)d.a)[b0 + (j + u) * rs_in];
                }
                // float add: plain adds, replayed with the engine's NaN
                // rule when the block's sum turns NaN; float max/min: an
                // integer max/min of order keys when the block has no NaN
                col_fold_batch<OP, CD, U>(acc, x);
            }
            for (; j < rn_in; ++j) {
                T x;
                if constexpr (CASTLD) x = load_int_widen<CD>(d.a, b0 + j * rs_in, d.adt);
                else x = ((const T*)d.a)[b0 + j * rs_in];
                if (!have) { acc = x; have = true; }
                else acc = BinOp<OP, CD>::apply(acc, x);
            }
            for (int k = d.nr - 2; k >= 0; --k) {
                idx[k]++;
                outer_off += d.rst[k];
                if (idx[k] < d.rshape[k]) break;
                outer_off -= d.rst[k] * d.rshape[k];
                idx[k] = 0;
            }
        }
        store_cast<CD>(d.o, out_off, d.odt, acc);
    }
}

// COL kernel, pipelined: one narrow axis, input in the loop dtype, too few
// outputs for one batch of loads per thread to keep HBM busy. One thread per
// output folds its column in order; its loads come in batches of U held in
// two register buffers, the next batch issued before the current one is
// folded, so U to 2U loads stay in flight per thread through the fold.
// One-warp CTAs, so the warps spread evenly over the SMs (32768 outputs are
// 1024 warps: 6 or 7 per SM, where 128-thread CTAs put 4 on some SMs and 8
// on others).
constexpr int COLP_THREADS = 32;
template <int OP, int CD, int U>
__global__ void __launch_bounds__(COLP_THREADS) k_red_col_pipe(RedDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t n = d.rshape[0], rs = d.rst[0];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += stride) {
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        const T* p = reinterpret_cast<const T*>(d.a) + base;
        T acc;
        memcpy(&acc, &d.seed, sizeof(T));
        int64_t j = 0;
        if (!d.has_seed && n > 0) { acc = p[0]; j = 1; }
        const int64_t nb = (n - j) / U;
        T xa[U], xb[U];
        if (nb > 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) xa[u] = p[(j + u) * rs];
            int64_t b = 0;
            for (; b + 2 <= nb; b += 2) {
                const T* q = p + (j + (b + 1) * U) * rs;
#pragma unroll
                for (int u = 0; u < U; ++u) xb[u] = q[u * rs];
                col_fold_batch<OP, CD, U>(acc, xa);
                if (b + 2 < nb) {
                    const T* q2 = q + U * rs;
#pragma unroll
                    for (int u = 0; u < U; ++u) xa[u] = q2[u * rs];
                }
                col_fold_batch<OP, CD, U>(acc, xb);
            }
            if (b < nb) col_fold_batch<OP, CD, U>(acc, xa);
        }
        for (int64_t i = j + nb * U; i < n; ++i) acc = BinOp<OP, CD>::apply(acc, p[i * rs]);
        store_cast<CD>(d.o, out_off, d.odt, acc);
    }
}

// COL kernel, split: one narrow axis folded by an order-free (associative)
// op. Too few outputs to keep HBM busy with one thread each, so the axis is
// cut into 2^K contiguous parts; task t folds part t / nout of output
// t % nout (adjacent threads, adjacent outputs) in order with 16 loads in
// flight, and k_red_row_top folds the parts in order and applies the seed.
template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS) k_red_col_split(RedDesc d) {
    typedef typename DT<CD>::T T;
    const int64_t P = (int64_t)1 << d.K;
    const int64_t len = d.rshape[0], rs = d.rst[0];
    const int64_t ntask = d.nout * P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask; t += stride) {
        const int64_t part = t / d.nout, o = t - part * d.nout;
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        const int64_t r0 = part * len / P, r1 = (part + 1) * len / P;
        const T* p = (const T*)d.a + base;
        T acc = p[r0 * rs];
        const int64_t j = r0 + 1;
        // batches of 16 loads in two register buffers, the next issued
        // before the current one is folded
        constexpr int U = 16;
        const int64_t nb = (r1 - j) / U;
        T xa[U], xb[U];
        if (nb > 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) xa[u] = p[(j + u) * rs];
            int64_t b = 0;
            for (; b + 2 <= nb; b += 2) {
                const T* q = p + (j + (b + 1) * U) * rs;
#pragma unroll
                for (int u = 0; u < U; ++u) xb[u] = q[u * rs];
                col_fold_batch<OP, CD, U>(acc, xa);
                if (b + 2 < nb) {
#pragma unroll
                    for (int u = 0; u < U; ++u) xa[u] = q[(U + u) * rs];
                }
                col_fold_batch<OP, CD, U>(acc, xb);
            }
            if (b < nb) {
                col_fold_batch<OP, CD, U>(acc, xa);
            }
        }
        for (int64_t k = j + nb * U; k < r1; ++k) acc = BinOp<OP, CD>::apply(acc, p[k * rs]);
        reinterpret_cast<T*>(d.scratch)[o * P + part] = acc;
    }
}

// 16-byte asynchronous global -> shared copies (cp.async, L2-only caching).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// COL kernel, staged: one narrow axis, contiguous kept axis. A CTA owns the
// outputs of one 128-byte column slice (32 float32 / 16 float64 columns);
// all 256 threads stream 64-row stages of it into a 3-stage shared-memory
// ring with cp.async while one warp folds each column sequentially in row
// order (the narrow fold of ufunc.rs:6748-6795 / sequential_group). Two
// stages are in flight while the third is folded, and seven such CTAs per
// SM keep HBM busy even when the outputs are too few for one thread each
// to hide the latency.
constexpr int COLST_ROWS = 64;    // rows per stage
constexpr int COLST_STAGES = 3;
constexpr int COLST_CTAS = 7;     // resident CTAs per SM the kernel is sized for
template <class T> constexpr int colst_cols() { return 128 / (int)sizeof(T); }
template <class T> constexpr size_t colst_smem() { return (size_t)COLST_STAGES * COLST_ROWS * 128; }

template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS, COLST_CTAS) k_red_col_staged(RedDesc d) {
    typedef typename DT<CD>::T T;
    constexpr int ES = (int)sizeof(T);
    constexpr int VE = 16 / ES;                 // elements per 16-byte chunk
    constexpr int COLS = colst_cols<T>();       // columns per CTA (one 128-byte slice)
    constexpr int CPR = COLS / VE;              // chunks per row: 8
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    const int64_t ncols = d.kshape[0];
    const int64_t rows = d.rshape[0];
    const int64_t rstride = d.rst[0];
    const T* a = reinterpret_cast<const T*>(d.a);
    const int64_t nst = (rows + COLST_ROWS - 1) / COLST_ROWS;
    const int64_t ntiles = (ncols + COLS - 1) / COLS;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t c0 = tile * COLS;
        auto issue = [&](int64_t st) {
            if (st < nst) {
                T* sb = buf + (st % COLST_STAGES) * COLST_ROWS * COLS;
                for (int q = threadIdx.x; q < COLST_ROWS * CPR; q += RED_THREADS) {
                    const int r = q / CPR, ch = q - r * CPR;
                    const int64_t row = st * COLST_ROWS + r, col = c0 + (int64_t)ch * VE;
                    if (row < rows && col < ncols) cp_async16(sb + r * COLS + ch * VE, a + row * rstride + col);
                }
            }
            cp_async_commit();  // empty groups keep the group count uniform
        };
        for (int st = 0; st < COLST_STAGES - 1; ++st) issue(st);
        T acc;
        memcpy(&acc, &d.seed, sizeof(T));
        bool have = d.has_seed != 0;
        const int64_t my = c0 + threadIdx.x;
        const bool owner = threadIdx.x < COLS && my < ncols;
        for (int64_t st = 0; st < nst; ++st) {
            issue(st + COLST_STAGES - 1);
            cp_async_wait<COLST_STAGES - 1>();
            __syncthreads();
            if (owner) {
                const T* sb = buf + (st % COLST_STAGES) * COLST_ROWS * COLS + threadIdx.x;
                const int nr = (int)(rows - st * COLST_ROWS < COLST_ROWS ? rows - st * COLST_ROWS : COLST_ROWS);
                int r = 0;
                if (!have) { acc = sb[0]; have = true; r = 1; }
                for (; r + 8 <= nr; r += 8) {
                    T x[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) x[u] = sb[(r + u) * COLS];
                    if constexpr (OP == OP_ADD && (CD == DT_F32 || CD == DT_F64)) {
                        // plain adds, replayed with the NaN rule only when
                        // the block's sum turns NaN; a NaN sum stays as is
                        if (acc == acc) {
                            T t = acc;
#pragma unroll
                            for (int u = 0; u < 8; ++u) t = plain_sum(t, x[u]);
                            if (t != t) {
                                t = acc;
#pragma unroll
                                for (int u = 0; u < 8; ++u) t = BinOp<OP, CD>::apply(t, x[u]);
                            }
                            acc = t;
                        } else {
                            acc = BinOp<OP, CD>::apply(acc, x[0]);  // quiets a signaling NaN once
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < 8; ++u) acc = BinOp<OP, CD>::apply(acc, x[u]);
                    }
                }
                for (; r < nr; ++r) acc = BinOp<OP, CD>::apply(acc, sb[r * COLS]);
            }
            __syncthreads();
        }
        if (owner) store_cast<CD>(d.o, my * d.kost[0], d.odt, acc);
    }
}

// ---------------------------------------------------------------------------
// Per-thread pairwise sum (iterative, explicit stack) for the general paths.
// get(i) returns element i of the run as the accumulator type.
// ---------------------------------------------------------------------------
template <class A, class Get, class Fold>
__device__ A pw_thread(Get get, int64_t n, Fold fold) {
    auto leaf = [&](int64_t b, int64_t len) -> A {
        if (len < 8) {
            A r = get(b);
            for (int64_t i = 1; i < len; ++i) r = fold(r, get(b + i));
            return r;
        }
        A r[8];
        for (int k = 0; k < 8; ++k) r[k] = get(b + k);
        int64_t i = 8;
        for (; i < len - len % 8; i += 8)
            for (int k = 0; k < 8; ++k) r[k] = fold(r[k], get(b + i + k));
        A res = fold(fold(fold(r[0], r[1]), fold(r[2], r[3])), fold(fold(r[4], r[5]), fold(r[6], r[7])));
        for (; i < len; ++i) res = fold(res, get(b + i));
        return res;
    };
    if (n <= PW_BLOCK) return leaf(0, n);
    // post-order walk; frame: node (b, len), state 0 = descend left,
    // 1 = descend right (left value saved), 2 = combine
    int64_t fb_[48], fl_[48];
    A fv[48];
    uint8_t fs[48];
    int sp = 0;
    fb_[0] = 0; fl_[0] = n; fs[0] = 0;
    A ret{};
    while (sp >= 0) {
        int64_t b = fb_[sp], len = fl_[sp];
        if (len <= PW_BLOCK) {
            ret = leaf(b, len);
            --sp;
            continue;
        }
        int64_t n2 = pw_split(len);
        if (fs[sp] == 0) {
            fs[sp] = 1;
            ++sp; fb_[sp] = b; fl_[sp] = n2; fs[sp] = 0;
        } else if (fs[sp] == 1) {
            fv[sp] = ret;
            fs[sp] = 2;
            ++sp; fb_[sp] = b + n2; fl_[sp] = len - n2; fs[sp] = 0;
        } else {
            ret = fold(fv[sp], ret);
            --sp;
        }
    }
    return ret;
}

// GEN kernel: one output per thread, the full narrow x wide nest.
// float add (f32/f64): reduce_axis_pairwise_narrow_wide (ufunc.rs:6658).
// float16 add/mul/sub/div: reduce_axis_f16_narrow_wide (ufunc.rs:6868).
template <int OP, int CD>
__global__ void __launch_bounds__(128) k_red_gen(RedDesc d) {
    typedef typename DT<CD>::T T;
    constexpr bool F16 = CD == DT_F16;
    typedef typename std::conditional<F16, float, T>::type A;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t ntotal = 1;
    for (int k = 0; k < d.nr; ++k) ntotal *= d.rshape[k];
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += stride) {
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        auto ld = [&](int64_t e) -> A {
            if constexpr (F16) return h2f(((const h16*)d.a)[e]);
            else return ((const T*)d.a)[e];
        };
        auto afold = [&](A x, A y) -> A {
            if constexpr (F16) return BinOp<OP, DT_F32>::apply(x, y);
            else return BinOp<OP, CD>::apply(x, y);
        };
        // pairwise_group (ufunc.rs:6504): inner run pairwise, outer runs
        // folded sequentially in NdIter order over runs[1..] (runs[1] slowest)
        auto wide_pairwise = [&](int64_t wb) -> A {
            if (d.nw == 0) return ld(wb);
            const int64_t isz = d.wshape[0], ist = d.wst[0];
            auto inner = [&](int64_t b) { return pw_thread<A>([&](int64_t i) { return ld(b + ist * i); }, isz, afold); };
            if (d.nw == 1) return inner(wb);
            int64_t nouter = 1;
            for (int k = 1; k < d.nw; ++k) nouter *= d.wshape[k];
            A acc{};
            for (int64_t q = 0; q < nouter; ++q) {
                int64_t rem = q, off = 0;
                for (int k = d.nw - 1; k >= 1; --k) {
                    int64_t id = rem % d.wshape[k];
                    rem /= d.wshape[k];
                    off += id * d.wst[k];
                }
                A v = inner(wb + off);
                acc = q == 0 ? v : afold(acc, v);
            }
            return acc;
        };
        // sequential over the wide elements in C order (outermost run first)
        auto wide_seq = [&](int64_t wb, bool seeded, A s) -> A {
            int64_t nel = 1;
            for (int k = 0; k < d.nw; ++k) nel *= d.wshape[k];
            A acc = s;
            bool have = seeded;
            for (int64_t q = 0; q < nel; ++q) {
                int64_t rem = q, off = 0;
                for (int k = 0; k < d.nw; ++k) {
                    int64_t id = rem % d.wshape[k];
                    rem /= d.wshape[k];
                    off += id * d.wst[k];
                }
                A v = ld(wb + off);
                if (!have) { acc = v; have = true; } else acc = afold(acc, v);
            }
            return acc;
        };
        auto compute_wide = [&](int64_t wb) -> A {
            if (d.nw == 0) return ld(wb);
            if constexpr (F16) { if (OP != OP_ADD) return wide_seq(wb, false, A{}); }
            return wide_pairwise(wb);
        };
        T res;
        T seedv;
        memcpy(&seedv, &d.seed, sizeof(T));
        if (d.nr == 0) {
            if constexpr (F16) {
                if (d.has_seed && OP != OP_ADD) res = f2h(wide_seq(base, true, h2f(seedv)));
                else if (d.has_seed) res = BinOp<OP, DT_F16>::apply(seedv, f2h(compute_wide(base)));
                else res = f2h(compute_wide(base));
            } else {
                res = BinOp<OP, CD>::apply(seedv, compute_wide(base));  // float add: seed always present
            }
        } else {
            bool have = d.has_seed;
            T acc = seedv;
            for (int64_t q = 0; q < ntotal; ++q) {
                int64_t rem = q, off = 0;
                for (int k = d.nr - 1; k >= 0; --k) {
                    int64_t id = rem % d.rshape[k];
                    rem /= d.rshape[k];
                    off += id * d.rst[k];
                }
                T part;
                if constexpr (F16) part = f2h(compute_wide(base + off));
                else part = compute_wide(base + off);
                if (!have) { acc = part; have = true; } else acc = BinOp<OP, CD>::apply(acc, part);
            }
            res = acc;
        }
        store_cast<CD>(d.o, out_off, d.odt, res);
    }
}

// Masked reductions (reduce_axis_masked, ufunc.rs:7213-7412, and
// reduce_axis_masked_f16_widen, 7414-7548). The seed always exists here.
template <int OP, int CD>
__global__ void __launch_bounds__(128) k_red_masked(RedDesc d) {
    typedef typename DT<CD>::T T;
    constexpr bool F16W = CD == DT_F16 && (OP == OP_ADD || OP == OP_MULTIPLY || OP == OP_SUBTRACT || OP == OP_DIVIDE);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    T seedv;
    memcpy(&seedv, &d.seed, sizeof(T));
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += stride) {
        // kept offsets for data and mask
        int64_t base = 0, mbase = 0, out_off = 0;
        {
            int64_t r = o;
            for (int k = d.nk - 1; k >= 0; --k) {
                int64_t id = r % d.kshape[k];
                r /= d.kshape[k];
                base += id * d.kst[k];
                mbase += id * d.mkst[k];
                out_off += id * d.kost[k];
            }
        }
        int64_t nn = 1;
        for (int k = 0; k < d.nr; ++k) nn *= d.rshape[k];
        int64_t nwe = 1;
        for (int k = 0; k < d.nwr; ++k) nwe *= d.wrshape[k];
        auto woff = [&](int64_t q, int64_t* dof, int64_t* mof) {
            int64_t rem = q, a = 0, m = 0;
            for (int k = d.nwr - 1; k >= 0; --k) {
                int64_t id = rem % d.wrshape[k];
                rem /= d.wrshape[k];
                a += id * d.wrst[k];
                m += id * d.mwst_raw[k];
            }
            *dof = a; *mof = m;
        };
        auto noff = [&](int64_t q, int64_t* dof, int64_t* mof) {
            int64_t rem = q, a = 0, m = 0;
            for (int k = d.nr - 1; k >= 0; --k) {
                int64_t id = rem % d.rshape[k];
                rem /= d.rshape[k];
                a += id * d.rst[k];
                m += id * d.mrst[k];
            }
            *dof = a; *mof = m;
        };
        constexpr bool PW = F16W || (OP == OP_ADD && (CD == DT_F32 || CD == DT_F64));
        if constexpr (PW) {
            typedef typename std::conditional<F16W, float, T>::type A;
            auto ld = [&](int64_t e) -> A {
                if constexpr (F16W) return h2f(((const h16*)d.a)[e]);
                else return ((const T*)d.a)[e];
            };
            auto afold = [&](A x, A y) -> A {
                if constexpr (F16W) return BinOp<OP, DT_F32>::apply(x, y);
                else return BinOp<OP, CD>::apply(x, y);
            };
            // compute_wide_masked over the raw wide dims (C order)
            auto cwm = [&](int64_t wb, int64_t mwb, A acc_in) -> A {
                if (d.nwr == 0) {
                    if (!d.m[mwb]) return acc_in;
                    if constexpr (F16W) return h2f(f2h(afold(acc_in, ld(wb))));
                    else return afold(acc_in, ld(wb));
                }
                A acc = acc_in;
                int64_t q = 0;
                while (q < nwe) {
                    int64_t dof, mof;
                    woff(q, &dof, &mof);
                    if (!d.m[mwb + mof]) { ++q; continue; }
                    int64_t q1 = q + 1;
                    for (; q1 < nwe; ++q1) { woff(q1, &dof, &mof); if (!d.m[mwb + mof]) break; }
                    int64_t len = q1 - q;
                    auto get = [&](int64_t i) { int64_t a_, m_; woff(q + i, &a_, &m_); return ld(wb + a_); };
                    A comb;
                    if constexpr (F16W) {
                        if (OP == OP_ADD) comb = afold(acc, pw_thread<A>(get, len, afold));
                        else if (OP == OP_MULTIPLY) {
                            A r = get(0);
                            for (int64_t i = 1; i < len; ++i) r = afold(r, get(i));
                            comb = afold(acc, r);
                        } else {
                            A r = acc;
                            for (int64_t i = 0; i < len; ++i) r = afold(r, get(i));
                            comb = r;
                        }
                        acc = h2f(f2h(comb));
                    } else {
                        acc = afold(acc, pw_thread<A>(get, len, afold));
                    }
                    q = q1;
                }
                return acc;
            };
            A acc;
            if constexpr (F16W) acc = h2f(seedv); else acc = seedv;
            if (d.nr == 0) acc = cwm(base, mbase, acc);
            else {
                for (int64_t q = 0; q < nn; ++q) {
                    int64_t dof, mof;
                    noff(q, &dof, &mof);
                    acc = cwm(base + dof, mbase + mof, acc);
                }
            }
            T res;
            if constexpr (F16W) res = f2h(acc); else res = acc;
            store_cast<CD>(d.o, out_off, d.odt, res);
        } else {
            // reduced axes in memory order; fold the masked-in elements
            T acc = seedv;
            for (int64_t q = 0; q < nn; ++q) {
                int64_t dof, mof;
                noff(q, &dof, &mof);
                if (d.m[mbase + mof]) acc = BinOp<OP, CD>::apply(acc, ((const T*)d.a)[base + dof]);
            }
            store_cast<CD>(d.o, out_off, d.odt, acc);
        }
    }
}

// ---------------------------------------------------------------------------
// argmin / argmax
// ---------------------------------------------------------------------------
template <int CD, bool MAX> struct ArgPol {
    typedef typename DT<CD>::T T;
    static __device__ __forceinline__ bool is_nan(T v) {
        if constexpr (CD == DT_F16) return isnan_h(v);
        else if constexpr (CD == DT_F32) return isnan_f(v);
        else if constexpr (CD == DT_F64) return isnan_d(v);
        else return false;
    }
    // (v, i) replaces (b, bi): strictly better, or not worse and earlier.
    // Equals the first-best of a sequential scan in index order.
    static __device__ __forceinline__ bool takes(T v, int64_t i, T b, int64_t bi) {
        if (i < 0) return false;
        if (bi < 0) return true;
        if (better(v, b)) return true;
        if (better(b, v)) return false;
        return i < bi;
    }
    // better(v, best) of reduce_axis_argext (ufunc.rs:8139-8160)
    static __device__ __forceinline__ bool better(T v, T b) {
        bool c;
        if constexpr (CD == DT_F16) c = MAX ? (h2f(v) > h2f(b)) : (h2f(v) < h2f(b));
        else c = MAX ? (v > b) : (v < b);
        if constexpr (dt_is_float(CD)) return c || (is_nan(v) && !is_nan(b));
        else return c;
    }
};

// One output per TPR-thread group; group elements: flat index i in [0, w),
// offset = unravel(i) over (rshape, rst) (C order) -- the argext axis, or the
// whole array for axis=None. Pairs combine left-first: the later pair only
// wins when strictly better, which is associative and equals the sequential
// scan.
template <int CD, bool MAX, int TPR>
__global__ void __launch_bounds__(RED_THREADS) k_argext(RedDesc d) {
    typedef ArgPol<CD, MAX> P;
    typedef typename DT<CD>::T T;
    constexpr int GROUPS = RED_THREADS / TPR;
    const int g = threadIdx.x / TPR, t = threadIdx.x % TPR;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t ntasks = d.nout * nseg;
    const int64_t seglen = (d.w + nseg - 1) / nseg;
    for (int64_t t0 = (int64_t)blockIdx.x * GROUPS; t0 < ntasks; t0 += (int64_t)gridDim.x * GROUPS) {
        int64_t task = t0 + g;
        bool live = task < ntasks;
        int64_t o = live ? task / nseg : 0, sg = live ? task % nseg : 0;
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        int64_t lo = sg * seglen, hi = lo + seglen;
        if (hi > d.w) hi = d.w;
        if (!live) hi = lo;
        T best{};
        int64_t bi = -1;
        constexpr int VE = 16 / (int)sizeof(T);
        const T* pc = (const T*)d.a + base;
        if (d.nr == 1 && d.rst[0] == 1 && VE > 1 && hi - lo >= (int64_t)VE * TPR &&
            ((reinterpret_cast<uintptr_t>(pc + lo)) & 15) == 0) {
            // contiguous: 16-byte vectors (thread t takes vectors t, t+TPR,
            // ... then the tail element lo + nv*VE + t), so each thread's
            // elements still come in increasing order; a vector without NaN
            // against a non-NaN best only needs "strictly greater"
            const int64_t nv = (hi - lo) / VE;
            constexpr int UV = 4;
            int64_t v = t;
            auto take = [&](const T (&x)[VE], int64_t e0) {
                bool nan = false;
                if constexpr (dt_is_float(CD)) {
                    if (bi >= 0 && P::is_nan(best)) return;  // nothing beats a NaN that came first
#pragma unroll
                    for (int k = 0; k < VE; ++k) nan |= P::is_nan(x[k]);
                }
                if (CD != DT_F16 && bi >= 0 && !nan) {
#pragma unroll
                    for (int k = 0; k < VE; ++k) {
                        const bool c = MAX ? (x[k] > best) : (x[k] < best);
                        if (c) { best = x[k]; bi = e0 + k; }
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < VE; ++k)
                        if (bi < 0 || P::better(x[k], best)) { best = x[k]; bi = e0 + k; }
                }
            };
            for (; v + (int64_t)(UV - 1) * TPR < nv; v += (int64_t)UV * TPR) {
                uint4 w[UV];
#pragma unroll
                for (int u = 0; u < UV; ++u) w[u] = __ldg(reinterpret_cast<const uint4*>(pc + lo + (v + (int64_t)u * TPR) * VE));
#pragma unroll
                for (int u = 0; u < UV; ++u) {
                    T x[VE];
                    memcpy(x, &w[u], 16);
                    take(x, lo + (v + (int64_t)u * TPR) * VE);
                }
            }
            for (; v < nv; v += TPR) {
                uint4 w = __ldg(reinterpret_cast<const uint4*>(pc + lo + v * VE));
                T x[VE];
                memcpy(x, &w, 16);
                take(x, lo + v * VE);
            }
            for (int64_t i = lo + nv * VE + t; i < hi; i += TPR) {
                const T x = pc[i];
                if (bi < 0 || P::better(x, best)) { best = x; bi = i; }
            }
        } else if (d.nr == 1) {
            // one strided run: no index arithmetic per element, eight loads
            // in flight per thread, each thread's elements in increasing order
            const T* p = (const T*)d.a + base;
            const int64_t ws = d.rst[0];
            int64_t i = lo + t;
            for (; i + 7 * TPR < hi; i += 8 * TPR) {
                T x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) x[u] = p[(i + (int64_t)u * TPR) * ws];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (bi < 0 || P::better(x[u], best)) { best = x[u]; bi = i + (int64_t)u * TPR; }
            }
            for (; i < hi; i += TPR) {
                T v = p[i * ws];
                if (bi < 0 || P::better(v, best)) { best = v; bi = i; }
            }
        } else {
            for (int64_t i = lo + t; i < hi; i += TPR) {
                int64_t off = 0, rem = i;
                for (int k = d.nr - 1; k >= 0; --k) {
                    int64_t id = rem % d.rshape[k];
                    rem /= d.rshape[k];
                    off += id * d.rst[k];
                }
                T v = ((const T*)d.a)[base + off];
                if (bi < 0 || P::better(v, best)) { best = v; bi = i; }
            }
        }
        // combine across the group, lower lanes (earlier indices) first
        if constexpr (TPR > 1) {
            const unsigned mask = TPR >= 32 ? 0xFFFFFFFFu : (((1u << TPR) - 1u) << ((threadIdx.x & 31) & ~(unsigned)(TPR - 1)));
            for (int s = 1; s < TPR && s < 32; s <<= 1) {
                T ov = __shfl_down_sync(mask, best, s, TPR < 32 ? TPR : 32);
                int64_t oi = __shfl_down_sync(mask, bi, s, TPR < 32 ? TPR : 32);
                if ((t & (2 * s - 1)) == 0 && P::takes(ov, oi, best, bi)) { best = ov; bi = oi; }
            }
            if constexpr (TPR > 32) {
                __shared__ T sv[RED_THREADS / 32];
                __shared__ int64_t si[RED_THREADS / 32];
                if ((t & 31) == 0) { sv[threadIdx.x / 32] = best; si[threadIdx.x / 32] = bi; }
                __syncthreads();
                if (t == 0) {
                    for (int w = 1; w < TPR / 32; ++w) {
                        int k = threadIdx.x / 32 + w;
                        if (P::takes(sv[k], si[k], best, bi)) { best = sv[k]; bi = si[k]; }
                    }
                }
                __syncthreads();
            }
        }
        if (live && t == 0) {
            if (d.K == 0) ((int64_t*)d.o)[out_off] = bi < 0 ? 0 : bi;
            else {
                int64_t* ixs = reinterpret_cast<int64_t*>(d.scratch);
                reinterpret_cast<T*>(ixs + ntasks)[task] = best;
                ixs[task] = bi;
            }
        }
    }
}

// Top of a split scan: one CTA per output combines its 2^K (value, index)
// partials. `takes` keeps the better value and, between equals (or two
// NaNs), the smaller index, so any combine order gives the sequential scan's
// answer; threads take strided partials, then a shuffle and a shared-memory
// tree finish.
template <int CD, bool MAX>
__global__ void __launch_bounds__(RED_THREADS) k_argext_top(RedDesc d) {
    typedef ArgPol<CD, MAX> P;
    typedef typename DT<CD>::T T;
    __shared__ T sv[RED_THREADS / 32];
    __shared__ int64_t si[RED_THREADS / 32];
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t ntasks = d.nout * nseg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t o = blockIdx.x; o < d.nout; o += gridDim.x) {
        const int64_t* ix = reinterpret_cast<const int64_t*>(d.scratch) + o * nseg;
        const T* v = reinterpret_cast<const T*>(reinterpret_cast<const int64_t*>(d.scratch) + ntasks) + o * nseg;
        T best{};
        int64_t bi = -1;
        for (int64_t s = threadIdx.x; s < nseg; s += RED_THREADS)
            if (P::takes(v[s], ix[s], best, bi)) { best = v[s]; bi = ix[s]; }
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            T ov = __shfl_down_sync(0xffffffffu, best, h);
            int64_t oi = __shfl_down_sync(0xffffffffu, bi, h);
            if (P::takes(ov, oi, best, bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { sv[warp] = best; si[warp] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < RED_THREADS / 32; ++w)
                if (P::takes(sv[w], si[w], best, bi)) { best = sv[w]; bi = si[w]; }
            int64_t in_off, out_off;
            kept_offsets(d, o, &in_off, &out_off);
            ((int64_t*)d.o)[out_off] = bi < 0 ? 0 : bi;
        }
        __syncthreads();
    }
}

// Column-order argext: one output per thread, sequential over the axis;
// with d.K > 0 the axis is cut into 2^K contiguous parts (task t scans part
// t / nout of output t % nout) whose (value, index) partials k_argext_top
// combines.
// One batch of an in-order argmin/argmax scan: `best`/`bi` updated from
// x[0..U) at indices i0..i0+U. Without a NaN on either side "better" is a
// strict comparison (float16 compares through float in P::better).
template <int CD, bool MAX, int U>
__device__ __forceinline__ void argext_batch(typename DT<CD>::T& best, int64_t& bi, const typename DT<CD>::T (&x)[U],
                                             int64_t i0) {
    typedef ArgPol<CD, MAX> P;
    bool nan = false;
    if constexpr (dt_is_float(CD)) {
        if (P::is_nan(best)) return;  // nothing beats a NaN that came first
#pragma unroll
        for (int u = 0; u < U; ++u) nan |= P::is_nan(x[u]);
    }
    if (CD != DT_F16 && !nan) {
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (MAX ? (x[u] > best) : (x[u] < best)) { best = x[u]; bi = i0 + u; }
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u) if (P::better(x[u], best)) { best = x[u]; bi = i0 + u; }
    }
}

// Column scan: task t = (part, output) scans rows [r0, r1) of its output's
// column in order, loads in batches of 16; for 4-byte and narrower values
// two register buffers, the next batch issued before the current one is
// scanned.
template <int CD, bool MAX>
__global__ void __launch_bounds__(RED_THREADS) k_argext_col(RedDesc d) {
    typedef ArgPol<CD, MAX> P;
    typedef typename DT<CD>::T T;
    constexpr int U = 16;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t ntask = d.nout * nseg;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask; t += stride) {
        const int64_t part = t / d.nout, o = t - part * d.nout;
        int64_t base, out_off;
        kept_offsets(d, o, &base, &out_off);
        const int64_t r0 = part * d.w / nseg, r1 = (part + 1) * d.w / nseg;
        const T* p = (const T*)d.a + base;
        T best = p[r0 * d.ws];
        int64_t bi = r0;
        const int64_t i = r0 + 1;
        const int64_t nb = (r1 - i) / U;
        T xa[U], xb[U];
        if constexpr (sizeof(T) > 4) {
            // 8-byte values: one batch at a time (a second buffer cost more
            // in occupancy than it gained in loads in flight)
            for (int64_t b = 0; b < nb; ++b) {
#pragma unroll
                for (int u = 0; u < U; ++u) xa[u] = p[(i + b * U + u) * d.ws];
                argext_batch<CD, MAX, U>(best, bi, xa, i + b * U);
            }
        } else if (nb > 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) xa[u] = p[(i + u) * d.ws];
            int64_t b = 0;
            for (; b + 2 <= nb; b += 2) {
                const int64_t i1 = i + (b + 1) * U;
#pragma unroll
                for (int u = 0; u < U; ++u) xb[u] = p[(i1 + u) * d.ws];
                argext_batch<CD, MAX, U>(best, bi, xa, i1 - U);
                if (b + 2 < nb) {
#pragma unroll
                    for (int u = 0; u < U; ++u) xa[u] = p[(i1 + U + u) * d.ws];
                }
                argext_batch<CD, MAX, U>(best, bi, xb, i1);
            }
            if (b < nb) argext_batch<CD, MAX, U>(best, bi, xa, i + b * U);
        }
        for (int64_t k = i + nb * U; k < r1; ++k) {
            T x = p[k * d.ws];
            if (P::better(x, best)) { best = x; bi = k; }
        }
        if (d.K == 0) {
            ((int64_t*)d.o)[out_off] = bi;
        } else {
            int64_t* ixs = reinterpret_cast<int64_t*>(d.scratch);
            reinterpret_cast<T*>(ixs + ntask)[o * nseg + part] = best;
            ixs[o * nseg + part] = bi;
        }
    }
}

// Top of a split scan with few partials per output: one thread per output.
template <int CD, bool MAX>
__global__ void __launch_bounds__(RED_THREADS) k_argext_top_small(RedDesc d) {
    typedef ArgPol<CD, MAX> P;
    typedef typename DT<CD>::T T;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t ntasks = d.nout * nseg;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < d.nout; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t* ix = reinterpret_cast<const int64_t*>(d.scratch) + o * nseg;
        const T* v = reinterpret_cast<const T*>(reinterpret_cast<const int64_t*>(d.scratch) + ntasks) + o * nseg;
        T best{};
        int64_t bi = -1;
        for (int64_t s = 0; s < nseg; ++s)
            if (P::takes(v[s], ix[s], best, bi)) { best = v[s]; bi = ix[s]; }
        int64_t in_off, out_off;
        kept_offsets(d, o, &in_off, &out_off);
        ((int64_t*)d.o)[out_off] = bi < 0 ? 0 : bi;
    }
}

// Argext over many short C-contiguous rows (16..256 bytes each): the
// staged ring and swizzle of k_red_rownar, one thread scanning one row in
// index order.
template <int CD, bool MAX>
__global__ void __launch_bounds__(RED_THREADS, 2) k_argext_nar(RedDesc d) {
    typedef ArgPol<CD, MAX> P;
    typedef typename DT<CD>::T T;
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr int STAGES = 3;
    constexpr int WCH = 32768 / 16;  // 16-byte chunks per stage
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    const int w = (int)d.w;
    const int m = w / VE;
    const int R = WCH / m < 2048 ? WCH / m : 2048;
    const int64_t nwin = (d.nout + R - 1) / R;
    const int64_t myw = nwin > blockIdx.x ? (nwin - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const uint4* a = reinterpret_cast<const uint4*>(d.a);
    auto swz = [](int g) { return g ^ ((g >> 3) & 7); };
    auto issue = [&](int64_t q) {
        if (q < myw) {
            const int64_t r0 = (blockIdx.x + q * (int64_t)gridDim.x) * R;
            const int64_t rows = d.nout - r0 < R ? d.nout - r0 : R;
            const int nch = (int)rows * m;
            uint4* sb = ring + (size_t)(q % STAGES) * WCH;
            const uint4* src = a + r0 * m;
            for (int c = threadIdx.x; c < nch; c += RED_THREADS) cp_async16(sb + swz(c), src + c);
        }
        cp_async_commit();
    };
    for (int s = 0; s < STAGES - 1; ++s) issue(s);
    for (int64_t q = 0; q < myw; ++q) {
        issue(q + STAGES - 1);
        cp_async_wait<STAGES - 1>();
        __syncthreads();
        const int64_t r0 = (blockIdx.x + q * (int64_t)gridDim.x) * R;
        const int rows = (int)(d.nout - r0 < R ? d.nout - r0 : R);
        const uint4* sb = ring + (size_t)(q % STAGES) * WCH;
        for (int r = threadIdx.x; r < rows; r += RED_THREADS) {
            const int g0 = r * m;
            T best{};
            int bi = 0;
            for (int c = 0; c < m; ++c) {
                uint4 v = sb[swz(g0 + c)];
                T x[VE];
                memcpy(x, &v, 16);
#pragma unroll
                for (int i = 0; i < VE; ++i) {
                    if ((c == 0 && i == 0) || P::better(x[i], best)) { best = x[i]; bi = c * VE + i; }
                }
            }
            ((int64_t*)d.o)[(r0 + r) * d.kost[0]] = bi;  // one kept dim
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// Launchers (ionp_reduce.cu)
cudaError_t launch_reduce_row(const RedDesc& d, int tpr, size_t smem, int grid, cudaStream_t s);
cudaError_t launch_reduce_row_top(const RedDesc& d, cudaStream_t s);
cudaError_t launch_reduce_col(const RedDesc& d, cudaStream_t s);
cudaError_t launch_reduce_col_split(const RedDesc& d, cudaStream_t s);
cudaError_t launch_reduce_gen(const RedDesc& d, cudaStream_t s);
cudaError_t launch_reduce_masked(const RedDesc& d, cudaStream_t s);
cudaError_t launch_argext(const RedDesc& d, int is_max, int mode, int tpr, cudaStream_t s);
bool reduce_row_supported(int op, int cd);

}  // namespace ionp
