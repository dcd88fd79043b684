// Wide-row reduction kernels for contiguous 4- and 8-byte runs: the common
// case of ufunc.reduce over the last axis (or over all axes) of a C-ordered
// array. They replace k_red_row's thread-per-leaf loads, where every lane of
// a warp reads 16 bytes of a different 512-byte leaf, by loads in which a
// warp touches whole 128-byte lines.
//
//  k_red_rowst : float add, numpy's pairwise tree (ufunc.rs:6416-6448).
//                One warp per run segment. The segment is cut at a fixed
//                depth Dw of its split tree into windows of at most 4096
//                elements; a window is a subtree, so its leaves never cross a
//                window edge. The warp streams its windows through its own
//                2-stage cp.async ring (16 bytes of padding after every 128
//                elements, so lanes reading different leaves hit distinct
//                banks). One lane sums one 128-element leaf: its 8
//                interleaved accumulators (elements k, k+8, ...) run as 8
//                independent chains of plain IEEE adds, combined
//                ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)); a leaf whose sum comes
//                out NaN is queued by warp ballot and summed again with the
//                engine's NaN-payload rule, 8 lanes per leaf. Leaf sums of a
//                full power-of-two window fold across lanes with shuffles,
//                others through a perfect-binary-tree slot array (left
//                operand first); window sums fold the same way per segment.
//  k_red_rowco : the order-free folds: integer add/multiply (wrapping),
//                bitwise and/or/xor, integer max/min, and float max/min,
//                whose only order dependence is that the first NaN in fold
//                order is the result (float_max/float_min return an operand
//                unchanged, and their non-NaN results do not depend on the
//                order, +0 winning a maximum tie and -0 a minimum tie). Lane l
//                of a warp reads 16 bytes at offset 16*l of each 512-byte
//                chunk (4 chunks in flight), folds them into its own
//                accumulator and remembers its first NaN with its index; the
//                accumulators meet in a warp and then a CTA tree, where the
//                NaN with the smallest index wins.
//
// Both take the segments of the K-level split of run_row (nout x 2^K units)
// and write either the output (K == 0) or one partial per unit for
// k_red_row_top.
#pragma once
#include "ionp_reduce.cuh"

#include <algorithm>
#include <climits>
#include <type_traits>
#include <map>
#include <set>

namespace ionp {

constexpr int RST_WIN = 4096;         // elements per window (a subtree of the split tree)
constexpr int RST_STAGES = 2;         // per-warp ring depth: one window in flight while one is summed
constexpr int RST_MAXDW = 6;          // at most 64 windows per segment
constexpr int RST_MAXDL = 7;          // at most 128 leaves per window (four per lane)
constexpr int RCO_CTAS = 5;
constexpr int RCO_U = 4;              // 512-byte chunks in flight per warp

// 16 bytes of padding after every 128 elements: one lane per 128-element
// leaf, so the lanes of a 16-byte shared load sit 4 banks apart
template <class T> constexpr int rst_pad() { return 16 / (int)sizeof(T); }
template <class T> constexpr int rst_win() { return RST_WIN; }
template <class T> constexpr int rst_win_phys() { return rst_win<T>() + rst_pad<T>() * (rst_win<T>() / 128); }
template <class T> constexpr int rst_warps() { return sizeof(T) == 4 ? 2 : 1; }  // warps per CTA
// window element e sits at e + pad * (e / 128) in the stage buffer
template <class T> __device__ __forceinline__ int rst_phys(int e) { return e + rst_pad<T>() * (e >> 7); }


__device__ __forceinline__ int pw_split32(int len) {
    int n2 = len / 2;
    return n2 - n2 % 8;
}

// Node `p` at depth Dw of the split tree of a segment of `len` elements;
// false when a leaf (<= 128 elements) closes the path above Dw and p is not
// the first path through it.
__device__ __forceinline__ bool rst_node(int64_t len, int Dw, int p, int64_t* off, int* nlen) {
    int64_t o = 0, l = len;
    for (int k = Dw - 1; k >= 0; --k) {
        if (l <= PW_BLOCK) {
            if (p & ((1 << (k + 1)) - 1)) return false;
            break;
        }
        int64_t n2 = pw_split(l);
        if ((p >> k) & 1) { o += n2; l -= n2; } else { l = n2; }
    }
    *off = o;
    *nlen = (int)l;
    return true;
}

template <class T> __device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// A warp folds a perfect-binary-tree slot array of 2^D <= 128 entries (lane
// l holds slots 4l..4l+3); the root lands in lane 0. A right subtree exists
// only where its left sibling does, so a missing right operand leaves the
// left one unchanged.
template <class P>
__device__ __forceinline__ typename P::A warp_slot_tree(const typename P::A* s, const uint8_t* v, int D, int lane) {
    typedef typename P::A A;
    const int ns = 1 << D;
    A x[4];
    int vx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int j = 4 * lane + i;
        vx[i] = j < ns && v[j];
        x[i] = vx[i] ? s[j] : A{};
    }
    if (vx[1]) x[0] = P::fold(x[0], x[1]);
    if (vx[3]) x[2] = P::fold(x[2], x[3]);
    if (vx[2]) x[0] = P::fold(x[0], x[2]);
    A a = x[0];
    int va = vx[0];
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
        A pa = __shfl_down_sync(0xffffffffu, a, h);
        int pv = __shfl_down_sync(0xffffffffu, va, h);
        if ((lane & (2 * h - 1)) == 0 && pv && va) a = P::fold(a, pa);
    }
    return a;
}

// Per-stage description of a window, written by the warp that issued its
// copies and read back when the warp folds it.
struct RstMeta {
    int64_t unit;
    int len, p, live, pad;
};

// Plain IEEE add (no NaN payload rule): equal to the engine's add whenever
// the result is not NaN.
template <class T> __device__ __forceinline__ T plain_add(T x, T y) {
    if constexpr (sizeof(T) == 8) return __dadd_rn(x, y);
    else return __fadd_rn(x, y);
}

// Per-warp shared memory of k_red_rowst: the window ring, the segment's
// window-sum slots, one window's leaf-sum slots, the ring's descriptions.
template <class T> constexpr size_t rst_warp_smem() {
    return ((size_t)RST_STAGES * rst_win_phys<T>() * sizeof(T) + (64 + 128) * sizeof(T) +
            (size_t)RST_STAGES * sizeof(RstMeta) + 64 + 128 + 127) / 128 * 128;  // each warp's ring 128-byte aligned
}
template <class T> constexpr size_t rst_smem() { return (size_t)rst_warps<T>() * rst_warp_smem<T>(); }

template <int OP, int CD>
__global__ void __launch_bounds__(32 * rst_warps<typename DT<CD>::T>()) k_red_rowst(RedDesc d) {
    typedef RPol<OP, CD> P;
    typedef typename P::A A;
    typedef typename DT<CD>::T T;
    static_assert(sizeof(A) == sizeof(T), "no widening in the staged kernel");
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr int PADE = rst_pad<T>();
    constexpr int WP = rst_win_phys<T>();
    constexpr int NWARP = rst_warps<T>();
    constexpr int WIN = rst_win<T>();
    constexpr int CPL = WIN / 64 / 32;   // candidate positions per lane
    constexpr int LPL = WIN / 128 / 32;  // leaves per lane in a full power-of-two window
    constexpr int DREG = LPL == 2 ? 6 : 5;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wbase = smem_raw + (size_t)warp * rst_warp_smem<T>();
    T* ring = reinterpret_cast<T*>(wbase);
    A* uslot = reinterpret_cast<A*>(ring + (size_t)RST_STAGES * WP);   // [64]
    A* lslot = uslot + 64;                                               // [128]
    RstMeta* meta = reinterpret_cast<RstMeta*>(lslot + 128);             // [RST_STAGES]
    uint8_t* uvalid = reinterpret_cast<uint8_t*>(meta + RST_STAGES);     // [64]
    uint8_t* lvalid = uvalid + 64;                                       // [128]
    const int Dw = d.Dw, Dl = d.Dl, NW = 1 << Dw;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t nunits = d.nout * nseg;
    const int64_t gw = (int64_t)blockIdx.x * NWARP + warp, GW = (int64_t)gridDim.x * NWARP;
    const int64_t myunits = nunits > gw ? (nunits - gw + GW - 1) / GW : 0;
    const int64_t Q = myunits * NW;
    for (int i = lane; i < 64; i += 32) uvalid[i] = 0;
    for (int i = lane; i < 128; i += 32) lvalid[i] = 0;
    const T* a = reinterpret_cast<const T*>(d.a);

    // the unit last issued: its base, and its windows' nodes (lane l holds
    // windows l and l + 32)
    int64_t cu = -1, cbase = 0;
    int64_t toff[2] = {0, 0};
    int tlen[2] = {0, 0};
    auto issue = [&](int64_t q) {
        if (q < Q) {
            const int64_t u = gw + (q >> Dw) * GW;
            const int p = (int)(q & (NW - 1));
            if (u != cu) {
                int64_t in_off, out_off, soff, slen;
                kept_offsets(d, u >> d.K, &in_off, &out_off);
                seg_of(d.w, d.K, u & (nseg - 1), &soff, &slen);
                cbase = in_off + soff;
                cu = u;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int pp = lane + 32 * h;
                    tlen[h] = -1;
                    if (pp < NW && !rst_node(slen, Dw, pp, &toff[h], &tlen[h])) tlen[h] = -1;
                }
            }
            const int hsel = p >> 5;
            const int64_t noff = __shfl_sync(0xffffffffu, hsel ? toff[1] : toff[0], p & 31);
            const int nlen = __shfl_sync(0xffffffffu, hsel ? tlen[1] : tlen[0], p & 31);
            const bool live = nlen >= 0;
            if (live) {
                T* sb = ring + (size_t)(q % RST_STAGES) * WP;
                const T* src = a + cbase + noff;
                if (nlen == WIN) {
                    // a full window: chunk lane + 32 i holds elements
                    // 128 i / VE ... of block (lane * VE) / 128 + ..., so both
                    // addresses advance by a constant per i
#pragma unroll
                    for (int i = 0; i < WIN / (32 * VE); ++i) {
                        const int e = (lane + 32 * i) * VE;
                        cp_async16(sb + e + PADE * (e >> 7), src + e);
                    }
                } else {
                    const int nch = nlen / VE;
                    for (int c = lane; c < nch; c += 32) cp_async16(sb + rst_phys<T>(c * VE), src + c * VE);
                    for (int e = nch * VE + lane; e < nlen; e += 32) cp_async_elem(sb + rst_phys<T>(e), src + e);
                }
            }
            if (lane == 0) {
                RstMeta& m = meta[q % RST_STAGES];
                m.unit = u;
                m.len = live ? nlen : 0;
                m.p = p;
                m.live = live;
            }
        }
        cp_async_commit();  // one group per window, empty or not
    };
    // the leaves that start at this lane's CPL candidate positions (CPL*lane
    // + h, 64 elements apart) for the current window length: LPL
    // 128-element leaves per lane in a full power-of-two window
    int cachedL = -1;
    int loff[CPL], llen[CPL], lsi[CPL];
    bool lhas[CPL];
#pragma unroll
    for (int h = 0; h < CPL; ++h) { loff[h] = 0; llen[h] = 0; lsi[h] = 0; lhas[h] = false; }
    for (int s = 0; s < RST_STAGES - 1; ++s) issue(s);
    for (int64_t q = 0; q < Q; ++q) {
        issue(q + RST_STAGES - 1);
        cp_async_wait<RST_STAGES - 1>();
        __syncwarp();
        const RstMeta m = meta[q % RST_STAGES];
        const int L = m.len, p = m.p;
        if (m.live) {
            const T* sb = ring + (size_t)(q % RST_STAGES) * WP;
            if (L != cachedL) {
                cachedL = L;
                const int ncand = (L + 63) / 64;
#pragma unroll
                for (int h = 0; h < CPL; ++h) {
                    const int c = CPL * lane + h;
                    lhas[h] = false;
                    if (c < ncand) {
                        const int mm = c * 64;
                        int off = 0, len = L, path = 0, depth = 0;
                        while (len > PW_BLOCK) {
                            const int n2 = pw_split32(len);
                            path <<= 1;
                            depth++;
                            if (mm < off + n2) len = n2; else { off += n2; len -= n2; path |= 1; }
                        }
                        lhas[h] = off > mm - 64;  // the leaf starts in this candidate window
                        loff[h] = off;
                        llen[h] = len;
                        lsi[h] = path << (Dl - depth);
                    }
                }
            }
            // a full power-of-two window: lane l sums leaves LPL*l + i, whose
            // slots are their indices
            const bool regular = L == WIN && Dl == DREG;
            A mine[LPL];
            bool mine_set[LPL];
#pragma unroll
            for (int i = 0; i < LPL; ++i) { mine[i] = A{}; mine_set[i] = false; }
            // each lane sums its leaves with plain adds, 8 independent
            // accumulator chains; leaves whose sum is NaN are queued and
            // then summed again with the engine's NaN rule, 8 lanes per
            // leaf, so one NaN does not hold the whole warp in a serial
            // replay
#pragma unroll
            for (int h = 0; h < CPL; ++h) {
                const int off = loff[h], len = llen[h];
                const bool fast = lhas[h] && len == PW_BLOCK && (off & (PW_BLOCK - 1)) == 0;
                bool redo = lhas[h] && !fast;
                if (fast) {
                    const T* src = sb + off + PADE * (off >> 7);
                    A r[8];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        T x[8];
#pragma unroll
                        for (int v = 0; v < 8 / VE; ++v) {
                            uint4 w = *reinterpret_cast<const uint4*>(src + 8 * j + v * VE);
                            memcpy(&x[v * VE], &w, 16);
                        }
#pragma unroll
                        for (int kk = 0; kk < 8; ++kk) r[kk] = j == 0 ? x[kk] : plain_add(r[kk], x[kk]);
                    }
                    const A res = plain_add(plain_add(plain_add(r[0], r[1]), plain_add(r[2], r[3])),
                                            plain_add(plain_add(r[4], r[5]), plain_add(r[6], r[7])));
                    if (res == res) {
                        if (regular) {
                            mine[h / 2] = res;  // candidate CPL*lane + h starts leaf (CPL*lane + h) / 2
                            mine_set[h / 2] = true;
                        } else {
                            lslot[lsi[h]] = res;
                            lvalid[lsi[h]] = 1;
                        }
                    } else {
                        redo = true;
                    }
                }
                unsigned q_mask = __ballot_sync(0xffffffffu, redo);
                while (q_mask) {
                    // up to 4 queued leaves at a time, one per 8-lane group
                    const int gq = lane >> 3, k = lane & 7;
                    unsigned mm = q_mask;
                    for (int i = 0; i < gq && mm; ++i) mm &= mm - 1;
                    const int src_lane = mm ? __ffs(mm) - 1 : 0;
                    const bool act = mm != 0;
                    const int qoff = __shfl_sync(0xffffffffu, off, src_lane);
                    const int qlen = __shfl_sync(0xffffffffu, len, src_lane);
                    const int qsi = __shfl_sync(0xffffffffu, lsi[h], src_lane);
                    for (int i = 0; i < 4 && q_mask; ++i) q_mask &= q_mask - 1;
                    if (act) {
                        const int lim = qlen & ~7;
                        const unsigned gm = 0xFFu << (lane & 24);
                        if (qlen >= 8) {
                            A r = sb[rst_phys<T>(qoff + k)];
                            for (int j = 8; j < lim; j += 8) r = P::fold(r, sb[rst_phys<T>(qoff + k + j)]);
                            A v = __shfl_xor_sync(gm, r, 1);
                            r = (k & 1) ? P::fold(v, r) : P::fold(r, v);
                            v = __shfl_xor_sync(gm, r, 2);
                            r = (k & 2) ? P::fold(v, r) : P::fold(r, v);
                            v = __shfl_xor_sync(gm, r, 4);
                            r = (k & 4) ? P::fold(v, r) : P::fold(r, v);
                            if (k == 0) {
                                for (int i = lim; i < qlen; ++i) r = P::fold(r, sb[rst_phys<T>(qoff + i)]);
                                lslot[qsi] = r;
                                lvalid[qsi] = 1;
                            }
                        } else if (k == 0) {  // a leaf of fewer than 8 elements folds in order
                            A r = sb[rst_phys<T>(qoff)];
                            for (int i = 1; i < qlen; ++i) r = P::fold(r, sb[rst_phys<T>(qoff + i)]);
                            lslot[qsi] = r;
                            lvalid[qsi] = 1;
                        }
                    }
                }
            }
            __syncwarp();
            A wsum;
            if (regular) {
                // the leaf sums of a perfect tree: the lane's own leaves
                // first, then across lanes, left operand first
#pragma unroll
                for (int i = 0; i < LPL; ++i)
                    if (!mine_set[i]) mine[i] = lslot[LPL * lane + i];
                A v = mine[0];
                if constexpr (LPL == 2) v = P::fold(mine[0], mine[1]);
#pragma unroll
                for (int hh = 1; hh < 32; hh <<= 1) {
                    const A o = __shfl_down_sync(0xffffffffu, v, hh);
                    if ((lane & (2 * hh - 1)) == 0) v = P::fold(v, o);
                }
                wsum = v;
            } else {
                wsum = warp_slot_tree<P>(lslot, lvalid, Dl, lane);
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; ++i) lvalid[lane + 32 * i] = 0;
            if (lane == 0) {
                uslot[p] = wsum;
                uvalid[p] = 1;
            }
            __syncwarp();
        }
        if (p == NW - 1) {  // the segment's last window (live or not)
            const int64_t u = m.unit;
            const A r = warp_slot_tree<P>(uslot, uvalid, Dw, lane);
            __syncwarp();
            uvalid[lane] = 0;
            uvalid[lane + 32] = 0;
            if (lane == 0) {
                if (d.K == 0) {
                    int64_t in_off, out_off;
                    kept_offsets(d, u, &in_off, &out_off);  // K == 0: the unit is the output index
                    store_cast<CD>(d.o, out_off, d.odt, P::finish(r, d.has_seed, d.seed));
                } else {
                    reinterpret_cast<A*>(d.scratch)[u] = r;
                }
            }
            __syncwarp();
        }
    }
    cp_async_wait<0>();
}

// Order-free accumulator of k_red_rowco.
//  * integers: the running fold, started from the op's identity (0 for add,
//    or and xor, 1 for multiply, all ones for and, the extreme value for
//    max/min), so every element costs one operation;
//  * float max/min: the non-NaN elements compared as ordered integer keys
//    (the bits with the magnitude flipped for negatives, so -0 < +0 and a
//    maximum tie picks +0 as float_max does), plus the first NaN and its
//    index; a 16-byte vector without NaN costs one integer max per element.
template <int CD> struct FKey {
    typedef typename DT<CD>::T T;
    typedef typename std::conditional<sizeof(T) == 8, long long, int>::type K;
    static __device__ __forceinline__ K key(T x) {
        K b;
        memcpy(&b, &x, sizeof(T));
        constexpr int SH = 8 * (int)sizeof(T) - 1;
        const K mag = (K)(~((unsigned long long)1 << SH) & (sizeof(T) == 8 ? ~0ull : 0xFFFFFFFFull));
        return b ^ ((b >> SH) & mag);
    }
    static __device__ __forceinline__ T val(K k) {
        const K b = key_inv(k);
        T x;
        memcpy(&x, &b, sizeof(T));
        return x;
    }
    static __device__ __forceinline__ K key_inv(K k) {
        constexpr int SH = 8 * (int)sizeof(T) - 1;
        const K mag = (K)(~((unsigned long long)1 << SH) & (sizeof(T) == 8 ? ~0ull : 0xFFFFFFFFull));
        return k ^ ((k >> SH) & mag);
    }
};

template <int OP, int CD> struct IntIdentity {
    typedef typename DT<CD>::T T;
    static __device__ __forceinline__ T get() {
        if constexpr (OP == OP_MULTIPLY) return (T)1;
        else if constexpr (OP == OP_BITWISE_AND) return (T)~(T)0;
        else if constexpr (OP == OP_MAXIMUM) return dt_is_sint(CD) ? (T)(1ull << (8 * sizeof(T) - 1)) : (T)0;
        else if constexpr (OP == OP_MINIMUM) return dt_is_sint(CD) ? (T)~(1ull << (8 * sizeof(T) - 1)) : (T)~(T)0;
        else return (T)0;
    }
};

template <int OP, int CD> struct CoAcc {
    typedef typename DT<CD>::T T;
    static constexpr bool FL = dt_is_float(CD);
    static constexpr bool MX = OP == OP_MAXIMUM;
    typedef typename FKey<CD>::K K;
    T v;        // integers: the fold so far
    K kv;       // floats: best key so far (sentinel: nothing yet)
    T nanv;
    int64_t nidx;
    static __device__ __forceinline__ K none() {
        if constexpr (sizeof(T) == 8) return MX ? (K)LLONG_MIN : (K)LLONG_MAX;
        else return MX ? (K)INT_MIN : (K)INT_MAX;
    }
    __device__ __forceinline__ void init() {
        nidx = INT64_MAX;
        nanv = T{};
        if constexpr (FL) kv = none();
        else v = IntIdentity<OP, CD>::get();
    }
    __device__ __forceinline__ void addk(K k) { kv = MX ? (k > kv ? k : kv) : (k < kv ? k : kv); }
    __device__ __forceinline__ void add(T x, int64_t idx) {
        if constexpr (FL) {
            if (x != x) {
                if (idx < nidx) { nidx = idx; nanv = x; }
                return;
            }
            addk(FKey<CD>::key(x));
        } else {
            v = BinOp<OP, CD>::apply(v, x);
        }
    }
    template <int VE> __device__ __forceinline__ void add_vec(const T (&x)[VE], int64_t e0) {
        if constexpr (FL) {
            bool nan = false;
#pragma unroll
            for (int i = 0; i < VE; ++i) nan |= x[i] != x[i];
            if (!nan) {
#pragma unroll
                for (int i = 0; i < VE; ++i) addk(FKey<CD>::key(x[i]));
            } else {
#pragma unroll
                for (int i = 0; i < VE; ++i) add(x[i], e0 + i);
            }
        } else {
#pragma unroll
            for (int i = 0; i < VE; ++i) v = BinOp<OP, CD>::apply(v, x[i]);
        }
    }
    __device__ __forceinline__ void merge(const CoAcc& o) {
        if constexpr (FL) {
            addk(o.kv);
            if (o.nidx < nidx) { nidx = o.nidx; nanv = o.nanv; }
        } else {
            v = BinOp<OP, CD>::apply(v, o.v);
        }
    }
    __device__ __forceinline__ void shfl_merge(int h) {
        CoAcc o;
        if constexpr (FL) {
            o.kv = __shfl_down_sync(0xffffffffu, kv, h);
            o.nanv = __shfl_down_sync(0xffffffffu, nanv, h);
            o.nidx = __shfl_down_sync(0xffffffffu, nidx, h);
        } else {
            o.v = __shfl_down_sync(0xffffffffu, v, h);
        }
        merge(o);
    }
    // the fold's result: the first NaN if there is one (every segment has
    // at least one element, so a float fold without NaN has a key)
    __device__ __forceinline__ T result() const {
        if constexpr (FL) {
            if (nidx != INT64_MAX) return nanv;
            return FKey<CD>::val(kv);
        }
        return v;
    }
};

template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS, RCO_CTAS) k_red_rowco(RedDesc d) {
    typedef typename DT<CD>::T T;
    typedef CoAcc<OP, CD> C;
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr int CH = 32 * VE;  // elements per 512-byte warp chunk
    constexpr int NWARP = RED_THREADS / 32;
    __shared__ C wacc[NWARP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t nunits = d.nout * nseg;
    for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
        int64_t in_off, out_off, soff, slen;
        kept_offsets(d, u >> d.K, &in_off, &out_off);
        seg_of(d.w, d.K, u & (nseg - 1), &soff, &slen);
        const T* base = reinterpret_cast<const T*>(d.a) + in_off + soff;
        const int64_t nch = (slen + CH - 1) / CH;
        const int64_t c0 = nch * warp / NWARP, c1 = nch * (warp + 1) / NWARP;
        C acc;
        acc.init();
        // whole chunks, RCO_U in flight; then the rest one at a time (the
        // segment's last chunk may be partial)
        const int64_t cfull = c1 < slen / CH ? c1 : (slen / CH > c0 ? slen / CH : c0);
        int64_t c = c0;
        for (; c + RCO_U <= cfull; c += RCO_U) {
            uint4 wv[RCO_U];
#pragma unroll
            for (int j = 0; j < RCO_U; ++j) wv[j] = __ldg(reinterpret_cast<const uint4*>(base + (c + j) * CH + lane * VE));
#pragma unroll
            for (int j = 0; j < RCO_U; ++j) {
                T x[VE];
                memcpy(x, &wv[j], 16);
                acc.template add_vec<VE>(x, (c + j) * CH + lane * VE);
            }
        }
        for (; c < c1; ++c) {
            const int64_t e = c * CH + lane * VE;
            if (e + VE <= slen) {
                uint4 wv = __ldg(reinterpret_cast<const uint4*>(base + e));
                T x[VE];
                memcpy(x, &wv, 16);
                acc.template add_vec<VE>(x, e);
            } else {
                for (int64_t i = e; i < slen; ++i) acc.add(base[i], i);
            }
        }
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) acc.shfl_merge(h);
        if (lane == 0) wacc[warp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            C r = wacc[0];
            for (int w = 1; w < NWARP; ++w) r.merge(wacc[w]);
            const T tot = r.result();
            if (d.K == 0) {
                if (d.has_seed) {
                    T s;
                    memcpy(&s, &d.seed, sizeof(T));
                    store_cast<CD>(d.o, out_off, d.odt, BinOp<OP, CD>::apply(s, tot));
                } else {
                    store_cast<CD>(d.o, out_off, d.odt, tot);
                }
            } else {
                reinterpret_cast<T*>(d.scratch)[u] = tot;
            }
        }
        __syncthreads();
    }
}

// Narrow rows (k_red_rownar): C-contiguous rows of 16..256 bytes (a float64
// row of 16 elements is 128 bytes). A CTA streams windows of up to 2048 whole
// rows (32 KiB) into a 3-stage cp.async ring; 16-byte chunk G of a window is
// stored at G ^ ((G >> 3) & 7), so the 8 lanes that one 16-byte shared load
// serves, each reading the same chunk of its own row, hit distinct banks.
// One thread folds one row with the leaf rule of pairwise_sum (8 interleaved
// accumulators, ufunc.rs:6416-6448) for float add and strictly left to right
// for every other op; every output is written directly.
constexpr int NAR_WIN_BYTES = 32768;
constexpr int NAR_STAGES = 3;
constexpr int NAR_CTAS = 2;
constexpr int NAR_MAXROWB = 256;
__device__ __forceinline__ int nar_swz(int g) { return g ^ ((g >> 3) & 7); }

template <int OP, int CD>
__global__ void __launch_bounds__(RED_THREADS, NAR_CTAS) k_red_rownar(RedDesc d) {
    typedef RPol<OP, CD> P;
    typedef typename P::A A;
    typedef typename DT<CD>::T T;
    static_assert(sizeof(A) == sizeof(T), "no widening in the narrow-row kernel");
    constexpr int VE = 16 / (int)sizeof(T);
    constexpr bool PW8 = !P::CHUNK && dt_is_float(CD);  // float add: the 8-accumulator leaf
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    constexpr int WCH = NAR_WIN_BYTES / 16;  // chunks per stage
    const int w = (int)d.w;
    const int m = w / VE;  // chunks per row
    const int R = WCH / m < 2048 ? WCH / m : 2048;
    const int64_t nwin = (d.nout + R - 1) / R;
    const int64_t myw = nwin > blockIdx.x ? (nwin - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const uint4* a = reinterpret_cast<const uint4*>(d.a);
    auto issue = [&](int64_t q) {
        if (q < myw) {
            const int64_t r0 = (blockIdx.x + q * (int64_t)gridDim.x) * R;
            const int64_t rows = d.nout - r0 < R ? d.nout - r0 : R;
            const int nch = (int)rows * m;
            uint4* sb = ring + (size_t)(q % NAR_STAGES) * WCH;
            const uint4* src = a + r0 * m;
            for (int c = threadIdx.x; c < nch; c += RED_THREADS) cp_async16(sb + nar_swz(c), src + c);
        }
        cp_async_commit();
    };
    for (int s = 0; s < NAR_STAGES - 1; ++s) issue(s);
    for (int64_t q = 0; q < myw; ++q) {
        issue(q + NAR_STAGES - 1);
        cp_async_wait<NAR_STAGES - 1>();
        __syncthreads();
        const int64_t r0 = (blockIdx.x + q * (int64_t)gridDim.x) * R;
        const int rows = (int)(d.nout - r0 < R ? d.nout - r0 : R);
        const uint4* sb = ring + (size_t)(q % NAR_STAGES) * WCH;
        for (int r = threadIdx.x; r < rows; r += RED_THREADS) {
            const int g0 = r * m;
            auto chunk = [&](int c, T (&x)[VE]) {
                uint4 v = sb[nar_swz(g0 + c)];
                memcpy(x, &v, 16);
            };
            A res;
            int done;  // elements folded
            if (PW8 && w >= 8) {
                A acc[8];
                const int lim = w & ~7;
#pragma unroll
                for (int cc = 0; cc < 8 / VE; ++cc) {
                    T x[VE];
                    chunk(cc, x);
#pragma unroll
                    for (int i = 0; i < VE; ++i) acc[cc * VE + i] = x[i];
                }
                for (int e = 8; e < lim; e += 8) {
#pragma unroll
                    for (int cc = 0; cc < 8 / VE; ++cc) {
                        T x[VE];
                        chunk(e / VE + cc, x);
#pragma unroll
                        for (int i = 0; i < VE; ++i) acc[cc * VE + i] = P::fold(acc[cc * VE + i], x[i]);
                    }
                }
                res = P::fold(P::fold(P::fold(acc[0], acc[1]), P::fold(acc[2], acc[3])),
                              P::fold(P::fold(acc[4], acc[5]), P::fold(acc[6], acc[7])));
                done = lim;
            } else {
                T x[VE];
                chunk(0, x);
                res = x[0];
#pragma unroll
                for (int i = 1; i < VE; ++i) res = P::fold(res, x[i]);
                done = VE;
            }
            for (int c = done / VE; c < m; ++c) {  // tail (or the rest of a sequential fold), in order
                T x[VE];
                chunk(c, x);
#pragma unroll
                for (int i = 0; i < VE; ++i)
                    if (c * VE + i >= done) res = P::fold(res, x[i]);
            }
            store_cast<CD>(d.o, (r0 + r) * d.kost[0], d.odt, P::finish(res, d.has_seed, d.seed));  // one kept dim
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Host side: which rows take these kernels, and their launch.
// ---------------------------------------------------------------------------
// k_red_pw32: float32 add over runs of 2^m >= 4096 elements, the common
// case of a row or whole-array sum. For such runs numpy's pairwise tree
// (ufunc.rs:6416-6448) halves exactly down to 128-element leaves, so the
// run is a perfect tree of 4096-element windows, each a perfect tree of 32
// leaves. One warp takes one window at a time:
//  * load: G lanes each issue one bulk copy (cp.async.bulk, the TMA engine,
//    unicast from this GPU's memory) of 32 / G consecutive leaves into a
//    shared group slot padded by 16 bytes, completing on the stage's
//    mbarrier; two stages per warp. Lane l takes leaf (l % G) * (32 / G) +
//    l / G, so the 8 lanes of each 16-byte shared-load phase read 8
//    different groups, on different banks (G = 8: four times fewer copies
//    than one per leaf, which measured 15 % faster);
//  * leaf: the lane sums its 128 elements as 8 independent chains of plain
//    adds (elements k, k+8, ...), combined ((r0+r1)+(r2+r3))+((r4+r5)+
//    (r6+r7)). A chain that comes out NaN is summed again with the engine's
//    add (the x86 NaN rules) and the combine redone with it: a result that
//    is not NaN had no NaN in it, so plain adds give the same bits;
//  * window: the 32 leaf sums fold across lanes by shuffles from the lane
//    holding the partner leaf, left operand first (a perfect tree);
//  * run: window sums fold on a binary-counter stack (push; while the two
//    top entries have the same height, fold them), which rebuilds the
//    perfect tree over a unit's 2^p windows.
// Every mbarrier wait has an iteration limit; a wait that gives up sets
// d.err, drains the warp's copies (again with a limit) and ends the warp.
// ---------------------------------------------------------------------------
constexpr int PW32_WIN = 4096;
constexpr int PW32_STACK = 24;
// ST stages per warp, NW warps per CTA
// G bulk copies per window, each of 32 / G leaves; a group's shared slot is
// padded by 16 bytes
template <int G> constexpr size_t pw32_stage_bytes() { return (size_t)G * ((32 / G) * 512 + 16); }
template <int ST, int G> constexpr size_t pw32_warp_smem() { return ST * pw32_stage_bytes<G>() + 64 + PW32_STACK * 8; }
template <int ST, int NW, int G> constexpr size_t pw32_smem() { return NW * pw32_warp_smem<ST, G>(); }
constexpr long long PW32_SPIN_LIMIT = 1LL << 26;

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(a), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    for (long long i = 0; i < PW32_SPIN_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(d), "l"(src), "r"(bytes), "r"(b) : "memory");
}

// the lane holding leaf L when G bulk copies of 32 / G leaves fill a window
template <int G> __host__ __device__ constexpr int pw32_leaf_lane(int L) { return (L % (32 / G)) * G + L / (32 / G); }

template <int OP, int CD, int PW32_STAGES, int PW32_WARPS, int G>
__global__ void __launch_bounds__(32 * PW32_WARPS) k_red_pw32(RedDesc d) {
    constexpr int LPG = 32 / G;                          // leaves per copy
    constexpr int GP = LPG * 128 + 4;                    // floats per group slot
    typedef RPol<OP, CD> P;
    static_assert(CD == DT_F32 && OP == OP_ADD, "float32 add only");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wb = smem_raw + (size_t)warp * pw32_warp_smem<PW32_STAGES, G>();
    float* ring = reinterpret_cast<float*>(wb);
    uint64_t* bar = reinterpret_cast<uint64_t*>(wb + PW32_STAGES * pw32_stage_bytes<G>());
    float* stk = reinterpret_cast<float*>(bar + 8);
    int* stk_h = reinterpret_cast<int*>(stk + PW32_STACK);
    const int64_t nseg = (int64_t)1 << d.K;
    const int64_t nunits = d.nout * nseg;
    const int64_t seglen = d.w >> d.K;
    const int64_t wpu = seglen / PW32_WIN;
    const int64_t gw = (int64_t)blockIdx.x * PW32_WARPS + warp, GW = (int64_t)gridDim.x * PW32_WARPS;
    const int64_t myunits = nunits > gw ? (nunits - gw + GW - 1) / GW : 0;
    const float* a = reinterpret_cast<const float*>(d.a);
    if (lane == 0) {
        for (int s = 0; s < PW32_STAGES; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncwarp();
    auto unit_base = [&](int64_t ui) -> const float* {
        const int64_t u = gw + ui * GW;
        int64_t in_off, out_off;
        kept_offsets(d, u >> d.K, &in_off, &out_off);
        return a + in_off + (u & (nseg - 1)) * seglen;
    };
    // the issue cursor runs PW32_STAGES - 1 windows ahead of the fold
    int64_t iu = 0, ij = 0, iq = 0;
    const float* ibase = myunits > 0 ? unit_base(0) : a;
    auto issue = [&]() {
        if (iu >= myunits) return;
        const int s = (int)(iq % PW32_STAGES);
        if (lane == 0) mbar_expect_tx(&bar[s], 32 * 512);
        __syncwarp();
        if (lane < G) bulk_g2s(ring + (size_t)s * G * GP + lane * GP, ibase + ij * PW32_WIN + lane * LPG * 128, LPG * 512, &bar[s]);
        ++iq;
        if (++ij == wpu) {
            ij = 0;
            if (++iu < myunits) ibase = unit_base(iu);
        }
    };
    for (int s = 0; s < PW32_STAGES - 1; ++s) issue();
    int top = 0;  // stack entries (lane 0)
    // Once the unit's stack holds a NaN, every window to its right is
    // irrelevant: all entries left of it are numbers, so each later node
    // takes the NaN from its left side. The unit's sum is then that NaN, and
    // its remaining windows are only waited for, not folded.
    bool unit_nan = false;  // warp-uniform
    float unit_val = 0.0f;  // lane 0
    int64_t q = 0;
    for (int64_t ui = 0; ui < myunits; ++ui) {
        for (int64_t j = 0; j < wpu; ++j, ++q) {
            issue();
            const int s = (int)(q % PW32_STAGES);
            if (!mbar_wait_bounded(&bar[s], (unsigned)((q / PW32_STAGES) & 1))) {
                // give up: record it, drain this warp's other copy, end the warp
                if (lane == 0 && d.err) atomicOr(d.err, 1u);
                for (int64_t q2 = q + 1; q2 < iq; ++q2)
                    if (!mbar_wait_bounded(&bar[q2 % PW32_STAGES], (unsigned)((q2 / PW32_STAGES) & 1))) break;
                return;
            }
            if (unit_nan) {
                __syncwarp();
                if (j == wpu - 1) {
                    if (lane == 0) {
                        const int64_t u = gw + ui * GW;
                        top = 0;
                        if (d.K == 0) {
                            int64_t in_off, out_off;
                            kept_offsets(d, u, &in_off, &out_off);
                            store_cast<CD>(d.o, out_off, d.odt, P::finish(unit_val, d.has_seed, d.seed));
                        } else {
                            reinterpret_cast<float*>(d.scratch)[u] = unit_val;
                        }
                    }
                    unit_nan = false;
                }
                continue;
            }
            // lane l holds leaf (l % G) * LPG + l / G: the 8 lanes of each
            // 16-byte shared load phase read 8 different groups, whose
            // 16-byte pads put them on different banks
            const float* lp = ring + (size_t)s * G * GP + (lane % G) * GP + (lane / G) * 128;
            float r[8];
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
                const float4 x0 = *reinterpret_cast<const float4*>(lp + 8 * jj);
                const float4 x1 = *reinterpret_cast<const float4*>(lp + 8 * jj + 4);
                const float x[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
                for (int k = 0; k < 8; ++k) r[k] = jj == 0 ? x[k] : __fadd_rn(r[k], x[k]);
            }
            float leaf = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                                   __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
            if (leaf != leaf) {
                // Only the first NaN chain needs its exact value: in the
                // left-first combine tree it is left of every later chain
                // at their common node, so a later NaN never wins; earlier
                // chains are NaN-free and exact, and an inf - inf among
                // them is redone by the exact combine below. The engine's
                // sequential add keeps the first NaN it meets, so the chain
                // is the first NaN element quieted -- or the default NaN
                // when the plain sum of the elements before it already
                // turned NaN (inf - inf) -- found without a sequential
                // replay of the engine's add.
                int kf = 7;
#pragma unroll
                for (int k = 6; k >= 0; --k) kf = (r[k] != r[k]) ? k : kf;
                float xc[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) xc[i] = lp[kf + 8 * i];
                int i0 = 16;
#pragma unroll
                for (int i = 15; i >= 0; --i) i0 = (xc[i] != xc[i]) ? i : i0;
                float pre = xc[0];
#pragma unroll
                for (int i = 1; i < 16; ++i) pre = (i < i0) ? __fadd_rn(pre, xc[i]) : pre;
                float chain = dnan_f();  // an inf - inf before any NaN element
#pragma unroll
                for (int i = 0; i < 16; ++i) chain = (i == i0 && !(i > 0 && pre != pre)) ? quiet_f(xc[i]) : chain;
#pragma unroll
                for (int k = 0; k < 8; ++k) r[k] = (k == kf) ? chain : r[k];
                leaf = P::fold(P::fold(P::fold(r[0], r[1]), P::fold(r[2], r[3])),
                               P::fold(P::fold(r[4], r[5]), P::fold(r[6], r[7])));
            }
            __syncwarp();  // every lane has read this stage before it is refilled
            // Leaf sums fold as a butterfly of plain adds: leaf bit t is lane
            // bit pw32_leaf_lane<G>(1 << t), and the lanes whose lower leaf
            // bits are clear hold the left-first subtree sums (IEEE addition
            // is commutative for non-NaN operands). Lane 0 ends with the
            // window sum; if it is NaN the tree is redone with the engine's
            // add from the kept leaf sums.
            float v = leaf;
#pragma unroll
            for (int t = 0; t < 5; ++t) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, pw32_leaf_lane<G>(1 << t)));
            if (__shfl_sync(0xffffffffu, v, 0) != __shfl_sync(0xffffffffu, v, 0)) {
                const int L = (lane % G) * LPG + lane / G;  // this lane's leaf
                v = leaf;
#pragma unroll
                for (int h = 1; h < 32; h <<= 1) {
                    const int M = (L + h) & 31;             // partner leaf (unused past 31)
                    const float o = __shfl_sync(0xffffffffu, v, pw32_leaf_lane<G>(M));
                    if ((L & (2 * h - 1)) == 0) v = P::fold(v, o);
                }
            }
            bool top_nan = false;
            if (lane == 0) {
                if (wpu == 1) {
                    stk[0] = v;
                } else {
                    stk[top] = v;
                    stk_h[top] = 0;
                    ++top;
                    while (top >= 2 && stk_h[top - 1] == stk_h[top - 2]) {
                        stk[top - 2] = P::fold(stk[top - 2], stk[top - 1]);
                        stk_h[top - 2] += 1;
                        --top;
                    }
                    unit_val = stk[top - 1];
                    top_nan = unit_val != unit_val;
                }
                if (j == wpu - 1) {
                    const int64_t u = gw + ui * GW;
                    const float total = stk[0];
                    top = 0;
                    if (d.K == 0) {
                        int64_t in_off, out_off;
                        kept_offsets(d, u, &in_off, &out_off);
                        store_cast<CD>(d.o, out_off, d.odt, P::finish(total, d.has_seed, d.seed));
                    } else {
                        reinterpret_cast<float*>(d.scratch)[u] = total;
                    }
                }
            }
            // a NaN on the stack settles the rest of the unit
            unit_nan = __shfl_sync(0xffffffffu, (int)top_nan, 0) != 0 && j != wpu - 1;
        }
    }
}

template <int ST, int NW, int G> inline int pw32_ctas_per_sm() {
    static int per_sm = 0;
    if (per_sm == 0) {
        auto k = k_red_pw32<OP_ADD, DT_F32, ST, NW, G>;
        int n = 0;
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pw32_smem<ST, NW, G>()) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 32 * NW, pw32_smem<ST, NW, G>()) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 1;
        }
        per_sm = n;
    }
    return per_sm;
}

// the configuration k_red_pw32 runs in: two stages per warp, two warps per
// CTA, eight bulk copies (of four leaves each) per window
constexpr int PW32_ST = 2, PW32_NW = 2, PW32_G = 8;

// warps of the float32 window kernel resident on the current device
inline int64_t pw32_resident_warps() {
    return (int64_t)sm_count() * pw32_ctas_per_sm<PW32_ST, PW32_NW, PW32_G>() * PW32_NW;
}

template <int OP, int CD, int ST, int NW, int G>
static cudaError_t launch_pw32(const RedDesc& din, cudaStream_t s) {
    auto k = k_red_pw32<OP, CD, ST, NW, G>;
    const int per_sm = pw32_ctas_per_sm<ST, NW, G>();
    const int64_t units = din.nout << din.K;
    const int64_t ctas = (units + NW - 1) / NW;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ctas, (int64_t)sm_count() * per_sm));
    k<<<grid, 32 * NW, pw32_smem<ST, NW, G>(), s>>>(din);
    count_launch();
    return cudaGetLastError();
}

// Runs k_red_pw32 handles: float32 add, input contiguous along the run in
// float32, 16-byte aligned run starts, a power-of-two run of at least one
// window whose K-level segments are whole windows.
inline bool pw32_ok(const RedDesc& d) {
    if (d.op != OP_ADD || d.cd != DT_F32 || d.adt != DT_F32 || d.ws != 1) return false;
    if (d.w < PW32_WIN || (d.w & (d.w - 1)) != 0) return false;
    if ((d.w >> d.K) < PW32_WIN) return false;
    if ((reinterpret_cast<uintptr_t>(d.a) & 15) != 0) return false;
    for (int i = 0; i < d.nk; ++i)
        if ((d.kst[i] * 4) % 16 != 0) return false;
    return true;
}

constexpr bool rowst_type_ok(int op, int cd) { return op == OP_ADD && (cd == DT_F32 || cd == DT_F64); }
constexpr bool rowco_type_ok(int op, int cd) {
    const bool w48 = cd == DT_I32 || cd == DT_I64 || cd == DT_U32 || cd == DT_U64 || cd == DT_F32 || cd == DT_F64;
    if (!w48) return false;
    if (op == OP_MAXIMUM || op == OP_MINIMUM) return true;
    return !dt_is_float(cd) && (op == OP_ADD || op == OP_MULTIPLY || op == OP_BITWISE_AND || op == OP_BITWISE_OR ||
                                op == OP_BITWISE_XOR);
}

// Contiguous runs whose every start is 16-byte aligned, long enough to keep a
// CTA busy per segment.
inline bool row_wide_ok(const RedDesc& d, int es) {
    if (d.ws != 1 || d.w < 2048 || d.adt != d.cd) return false;
    if ((reinterpret_cast<uintptr_t>(d.a) & 15) != 0) return false;
    for (int i = 0; i < d.nk; ++i)
        if ((d.kst[i] * es) % 16 != 0) return false;
    return true;
}

inline int rst_depth(int64_t n, std::map<int64_t, int>& memo) {
    if (n <= PW_BLOCK) return 0;
    auto it = memo.find(n);
    if (it != memo.end()) return it->second;
    int64_t n2 = pw_split(n);
    int dd = 1 + std::max(rst_depth(n2, memo), rst_depth(n - n2, memo));
    memo[n] = dd;
    return dd;
}

// Window depth Dw (all nodes at that depth fit one window) and leaf-slot
// depth Dl for the segments of run_row's K-level split; false when either
// slot array would exceed 64 entries.
inline bool rst_plan(int64_t w, int K, int win, int* Dw, int* Dl) {
    std::set<int64_t> cur{w};
    for (int i = 0; i < K; ++i) {
        std::set<int64_t> nx;
        for (int64_t l : cur) {
            int64_t n2 = pw_split(l);
            nx.insert(n2);
            nx.insert(l - n2);
        }
        cur.swap(nx);
    }
    int dw = 0;
    while (*cur.rbegin() > win) {
        std::set<int64_t> nx;
        for (int64_t l : cur) {
            if (l <= PW_BLOCK) { nx.insert(l); continue; }
            int64_t n2 = pw_split(l);
            nx.insert(n2);
            nx.insert(l - n2);
        }
        cur.swap(nx);
        if (++dw > RST_MAXDW) return false;
    }
    std::map<int64_t, int> memo;
    int dl = 0;
    for (int64_t l : cur) dl = std::max(dl, rst_depth(l, memo));
    if (dl > RST_MAXDL) return false;
    *Dw = dw;
    *Dl = dl;
    return true;
}

// C-contiguous rows of 16..256 bytes, each a whole number of 16-byte chunks.
inline bool row_narrow_ok(const RedDesc& d, int es) {
    if (d.ws != 1 || d.adt != d.cd || d.K != 0 || d.nk != 1 || d.kst[0] != d.w) return false;
    const int64_t rb = d.w * es;
    if (rb % 16 != 0 || rb < 16 || rb > NAR_MAXROWB) return false;
    return (reinterpret_cast<uintptr_t>(d.a) & 15) == 0 && d.nout >= sm_count() * 256;
}
constexpr bool rownar_type_ok(int op, int cd) { return rowst_type_ok(op, cd) || rowco_type_ok(op, cd); }

// Launch the wide-row kernel for (OP, CD) if the run qualifies; returns
// cudaErrorNotSupported (nothing launched) otherwise.
template <int OP, int CD>
static cudaError_t launch_row_wide(const RedDesc& din, cudaStream_t s) {
    typedef typename DT<CD>::T T;
    if constexpr (rownar_type_ok(OP, CD)) {
        if (row_narrow_ok(din, (int)sizeof(T))) {
            const int64_t R = std::min<int64_t>(2048, (NAR_WIN_BYTES / 16) / (din.w * (int64_t)sizeof(T) / 16));
            const int64_t nwin = (din.nout + R - 1) / R;
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nwin, (int64_t)sm_count() * NAR_CTAS));
            auto k = k_red_rownar<OP, CD>;
            const size_t smem = (size_t)NAR_STAGES * NAR_WIN_BYTES;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k<<<grid, RED_THREADS, smem, s>>>(din);
            count_launch();
            return cudaGetLastError();
        }
    }
    if constexpr (OP == OP_ADD && CD == DT_F32) {
        if (pw32_ok(din)) {
            return launch_pw32<OP, CD, PW32_ST, PW32_NW, PW32_G>(din, s);
        }
    }
    if constexpr (rowst_type_ok(OP, CD)) {
        if (!row_wide_ok(din, (int)sizeof(T))) return cudaErrorNotSupported;
        RedDesc d = din;
        if (!rst_plan(d.w, d.K, rst_win<T>(), &d.Dw, &d.Dl)) return cudaErrorNotSupported;
        const int64_t units = d.nout << d.K;
        auto k = k_red_rowst<OP, CD>;
        const size_t smem = rst_smem<T>();
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * rst_warps<T>(), smem);
        const int64_t ctas = (units + rst_warps<T>() - 1) / rst_warps<T>();
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ctas, (int64_t)sm_count() * std::max(per_sm, 1)));
        k<<<grid, 32 * rst_warps<T>(), smem, s>>>(d);
        count_launch();
        return cudaGetLastError();
    } else if constexpr (rowco_type_ok(OP, CD)) {
        if (!row_wide_ok(din, (int)sizeof(T))) return cudaErrorNotSupported;
        const int64_t units = din.nout << din.K;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)sm_count() * RCO_CTAS));
        k_red_rowco<OP, CD><<<grid, RED_THREADS, 0, s>>>(din);
        count_launch();
        return cudaGetLastError();
    } else {
        return cudaErrorNotSupported;
    }
}

}  // namespace ionp
