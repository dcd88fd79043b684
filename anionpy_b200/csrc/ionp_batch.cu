// Batched execution of many small ufunc calls: one persistent kernel drains a
// device-side queue of call descriptors, captured once in a CUDA graph and
// replayed. The reference runs every call on its own (ionp-py/src/lib.rs:9205
// __call__, lib.rs:9959 reduce); this engine adds the batch so that a stream of
// thousands of small calls costs one launch instead of thousands.
//
// Every call keeps the exact arithmetic of its standalone entry point: binary
// calls use the same scalar op table (BinOp, cast on load to the loop dtype,
// cast on store), reductions the same fold orders (pairwise tree on a
// contiguous innermost run, sequential fold in row order otherwise, float16
// widening, integer widening to int64/uint64). A call's schedule (block tile,
// vector width, elements per thread, reduction split) only changes how its
// work is cut into tiles and mapped to threads, never a result bit.
//
// Queue layout: call descriptors are stored in queue order (largest tiles
// first, so the long reductions start early and the tail is short); a tile
// -> call map gives each global tile index its descriptor. CTAs claim tiles
// with one atomicAdd on a global counter and copy the descriptor of a new
// call into shared memory once. Reductions split in two (schedule
// red_split = 2) combine their halves with a last-arriver counter: the CTA
// that finishes second folds (left, right) in order, so no CTA ever waits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#include "ionp_host.h"
#include "ionp_reduce_launch.cuh"
#include "ionp_ew_launch.cuh"

namespace ionp {
namespace {

constexpr int BT_THREADS = 256;
enum : int32_t { BK_BINARY = 0, BK_ROW = 1, BK_COL = 2 };

// n / d for 0 <= n < 2^31, 1 <= d < 2^31, as one multiply and shift:
// m = ceil(2^(32+s) / d) with 2^s >= d makes the error term smaller than the
// distance from n/d to the next integer.
struct FastDiv {
    uint64_t m;
    uint32_t d;
    int32_t s;
};
FastDiv make_div(uint32_t d) {
    FastDiv f;
    f.d = d ? d : 1;
    f.s = 0;
    while ((1ull << f.s) < f.d) ++f.s;
    f.m = ((1ull << (32 + f.s)) + f.d - 1) / f.d;
    return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    return (uint32_t)(((uint64_t)n * f.m) >> (32 + f.s));
}

// Device descriptor of one call (queue entry).
struct BatchCall {
    int32_t kind, op, cd;
    int32_t dta, dtb, dto;
    int32_t nd;          // binary: merged dims (1..4)
    int32_t vec;         // binary: 16-byte vector path
    int32_t a_sc, b_sc;  // vector path: 0-d operand
    int32_t tpr, D;      // row: threads per output, slot-tree depth
    int32_t split;       // reduce: 1 or 2 tiles per output group
    int32_t has_seed;
    int32_t bt, vw, ept; // schedule
    int32_t user_id;
    int32_t shape[4];
    FastDiv div[4];
    int64_t sa[4], sb[4], so[4];
    const void* a;
    const void* b;
    void* o;
    int64_t n;           // binary: output elements; reduce: outputs
    int64_t per_tile;    // binary: elements per tile; reduce: outputs per tile
    int64_t ntiles;
    int64_t tile0;
    int64_t w, rs;       // reduce: extent and stride of the reduced axis
    int64_t ostride;     // reduce: input distance between consecutive outer indices
    int64_t inner;       // col: kept inner extent
    int64_t cols;        // col: inner outputs per tile
    int64_t ninner;      // col: tiles across the inner extent
    int32_t stage;       // col: elements per shared-memory stage
    int32_t copies;      // times the call is queued (the autotuner's throughput runs; else 1)
    int64_t ntiles_one;  // tiles of one copy
    uint64_t seed;
    void* partial;       // split: `split` partials per output
    uint32_t* arrive;    // split: arrival counter per output
    uint32_t* flags;     // FPE word of the call
};
static_assert(sizeof(BatchCall) % 4 == 0, "descriptor copies as 32-bit words");

// ------------------------------------------------------------------ binary
// Tile bodies are separate (not inlined) device functions: the persistent
// kernel dispatches over ~130 of them, and inlining them all into one body
// makes register allocation of that body intractable.
template <int OP, int CD>
__device__ __noinline__ void bin_tile(const BatchCall& c, int64_t local) {
    typedef BinOp<OP, CD> Op;
    typedef typename DT<CD>::T T;
    typedef typename Op::R R;
    constexpr bool FPE = FpeKind<OP, CD>::value != 0;
    // independent vectors / elements in flight per thread; float16 loops
    // (software half arithmetic) keep one to bound the code size
    constexpr int U = CD == DT_F16 ? 1 : 2;
    uint32_t bits = 0;
    const int nthr = c.bt < BT_THREADS ? c.bt : BT_THREADS;
    const int tid = threadIdx.x;
    const int64_t e0 = local * c.per_tile;
    const int64_t e1 = (e0 + c.per_tile < c.n) ? e0 + c.per_tile : c.n;
    R* o = (R*)c.o;  // the batch stores the loop's result dtype
    if (c.vec) {
        constexpr int N = Vec16<T>::N;
        const T* a = (const T*)c.a;
        const T* b = (const T*)c.b;
        const T a0 = a[0], b0 = b[0];
        const int64_t v0 = e0 / N, nv = e1 / N - v0;     // whole vectors of this tile
        const int unit = c.vw;                              // consecutive vectors per unit
        const int64_t per_pass = (int64_t)nthr * c.ept * unit;
        if (tid < nthr) {
            const int nmine = c.ept * unit;
            for (int64_t p0 = 0; p0 < nv; p0 += per_pass) {
                for (int q0 = 0; q0 < nmine; q0 += U) {
                    Vec16<T> xa[U], xb[U];
                    int64_t vi[U];
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        const int q = q0 + j;
                        const int k = q / unit, u = q - k * unit;
                        vi[j] = p0 + ((int64_t)k * nthr + tid) * unit + u;
                        if (q < nmine && vi[j] < nv) {
                            if (!c.a_sc) xa[j] = ldv(a, v0 + vi[j]); else for (int i = 0; i < N; ++i) xa[j].v[i] = a0;
                            if (!c.b_sc) xb[j] = ldv(b, v0 + vi[j]); else for (int i = 0; i < N; ++i) xb[j].v[i] = b0;
                        }
                    }
#pragma unroll
                    for (int j = 0; j < U; ++j) {
                        if (q0 + j < nmine && vi[j] < nv) {
                            R r[N];
#pragma unroll
                            for (int i = 0; i < N; ++i) {
                                r[i] = Op::apply(xa[j].v[i], xb[j].v[i]);
                                if constexpr (FPE) bits |= fpe_bits<OP, CD>(xa[j].v[i], xb[j].v[i], r[i]);
                            }
                            stv<R, N>(o, v0 + vi[j], r);
                        }
                    }
                }
            }
            // ragged end of the call (only the last tile has one)
            for (int64_t e = (v0 + nv) * N + tid; e < e1; e += nthr) {
                T x = c.a_sc ? a0 : a[e], y = c.b_sc ? b0 : b[e];
                R r = Op::apply(x, y);
                if constexpr (FPE) bits |= fpe_bits<OP, CD>(x, y, r);
                o[e] = r;
            }
        }
    } else if (tid < nthr) {
        const int nd = c.nd;
        for (int64_t base = e0 + tid; base < e1; base += U * (int64_t)nthr) {
            T x[U], y[U];
            int64_t oo[U];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const int64_t e = base + (int64_t)j * nthr;
                if (e < e1) {
                    uint32_t idx = (uint32_t)e;
                    int64_t fa = 0, fb_ = 0, fo = 0;
                    for (int k = nd - 1; k >= 1; --k) {
                        uint32_t q = fdiv(idx, c.div[k]);
                        uint32_t r = idx - q * (uint32_t)c.shape[k];
                        fa += (int64_t)r * c.sa[k];
                        fb_ += (int64_t)r * c.sb[k];
                        fo += (int64_t)r * c.so[k];
                        idx = q;
                    }
                    fa += (int64_t)idx * c.sa[0];
                    fb_ += (int64_t)idx * c.sb[0];
                    fo += (int64_t)idx * c.so[0];
                    x[j] = load_cast<CD>(c.a, fa, c.dta);
                    y[j] = load_cast<CD>(c.b, fb_, c.dtb);
                    oo[j] = fo;
                }
            }
#pragma unroll
            for (int j = 0; j < U; ++j) {
                if (base + (int64_t)j * nthr < e1) {
                    R r = Op::apply(x[j], y[j]);
                    if constexpr (FPE) bits |= fpe_bits<OP, CD>(x[j], y[j], r);
                    o[oo[j]] = r;
                }
            }
        }
    }
    if constexpr (FPE) flush_flags(bits, c.flags);
}

template <int OP>
__device__ __forceinline__ void bin_dispatch(const BatchCall& c, int64_t local) {
#define IONP_BCASE(D) \
    case D:           \
        if constexpr (bin_valid<OP, D>()) bin_tile<OP, D>(c, local); \
        break;
    switch (c.cd) { IONP_DTS(IONP_BCASE) }
#undef IONP_BCASE
}

// --------------------------------------------------------------- reduction
// Split combine: each part parks its partial; the tile that arrives last
// folds the `split` partials left to right (part 0 first), then finishes.
template <class P, int CD>
__device__ __forceinline__ void split_combine(const BatchCall& c, int64_t o, int64_t rep, int h, typename P::A part,
                                              bool is_final_value) {
    typedef typename P::A A;
    const int np = c.split;
    const int64_t slot = rep * c.n + o;  // each queued copy has its own partials
    A* pp = reinterpret_cast<A*>(c.partial) + slot * np;
    pp[h] = part;
    __threadfence();
    const unsigned prev = atomicAdd(&c.arrive[slot], 1u);
    if (prev == (unsigned)(np - 1)) {
        __threadfence();
        A tot = *(volatile A*)&pp[0];
        for (int k = 1; k < np; ++k) tot = P::fold(tot, *(volatile A*)&pp[k]);
        if (is_final_value) store_cast<CD>(c.o, o, c.dto, (typename P::T)tot);
        else store_cast<CD>(c.o, o, c.dto, P::finish(tot, c.has_seed, c.seed));
    }
}

template <int OP, int CD, bool CASTLD, int TPR>
__device__ __noinline__ void row_tile(const BatchCall& c, int64_t local, int64_t rep, unsigned char* smem) {
    typedef RPol<OP, CD, CASTLD> P;
    typedef typename P::A A;
    constexpr int G = BT_THREADS / TPR;
    const int g = threadIdx.x / TPR, t = threadIdx.x % TPR;
    const int nslots = TPR >= 32 ? (1 << c.D) : 1;
    A* slots = reinterpret_cast<A*>(smem) + (size_t)g * nslots;
    uint8_t* valid = reinterpret_cast<uint8_t*>(reinterpret_cast<A*>(smem) + (size_t)G * nslots) + (size_t)g * nslots;
    if (c.split == 2) {
        // TPR == 256: this tile is one half of one output's run, split at the
        // root of the pairwise tree (any split for the associative ops)
        if constexpr (TPR == BT_THREADS) {
            const int64_t o = local >> 1;
            const int h = (int)(local & 1);
            const int64_t n2 = pw_split(c.w);
            const int64_t soff = h ? n2 : 0, slen = h ? c.w - n2 : n2;
            A r = group_tree_t<P, TPR>(c.a, c.dta, c.rs, o * c.ostride, soff, slen, c.D, slots, valid, t);
            if (t == 0) split_combine<P, CD>(c, o, rep, h, r, false);
        }
        return;
    }
    const int64_t o_first = local * c.per_tile;
    for (int64_t k0 = 0; k0 < c.per_tile; k0 += G) {
        const int64_t o = o_first + k0 + g;
        const bool live = (k0 + g < c.per_tile) && o < c.n;
        A r{};
        if constexpr (TPR == 1) {
            if (live) r = leaf_thread<P>(c.a, c.dta, o * c.ostride, c.rs, 0, c.w);
        } else if constexpr (TPR == BT_THREADS) {
            const int64_t oo = o_first + k0;
            if (oo >= c.n) break;  // uniform over the CTA
            r = group_tree_t<P, TPR>(c.a, c.dta, c.rs, oo * c.ostride, 0, c.w, c.D, slots, valid, t);
        } else {
            if (live) r = group_tree_t<P, TPR>(c.a, c.dta, c.rs, o * c.ostride, 0, c.w, c.D, slots, valid, t);
        }
        if (live && t == 0) store_cast<CD>(c.o, o, c.dto, P::finish(r, c.has_seed, c.seed));
        if constexpr (TPR == BT_THREADS) __syncthreads();
    }
}

// Column tile: one outer index, `cols` adjacent inner outputs, one part of
// the reduced extent. The whole CTA streams stages of (rows x cols) elements
// (coalesced along the inner axis) through shared memory, loading the next
// stage into registers while the owner threads fold the current one in row
// order, so a few long sequential folds still keep many loads in flight.
template <int OP, int CD, bool CASTLD>
__device__ __noinline__ void col_tile(const BatchCall& c, int64_t local, int64_t rep, unsigned char* smem) {
    typedef typename DT<CD>::T T;
    constexpr int PER = 8;  // elements each thread loads per stage
    auto ld = [&](int64_t e) -> T {
        if constexpr (CASTLD) return load_int_widen<CD>(c.a, e, c.dta);
        else return reinterpret_cast<const T*>(c.a)[e];
    };
    const int np = c.split;
    const int64_t chunk = local / np;
    const int h = (int)(local - chunk * np);
    const int64_t outer = chunk / c.ninner;
    const int64_t i0 = (chunk - outer * c.ninner) * c.cols;
    const int cn = (int)(c.inner - i0 < c.cols ? c.inner - i0 : c.cols);
    const int64_t j0 = c.w * h / np, j1 = c.w * (h + 1) / np;
    const int64_t base = outer * c.ostride + i0;
    const int rows = c.stage / cn > 0 ? c.stage / cn : 1;
    T* buf = reinterpret_cast<T*>(smem);
    const int tid = threadIdx.x;
    const bool owner = tid < cn;
    T acc;
    bool have = false;
    if (owner && h == 0 && c.has_seed) { memcpy(&acc, &c.seed, sizeof(T)); have = true; }
    T v[PER];
    auto load_stage = [&](int64_t js) {
        const int nr = (int)(j1 - js < rows ? j1 - js : rows);
        const int tot = nr * cn;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int q = tid + k * BT_THREADS;
            if (q < tot) {
                const int r = q / cn, col = q - r * cn;
                v[k] = ld(base + (js + r) * c.inner + col);
            }
        }
    };
    if (j0 < j1) load_stage(j0);
    for (int64_t js = j0; js < j1; js += rows) {
        const int nr = (int)(j1 - js < rows ? j1 - js : rows);
        const int tot = nr * cn;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int q = tid + k * BT_THREADS;
            if (q < tot) buf[q] = v[k];
        }
        __syncthreads();
        if (js + rows < j1) load_stage(js + rows);  // next stage in flight during the fold
        if (owner) {
            for (int r = 0; r < nr; ++r) {
                const T x = buf[r * cn + tid];
                if (!have) { acc = x; have = true; }
                else acc = BinOp<OP, CD>::apply(acc, x);
            }
        }
        __syncthreads();
    }
    if (owner) {
        const int64_t o = outer * c.inner + i0 + tid;
        if (np > 1) {
            typedef RPol<OP, CD> PF;  // the accumulator is the compute dtype for these folds
            if constexpr (std::is_same<typename PF::A, T>::value) split_combine<PF, CD>(c, o, rep, h, acc, true);
        } else {
            store_cast<CD>(c.o, o, c.dto, acc);
        }
    }
}

template <int OP, int CD, bool CASTLD>
__device__ __forceinline__ void red_tile(const BatchCall& c, int64_t local, int64_t rep, unsigned char* smem) {
    if (c.kind == BK_COL) { col_tile<OP, CD, CASTLD>(c, local, rep, smem); return; }
    switch (c.tpr) {
        case 1: row_tile<OP, CD, CASTLD, 1>(c, local, rep, smem); break;
        case 32: row_tile<OP, CD, CASTLD, 32>(c, local, rep, smem); break;
        default: row_tile<OP, CD, CASTLD, BT_THREADS>(c, local, rep, smem); break;
    }
}

__device__ __forceinline__ void red_dispatch(const BatchCall& c, int64_t local, int64_t rep, unsigned char* smem) {
    if (c.op == OP_ADD) {
        switch (c.cd) {
            case DT_I64: red_tile<OP_ADD, DT_I64, true>(c, local, rep, smem); break;
            case DT_U64: red_tile<OP_ADD, DT_U64, true>(c, local, rep, smem); break;
            case DT_F16: red_tile<OP_ADD, DT_F16, false>(c, local, rep, smem); break;
            case DT_F32: red_tile<OP_ADD, DT_F32, false>(c, local, rep, smem); break;
            case DT_F64: red_tile<OP_ADD, DT_F64, false>(c, local, rep, smem); break;
        }
        return;
    }
#define IONP_MCASE(D) \
    case D: red_tile<OP_MAXIMUM, D, false>(c, local, rep, smem); break;
    switch (c.cd) { IONP_DTS(IONP_MCASE) }
#undef IONP_MCASE
}

// The persistent kernel: claim tiles until the queue is drained.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void run_tile(const BatchCall& c, int64_t t, unsigned char* smem) {
    int64_t local = t - c.tile0;
    const int64_t rep = local / c.ntiles_one;  // the copy (0 outside autotuner runs)
    local -= rep * c.ntiles_one;
    if (c.kind == BK_BINARY) {
        switch (c.op) {
            case OP_ADD: bin_dispatch<OP_ADD>(c, local); break;
            case OP_SUBTRACT: bin_dispatch<OP_SUBTRACT>(c, local); break;
            case OP_MULTIPLY: bin_dispatch<OP_MULTIPLY>(c, local); break;
            case OP_MAXIMUM: bin_dispatch<OP_MAXIMUM>(c, local); break;
            case OP_LESS: bin_dispatch<OP_LESS>(c, local); break;
            case OP_LOGICAL_AND: bin_dispatch<OP_LOGICAL_AND>(c, local); break;
        }
    } else {
        red_dispatch(c, local, rep, smem);
    }
}

// The persistent kernel: claim tiles until the queue is drained. The next
// tile is claimed, and its descriptor (when it belongs to another call)
// copied into the second shared-memory slot with cp.async, while the
// current tile runs, so neither the claim nor the descriptor load sits on
// the critical path.
__global__ void __launch_bounds__(BT_THREADS) k_batch(const BatchCall* __restrict__ calls,
                                                      const int32_t* __restrict__ tile_call, int64_t ntiles,
                                                      unsigned long long* next) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ BatchCall sc[2];
    __shared__ int64_t s_tile;
    __shared__ int32_t s_call;
    constexpr int WORDS = (int)(sizeof(BatchCall) / 4);
    if (threadIdx.x == 0) {
        const int64_t t0 = (int64_t)atomicAdd(next, 1ull);
        s_tile = t0;
        s_call = t0 < ntiles ? tile_call[t0] : -1;
    }
    __syncthreads();
    int64_t t = s_tile;
    int have0 = s_call, have1 = -1;  // descriptor held by slot 0 / 1 (uniform)
    int use = 0;
    if (t < ntiles) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(calls + have0);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sc[0]);
        for (int i = threadIdx.x; i < WORDS; i += BT_THREADS) dst[i] = src[i];
    }
    __syncthreads();
    while (t < ntiles) {
        if (threadIdx.x == 0) {
            const int64_t t2 = (int64_t)atomicAdd(next, 1ull);
            s_tile = t2;
            s_call = t2 < ntiles ? tile_call[t2] : -1;
        }
        __syncthreads();
        const int64_t t2 = s_tile;
        const int c2 = s_call;
        const int cur = use ? have1 : have0;
        const int oth = use ? have0 : have1;
        if (c2 >= 0 && c2 != cur && c2 != oth) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(calls + c2);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sc[use ^ 1]);
            for (int i = threadIdx.x; i < WORDS; i += BT_THREADS) cp_async4(dst + i, src + i);
            if (use) have0 = c2; else have1 = c2;
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        run_tile(sc[use], t, smem);
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        t = t2;
        if (c2 >= 0 && c2 != cur) use ^= 1;
    }
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

int tree_depth(int64_t n) {
    if (n <= PW_BLOCK) return 0;
    int64_t n2 = pw_split(n);
    return 1 + std::max(tree_depth(n2), tree_depth(n - n2));
}

bool c_contiguous(const IonpArr* a) {
    int64_t acc = 1;
    for (int i = a->ndim - 1; i >= 0; --i) {
        if (a->shape[i] != 1 && a->strides[i] != acc) return false;
        acc *= a->shape[i];
    }
    return true;
}

}  // namespace
}  // namespace ionp

using namespace ionp;

// ===========================================================================
// host side
// ===========================================================================
struct IonpBatch {
    struct Orig {
        int kind, op, axis, keepdims;
        IonpArr a, b, out;
    };
    std::vector<BatchCall> calls;   // caller order
    std::vector<Orig> orig;
    std::vector<IonpSchedule> sched;
    int device = 0;
    int sms = sm_count();
    // device state (from the caching allocator)
    BatchCall* d_calls = nullptr;
    int32_t* d_tile_call = nullptr;
    unsigned long long* d_next = nullptr;
    uint32_t* d_flags = nullptr;
    void* d_partial = nullptr;
    uint32_t* d_arrive = nullptr;
    size_t partial_bytes = 0, arrive_bytes = 0;
    int64_t ntiles = 0;
    size_t smem = 0;
    int grid = 0;
    bool finalized = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t capture_stream = nullptr;
    // single-call timing area
    BatchCall* d_one = nullptr;
    int32_t* d_one_map = nullptr;
    int64_t one_cap = 0;
    char* d_pool = nullptr;  // the autotuner's operand pool
};

namespace {

void release_device(IonpBatch* b) {
    cudaStream_t s = nullptr;
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    if (b->d_calls) scratch_free(b->d_calls, s);
    if (b->d_tile_call) scratch_free(b->d_tile_call, s);
    if (b->d_next) scratch_free(b->d_next, s);
    if (b->d_flags) scratch_free(b->d_flags, s);
    if (b->d_partial) scratch_free(b->d_partial, s);
    if (b->d_arrive) scratch_free(b->d_arrive, s);
    if (b->d_one) scratch_free(b->d_one, s);
    if (b->d_one_map) scratch_free(b->d_one_map, s);
    if (b->d_pool) scratch_free(b->d_pool, s);
    b->d_pool = nullptr;
    b->d_calls = nullptr; b->d_tile_call = nullptr; b->d_next = nullptr; b->d_flags = nullptr;
    b->d_partial = nullptr; b->d_arrive = nullptr; b->d_one = nullptr; b->d_one_map = nullptr;
    b->one_cap = 0;
    b->finalized = false;
}

int32_t check_schedule(const IonpSchedule* s) {
    if (!s) return IONP_OK;
    bool ok = (s->block_tile == 128 || s->block_tile == 256 || s->block_tile == 512 || s->block_tile == 1024) &&
              (s->vec_width == 1 || s->vec_width == 2 || s->vec_width == 4) &&
              (s->elems_per_thread == 1 || s->elems_per_thread == 4) && (s->red_split == 1 || s->red_split == 2);
    return ok ? IONP_OK : set_err(IONP_ERR_INVALID, "schedule outside the 48-point space");
}

void tile_geometry(BatchCall& c, const IonpSchedule& s);

// Tile geometry of one call under its schedule (fills per_tile, ntiles,
// split and D; everything else was planned when the call was added). One
// copy of the call.
void tile_call(BatchCall& c, const IonpSchedule& s) {
    tile_geometry(c, s);
    c.copies = 1;
    c.ntiles_one = c.ntiles;
}

void tile_geometry(BatchCall& c, const IonpSchedule& s) {
    c.bt = s.block_tile;
    c.vw = s.vec_width;
    c.ept = s.elems_per_thread;
    const int64_t work = (int64_t)s.block_tile * s.elems_per_thread * s.vec_width;
    if (c.kind == BK_BINARY) {
        const int64_t per = c.vec ? work * (16 / dt_size(c.cd)) : work * 4;
        c.per_tile = per;
        c.ntiles = ceil_div(c.n, per);
        c.split = 1;
        return;
    }
    const bool assoc = red_assoc(c.op, c.cd);
    if (c.kind == BK_ROW) {
        c.tpr = c.w <= PW_BLOCK ? 1 : c.w <= 2048 ? 32 : BT_THREADS;
        // runs longer than 2^18 always split at the root: the slot tree of
        // a half then fits 36 KB of shared memory (four CTAs per SM)
        c.split = ((s.red_split == 2 || c.w > ((int64_t)1 << 18)) && c.tpr == BT_THREADS) ? 2 : 1;
        if (c.split == 2) {
            const int64_t n2 = pw_split(c.w);
            c.D = std::max(tree_depth(n2), tree_depth(c.w - n2));
            c.per_tile = 1;
            c.ntiles = 2 * c.n;
        } else {
            c.D = c.tpr >= 32 ? tree_depth(c.w) : 0;
            c.per_tile = std::max<int64_t>(1, (work * 4) / std::max<int64_t>(c.w, 1));
            if (c.tpr == 1) c.per_tile = std::max<int64_t>(c.per_tile, 1);
            c.ntiles = ceil_div(c.n, c.per_tile);
        }
        return;
    }
    // column: `cols` adjacent inner outputs per tile (the block tile, at
    // most one per thread); stages of 1024 x elems_per_thread/2 (at least
    // 1024, at most 2048) elements; red_split = 2 cuts the reduced extent
    // into parts of >= 4096 rows (up to 32), exact only for the associative
    // folds
    c.cols = std::min<int64_t>(c.inner, std::min(s.block_tile, BT_THREADS));
    c.ninner = ceil_div(c.inner, c.cols);
    c.stage = s.elems_per_thread == 4 ? 2048 : 1024;
    c.per_tile = c.cols;
    int np = 1;
    if (s.red_split == 2 && assoc) np = (int)std::min<int64_t>(32, std::max<int64_t>(2, c.w / 4096));
    if (np > c.w) np = (int)std::max<int64_t>(c.w, 1);
    c.split = np;
    c.ntiles = (c.n / c.inner) * c.ninner * np;
}

size_t row_smem(const BatchCall& c) {
    if (c.kind == BK_COL) return (size_t)c.stage * dt_size(c.cd);
    if (c.kind != BK_ROW || c.tpr < 32) return 0;
    size_t acc = (c.cd == DT_F16 && c.op == OP_ADD) ? 4 : (size_t)dt_size(c.cd);
    size_t groups = BT_THREADS / c.tpr;
    return groups * ((size_t)1 << c.D) * (acc + 1) + 16;
}

int64_t tile_cost(const BatchCall& c) {
    if (c.kind == BK_BINARY) return c.per_tile * (dt_size(c.dta) + dt_size(c.dtb) + dt_size(c.dto));
    if (c.kind == BK_ROW) return (c.split == 2 ? c.w / 2 : c.per_tile * c.w) * dt_size(c.dta);
    return c.cols * (c.w / c.split) * dt_size(c.dta);
}

// Block tile 512, one 16-byte unit per thread, no split (schedule 24 of the
// 48): the single schedule that made whole 10,000-call mixed streams fastest
// on two of the three streams timed with every schedule.
void set_default_schedule(IonpSchedule* s) {
    s->block_tile = 512;
    s->vec_width = 1;
    s->elems_per_thread = 1;
    s->red_split = 1;
}

int32_t upload_and_plan(IonpBatch* b, cudaStream_t s) {
    release_device(b);
    const int nc = (int)b->calls.size();
    std::vector<BatchCall> q(b->calls);
    size_t smem = 0;
    for (int i = 0; i < nc; ++i) {
        tile_call(q[i], b->sched[i]);
        smem = std::max(smem, row_smem(q[i]));
    }
    std::vector<int> order(nc);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tile_cost(q[x]) > tile_cost(q[y]); });
    std::vector<BatchCall> qq(nc);
    int64_t tiles = 0;
    size_t part = 0, arr = 0;
    for (int k = 0; k < nc; ++k) {
        qq[k] = q[order[k]];
        qq[k].tile0 = tiles;
        tiles += qq[k].ntiles;
        if (qq[k].kind != BK_BINARY && qq[k].split > 1) {
            part += (size_t)qq[k].n * qq[k].split * 8;
            arr += (size_t)qq[k].n * 4;
        }
    }
    if (tiles >= (int64_t)1 << 31) return set_err(IONP_ERR_UNSUPPORTED, "batch has too many tiles");
    std::vector<int32_t> map((size_t)tiles);
    for (int k = 0; k < nc; ++k)
        for (int64_t t = 0; t < qq[k].ntiles; ++t) map[(size_t)(qq[k].tile0 + t)] = k;
    b->d_calls = (BatchCall*)scratch_alloc(sizeof(BatchCall) * std::max(nc, 1), s);
    b->d_tile_call = (int32_t*)scratch_alloc(sizeof(int32_t) * std::max<int64_t>(tiles, 1), s);
    b->d_next = (unsigned long long*)scratch_alloc(256, s);
    b->d_flags = (uint32_t*)scratch_alloc(sizeof(uint32_t) * std::max(nc, 1), s);
    if (part) {
        b->d_partial = scratch_alloc(part, s);
        b->d_arrive = (uint32_t*)scratch_alloc(arr, s);
    }
    if (!b->d_calls || !b->d_tile_call || !b->d_next || !b->d_flags || (part && (!b->d_partial || !b->d_arrive))) {
        release_device(b);
        return IONP_ERR_OOM;
    }
    b->partial_bytes = part;
    b->arrive_bytes = arr;
    size_t po = 0, ao = 0;
    for (int k = 0; k < nc; ++k) {
        BatchCall& c = qq[k];
        c.flags = b->d_flags + c.user_id;
        if (c.kind != BK_BINARY && c.split > 1) {
            c.partial = (char*)b->d_partial + po;
            c.arrive = (uint32_t*)((char*)b->d_arrive + ao);
            po += (size_t)c.n * c.split * 8;
            ao += (size_t)c.n * 4;
        }
    }
    int32_t st;
    if ((st = cuda_err(cudaMemcpyAsync(b->d_calls, qq.data(), sizeof(BatchCall) * nc, cudaMemcpyHostToDevice, s), "batch upload")))
        return st;
    if ((st = cuda_err(cudaMemcpyAsync(b->d_tile_call, map.data(), sizeof(int32_t) * tiles, cudaMemcpyHostToDevice, s), "batch upload")))
        return st;
    if ((st = cuda_err(cudaStreamSynchronize(s), "batch upload"))) return st;  // host vectors go out of scope
    b->ntiles = tiles;
    b->smem = smem;
    if (smem > 48 * 1024 &&
        (st = cuda_err(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "batch smem")))
        return st;
    int per_sm = 0;
    if ((st = cuda_err(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, BT_THREADS, smem), "batch occupancy")))
        return st;
    per_sm = std::max(per_sm, 1);
    b->grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)per_sm * b->sms));
    b->finalized = true;
    return IONP_OK;
}

int32_t enqueue_run(IonpBatch* b, cudaStream_t s) {
    int32_t st;
    if ((st = cuda_err(cudaMemsetAsync(b->d_next, 0, sizeof(unsigned long long), s), "batch reset"))) return st;
    if ((st = cuda_err(cudaMemsetAsync(b->d_flags, 0, sizeof(uint32_t) * std::max<size_t>(b->calls.size(), 1), s), "batch reset")))
        return st;
    if (b->arrive_bytes && (st = cuda_err(cudaMemsetAsync(b->d_arrive, 0, b->arrive_bytes, s), "batch reset"))) return st;
    if (b->ntiles == 0) return IONP_OK;
    k_batch<<<b->grid, BT_THREADS, b->smem, s>>>(b->d_calls, b->d_tile_call, b->ntiles, b->d_next);
    count_launch();
    return cuda_err(cudaGetLastError(), "batch launch");
}

}  // namespace

extern "C" {

int32_t ionp_schedule_from_index(int32_t idx, IonpSchedule* s) {
    if (!s || idx < 0 || idx >= IONP_NUM_SCHEDULES) return set_err(IONP_ERR_INVALID, "schedule index out of range");
    static const int BT[4] = {128, 256, 512, 1024}, VW[3] = {1, 2, 4}, EPT[2] = {1, 4}, SP[2] = {1, 2};
    s->block_tile = BT[idx / 12];
    s->vec_width = VW[(idx / 4) % 3];
    s->elems_per_thread = EPT[(idx / 2) % 2];
    s->red_split = SP[idx % 2];
    return IONP_OK;
}

int32_t ionp_batch_create(IonpBatch** out) {
    if (!out) return set_err(IONP_ERR_INVALID, "NULL batch pointer");
    IonpBatch* b = new IonpBatch();
    int32_t st = cuda_err(cudaGetDevice(&b->device), "batch device");
    if (!st) st = cuda_err(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device), "batch device");
    if (st) { delete b; return st; }
    *out = b;
    return IONP_OK;
}

int32_t ionp_batch_destroy(IonpBatch* b) {
    if (!b) return IONP_OK;
    cudaDeviceSynchronize();
    release_device(b);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    delete b;
    return IONP_OK;
}

int32_t ionp_batch_add_binary(IonpBatch* b, int32_t op, const IonpArr* a, const IonpArr* bb, IonpArr* out,
                              const IonpSchedule* sched, int32_t* call_id) {
    int32_t st;
    if (!b) return set_err(IONP_ERR_INVALID, "NULL batch");
    if ((st = check_arr(a, "a")) || (st = check_arr(bb, "b")) || (st = check_arr(out, "out"))) return st;
    if ((st = check_schedule(sched))) return st;
    if (!(op == OP_ADD || op == OP_SUBTRACT || op == OP_MULTIPLY || op == OP_MAXIMUM || op == OP_LESS || op == OP_LOGICAL_AND))
        return set_err(IONP_ERR_UNSUPPORTED, std::string("ufunc '") + op_name(op) + "' is not batched; call ionp_binary");
    int cd, rd;
    if ((st = binary_loop(op, a->dtype, bb->dtype, &cd, &rd))) return st;
    if (out->dtype != rd) return set_err(IONP_ERR_UNSUPPORTED, "batched calls write the loop's result dtype; call ionp_binary");
    const int nd = out->ndim;
    if (numel(out) >= ((int64_t)1 << 31)) return set_err(IONP_ERR_UNSUPPORTED, "call too large for a batch; call ionp_binary");
    MergeIn mi;
    mi.nd = nd;
    mi.nops = 3;
    for (int i = 0; i < nd; ++i) { mi.shape[i] = out->shape[i]; mi.st[0][i] = out->strides[i]; }
    if (!bcast_strides(a, nd, out->shape, mi.st[1]) || !bcast_strides(bb, nd, out->shape, mi.st[2]))
        return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " +
                                               fmt_shape(a->shape, a->ndim) + " " + fmt_shape(bb->shape, bb->ndim) + " ");
    MergeOut mo = merge_dims(mi);
    if (mo.nd > 4) return set_err(IONP_ERR_UNSUPPORTED, "more than 4 merged dims; call ionp_binary");
    BatchCall c;
    memset(&c, 0, sizeof(c));
    c.kind = BK_BINARY;
    c.op = op;
    c.cd = cd;
    c.dta = a->dtype;
    c.dtb = bb->dtype;
    c.dto = out->dtype;
    c.nd = mo.nd;
    c.n = numel(out);
    for (int i = 0; i < mo.nd; ++i) {
        c.shape[i] = (int32_t)mo.shape[i];
        c.div[i] = make_div((uint32_t)mo.shape[i]);
        c.so[i] = mo.st[0][i];
        c.sa[i] = mo.st[1][i];
        c.sb[i] = mo.st[2][i];
    }
    c.a = elem_ptr(a);
    c.b = elem_ptr(bb);
    c.o = (void*)elem_ptr(out);
    if (mo.nd == 1 && mo.st[0][0] == 1 && a->dtype == cd && bb->dtype == cd && out->dtype == rd) {
        bool a_ok = mo.st[1][0] == 1 || mo.st[1][0] == 0, b_ok = mo.st[2][0] == 1 || mo.st[2][0] == 0;
        bool al = (uintptr_t)c.o % 16 == 0 && (mo.st[1][0] == 0 || (uintptr_t)c.a % 16 == 0) &&
                  (mo.st[2][0] == 0 || (uintptr_t)c.b % 16 == 0);
        if (a_ok && b_ok && al) {
            c.vec = 1;
            c.a_sc = mo.st[1][0] == 0;
            c.b_sc = mo.st[2][0] == 0;
        }
    }
    c.user_id = (int32_t)b->calls.size();
    IonpSchedule s;
    if (sched) s = *sched; else set_default_schedule(&s);
    b->calls.push_back(c);
    b->sched.push_back(s);
    IonpBatch::Orig o;
    memset(&o, 0, sizeof(o));
    o.kind = BK_BINARY; o.op = op; o.a = *a; o.b = *bb; o.out = *out;
    b->orig.push_back(o);
    b->finalized = false;
    if (call_id) *call_id = c.user_id;
    return IONP_OK;
}

int32_t ionp_batch_add_reduce(IonpBatch* b, int32_t op, const IonpArr* a, int32_t axis, int32_t keepdims, IonpArr* out,
                              const IonpSchedule* sched, int32_t* call_id) {
    int32_t st;
    if (!b) return set_err(IONP_ERR_INVALID, "NULL batch");
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    if ((st = check_schedule(sched))) return st;
    if (op != OP_ADD && op != OP_MAXIMUM)
        return set_err(IONP_ERR_UNSUPPORTED, std::string("ufunc '") + op_name(op) + "'.reduce is not batched; call ionp_reduce");
    const int nd = a->ndim;
    if (nd == 0 || axis < 0 || axis >= nd) return set_err(IONP_ERR_AXIS, "batched reductions take one normalized axis");
    if (!c_contiguous(a) || !c_contiguous(out))
        return set_err(IONP_ERR_UNSUPPORTED, "batched reductions need C-contiguous input and output; call ionp_reduce");
    int cd;
    if ((st = reduce_cd(op, a->dtype, &cd))) return st;
    if (a->dtype != cd && !(op == OP_ADD && (cd == DT_I64 || cd == DT_U64)))
        return set_err(IONP_ERR_UNSUPPORTED, "the input would need a converted copy; call ionp_reduce");
    if (out->dtype != cd) return set_err(IONP_ERR_UNSUPPORTED, "batched reductions write the compute dtype");
    int64_t outer = 1, inner = 1, ext = a->shape[axis];
    for (int i = 0; i < axis; ++i) outer *= a->shape[i];
    for (int i = axis + 1; i < nd; ++i) inner *= a->shape[i];
    const int want_nd = keepdims ? nd : nd - 1;
    if (out->ndim != want_nd || numel(out) != outer * inner) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
    if (ext == 0) return set_err(IONP_ERR_UNSUPPORTED, "empty reduced extent; call ionp_reduce");
    if (outer * inner >= ((int64_t)1 << 31) || numel(a) >= ((int64_t)1 << 40))
        return set_err(IONP_ERR_UNSUPPORTED, "call too large for a batch; call ionp_reduce");
    BatchCall c;
    memset(&c, 0, sizeof(c));
    c.op = op;
    c.cd = cd;
    c.dta = a->dtype;
    c.dto = out->dtype;
    c.a = elem_ptr(a);
    c.o = (void*)elem_ptr(out);
    c.n = outer * inner;
    c.w = ext;
    uint64_t seed = 0;
    if (op == OP_ADD) {  // identity 0 of every add loop (add.reduce seeds with it)
        c.has_seed = 1;
        if (cd == DT_F16) seed = 0;
        c.seed = seed;
    }
    // the reduced axis is the pairwise "wide" run (float add) / the row
    // kernel's run when everything after it has extent 1; otherwise it folds
    // sequentially per output (ufunc.rs:6658-6806, sequential_group 6546)
    if (inner == 1) {
        c.kind = BK_ROW;
        c.rs = 1;
        c.ostride = ext;
    } else {
        c.kind = BK_COL;
        c.rs = inner;
        c.inner = inner;
        c.ostride = ext * inner;
    }
    c.user_id = (int32_t)b->calls.size();
    IonpSchedule s;
    if (sched) s = *sched; else set_default_schedule(&s);
    b->calls.push_back(c);
    b->sched.push_back(s);
    IonpBatch::Orig o;
    memset(&o, 0, sizeof(o));
    o.kind = c.kind; o.op = op; o.a = *a; o.out = *out; o.axis = axis; o.keepdims = keepdims;
    b->orig.push_back(o);
    b->finalized = false;
    if (call_id) *call_id = c.user_id;
    return IONP_OK;
}

int32_t ionp_batch_set_schedule(IonpBatch* b, int32_t call, const IonpSchedule* sched) {
    int32_t st;
    if (!b || !sched || call < 0 || call >= (int32_t)b->calls.size()) return set_err(IONP_ERR_INVALID, "bad call index");
    if ((st = check_schedule(sched))) return st;
    b->sched[call] = *sched;
    b->finalized = false;
    return IONP_OK;
}

int32_t ionp_batch_finalize(IonpBatch* b, IonpStream stream) {
    if (!b) return set_err(IONP_ERR_INVALID, "NULL batch");
    return upload_and_plan(b, (cudaStream_t)stream);
}

int32_t ionp_batch_run(IonpBatch* b, int32_t use_graph, IonpStream stream) {
    NvtxRange nvtx_("ionp_batch_run");
    int32_t st;
    if (!b) return set_err(IONP_ERR_INVALID, "NULL batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->finalized && (st = upload_and_plan(b, s))) return st;
    if (!use_graph) return enqueue_run(b, s);
    if (!b->gexec) {
        if (!b->capture_stream &&
            (st = cuda_err(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking), "capture stream")))
            return st;
        if ((st = cuda_err(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal), "begin capture")))
            return st;
        int32_t est = enqueue_run(b, b->capture_stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
        if (est) { if (g) cudaGraphDestroy(g); return est; }
        if ((st = cuda_err(e, "end capture"))) return st;
        b->graph = g;
        if ((st = cuda_err(cudaGraphInstantiate(&b->gexec, g, 0), "graph instantiate"))) return st;
    }
    return cuda_err(cudaGraphLaunch(b->gexec, s), "graph launch");
}

int32_t ionp_batch_run_per_call(IonpBatch* b, IonpStream stream) {
    NvtxRange nvtx_("ionp_batch_run_per_call");
    if (!b) return set_err(IONP_ERR_INVALID, "NULL batch");
    for (size_t i = 0; i < b->orig.size(); ++i) {
        IonpBatch::Orig& o = b->orig[i];
        int32_t st;
        if (o.kind == BK_BINARY) st = ionp_binary(o.op, &o.a, &o.b, &o.out, nullptr, nullptr, stream);
        else {
            int32_t ax = o.axis;
            st = ionp_reduce(o.op, &o.a, &ax, 1, o.keepdims, -1, nullptr, nullptr, &o.out, stream);
        }
        if (st) return st;
    }
    return IONP_OK;
}

int32_t ionp_batch_fpe(IonpBatch* b, uint32_t* words, IonpStream stream) {
    if (!b || !words) return set_err(IONP_ERR_INVALID, "bad arguments");
    if (!b->finalized) return set_err(IONP_ERR_INVALID, "batch has not run");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t st = cuda_err(cudaMemcpyAsync(words, b->d_flags, sizeof(uint32_t) * b->calls.size(), cudaMemcpyDeviceToHost, s), "fpe read");
    if (st) return st;
    return cuda_err(cudaStreamSynchronize(s), "fpe read");
}

int32_t ionp_batch_info(IonpBatch* b, int64_t* info) {
    if (!b || !info) return set_err(IONP_ERR_INVALID, "bad arguments");
    info[0] = (int64_t)b->calls.size();
    info[1] = b->ntiles;
    info[2] = b->grid;
    info[3] = (int64_t)b->smem;
    int64_t bytes = 0;
    for (const BatchCall& c : b->calls) {
        if (c.kind == BK_BINARY) {
            const IonpBatch::Orig& o = b->orig[c.user_id];
            bytes += numel(&o.a) * dt_size(c.dta) + numel(&o.b) * dt_size(c.dtb) + c.n * dt_size(c.dto);
        } else {
            bytes += c.n * c.w * dt_size(c.dta) + c.n * dt_size(c.dto);
        }
    }
    info[4] = bytes;
    return IONP_OK;
}

// Feature vector of one call for the schedule picker (IONP_PICKER_FEATURES
// floats): op class, call kind, operand and result widths, merged shape,
// stride class, reduction geometry.
int32_t ionp_batch_features(IonpBatch* b, int32_t call, float* f) {
    if (!b || !f || call < 0 || call >= (int32_t)b->calls.size()) return set_err(IONP_ERR_INVALID, "bad arguments");
    const BatchCall& c = b->calls[call];
    for (int i = 0; i < IONP_PICKER_FEATURES; ++i) f[i] = 0.0f;
    auto lg = [](double v) { return (float)(std::log2(std::max(v, 1.0)) / 20.0); };
    auto lb = [](int dt) { return (float)(std::log2((double)dt_size(dt)) / 3.0); };
    int opc = 0;
    if (c.kind == BK_BINARY) {
        switch (c.op) {
            case OP_ADD: opc = 0; break; case OP_SUBTRACT: opc = 1; break; case OP_MULTIPLY: opc = 2; break;
            case OP_MAXIMUM: opc = 3; break; case OP_LESS: opc = 4; break; default: opc = 5; break;
        }
    } else {
        opc = c.op == OP_ADD ? 6 : 7;
    }
    f[opc] = 1.0f;
    f[8 + c.kind] = 1.0f;
    f[11] = lb(c.dta);
    f[12] = c.kind == BK_BINARY ? lb(c.dtb) : lb(c.dta);
    f[13] = lb(c.dto);
    f[14] = (c.dta == c.cd && (c.kind != BK_BINARY || c.dtb == c.cd)) ? 1.0f : 0.0f;
    f[20] = lg((double)c.n);
    int sclass = 0;  // 0 contiguous, 1 broadcast, 2 permuted, 3 strided
    if (c.kind == BK_BINARY) {
        f[15] = c.nd / 4.0f;
        for (int i = 0; i < c.nd; ++i) f[16 + i] = lg((double)c.shape[c.nd - 1 - i]);
        bool zero = false;
        for (int i = 0; i < c.nd; ++i) zero = zero || c.sa[i] == 0 || c.sb[i] == 0;
        const int64_t ia = std::llabs(c.sa[c.nd - 1]), ib = std::llabs(c.sb[c.nd - 1]), io = std::llabs(c.so[c.nd - 1]);
        if (zero) sclass = 1;
        else if (ia == 1 && ib == 1 && io == 1) sclass = 0;
        else if (io == 1 && (ia > 1 || ib > 1)) sclass = 2;
        else sclass = 3;
    } else {
        f[15] = 0.25f;
        f[16] = lg((double)(c.n / std::max<int64_t>(c.kind == BK_COL ? c.inner : 1, 1)));
        f[17] = lg((double)c.w);
        f[18] = lg((double)(c.kind == BK_COL ? c.inner : 1));
        sclass = c.kind == BK_ROW ? 0 : 3;
    }
    f[21 + sclass] = 1.0f;
    f[25] = c.vec ? 1.0f : 0.0f;
    f[26] = lg((double)(c.kind == BK_BINARY ? 1 : c.w));
    f[27] = dt_is_float(c.cd) ? 1.0f : 0.0f;
    f[28] = c.cd == DT_F16 ? 1.0f : 0.0f;
    f[29] = (c.kind != BK_BINARY && c.dta != c.cd) ? 1.0f : 0.0f;
    f[30] = lb(c.cd);
    f[31] = 1.0f;
    return IONP_OK;
}

// Device time of one call of the batch under each of the given schedules,
// as the batch sees it. The call is queued `copies` times in one persistent
// launch -- enough copies for four tiles per resident CTA (at most 4096),
// limited so that all copies fit a 1 GiB pool -- and every copy reads and
// writes its OWN region of that pool, so the copies stream from HBM like the
// distinct calls of a real batch instead of re-reading one L2-resident
// input. Timing needs only the call's shapes, strides and dtypes; the pool's
// contents are whatever it holds. The launch is run `reps` times back to
// back between two events after one untimed run; time per copy is reported.
}  // extern "C"

namespace ionp {
namespace {
constexpr size_t TIME_POOL = (size_t)1 << 30;

// memory extent [lo, hi] in elements of an operand over the merged dims
void extent(const int64_t* st, const int32_t* shape, int nd, int64_t* lo, int64_t* hi) {
    *lo = 0; *hi = 0;
    for (int i = 0; i < nd; ++i) {
        const int64_t e = (int64_t)(shape[i] - 1) * st[i];
        if (e < 0) *lo += e; else *hi += e;
    }
}
size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// copy r of the template: its own operand regions, tiles and partials
__global__ void k_replicate(const BatchCall* __restrict__ tmpl, BatchCall* __restrict__ out, int K, char* pool,
                            int64_t span_a, int64_t span_b, int64_t span_o, int64_t lo_a, int64_t lo_b, int64_t lo_o,
                            char* part, int64_t part_stride, uint32_t* arrive, int64_t arrive_stride) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= K) return;
    BatchCall c = *tmpl;
    char* base = pool + (int64_t)r * (span_a + span_b + span_o);
    c.a = base - lo_a;
    c.b = base + span_a - lo_b;
    c.o = base + span_a + span_b - lo_o;
    c.tile0 = (int64_t)r * c.ntiles_one;
    if (part) {
        c.partial = part + (int64_t)r * part_stride;
        c.arrive = arrive + (int64_t)r * arrive_stride;
    }
    out[r] = c;
}
// copy-major tile map: tile t belongs to copy t / ntiles_one
__global__ void k_copy_map(int32_t* map, int64_t n, int64_t per) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        map[t] = (int32_t)(t / per);
}
}  // namespace
}  // namespace ionp

extern "C" {

int32_t ionp_batch_time_call(IonpBatch* b, int32_t call, int32_t nsched, const IonpSchedule* scheds, int32_t reps,
                             float* us_out, IonpStream stream) {
    int32_t st = IONP_OK;
    if (!b || call < 0 || call >= (int32_t)b->calls.size() || nsched <= 0 || !scheds || !us_out || reps <= 0)
        return set_err(IONP_ERR_INVALID, "bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->finalized && (st = upload_and_plan(b, s))) return st;
    constexpr int KMAX = 4096;
    if (!b->d_one) {
        b->d_one = (BatchCall*)scratch_alloc(sizeof(BatchCall) * (KMAX + 1), s);
        if (!b->d_one) return IONP_ERR_OOM;
    }
    if (!b->d_pool) {
        b->d_pool = (char*)scratch_alloc(TIME_POOL, s);
        if (!b->d_pool) return IONP_ERR_OOM;
    }
    // operand extents (bytes) of one copy, each 256-byte aligned
    const BatchCall& c0 = b->calls[call];
    int64_t lo_a = 0, lo_b = 0, lo_o = 0, hi_a = 0, hi_b = 0, hi_o = 0;
    if (c0.kind == BK_BINARY) {
        extent(c0.sa, c0.shape, c0.nd, &lo_a, &hi_a);
        extent(c0.sb, c0.shape, c0.nd, &lo_b, &hi_b);
        extent(c0.so, c0.shape, c0.nd, &lo_o, &hi_o);
    } else {
        hi_a = c0.n * c0.w - 1;
        hi_o = c0.n - 1;
    }
    const int64_t span_a = (int64_t)round256((size_t)(hi_a - lo_a + 1) * dt_size(c0.dta));
    const int64_t span_b = c0.kind == BK_BINARY ? (int64_t)round256((size_t)(hi_b - lo_b + 1) * dt_size(c0.dtb)) : 0;
    const int64_t span_o = (int64_t)round256((size_t)(hi_o - lo_o + 1) * dt_size(c0.dto));
    const int64_t per_copy = span_a + span_b + span_o;
    if ((size_t)per_copy > TIME_POOL)
        return set_err(IONP_ERR_UNSUPPORTED, "ionp_batch_time_call: the call's operands exceed the 1 GiB timing pool");
    cudaEvent_t e0, e1;
    if ((st = cuda_err(cudaEventCreate(&e0), "time events"))) return st;
    if ((st = cuda_err(cudaEventCreate(&e1), "time events"))) { cudaEventDestroy(e0); return st; }
    for (int k = 0; k < nsched; ++k) {
        if ((st = check_schedule(&scheds[k]))) break;
        BatchCall c = c0;
        tile_call(c, scheds[k]);
        c.flags = b->d_flags + c.user_id;
        const size_t smem = row_smem(c);
        if (smem > 48 * 1024 &&
            (st = cuda_err(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "time smem")))
            break;
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, BT_THREADS, smem);
        const int64_t slots = (int64_t)std::max(per_sm, 1) * b->sms;
        int64_t K = 1;
        if (c.ntiles_one > 0) K = std::min<int64_t>(KMAX, std::max<int64_t>(1, ceil_div(4 * slots, c.ntiles_one)));
        K = std::max<int64_t>(1, std::min<int64_t>(K, (int64_t)(TIME_POOL / (size_t)std::max<int64_t>(per_copy, 1))));
        const int64_t ntiles = c.ntiles_one * K;
        if (ntiles > b->one_cap) {
            if (b->d_one_map) scratch_free(b->d_one_map, s);
            b->one_cap = std::max<int64_t>(ntiles, 4096);
            b->d_one_map = (int32_t*)scratch_alloc(sizeof(int32_t) * b->one_cap, s);
            if (!b->d_one_map) { b->one_cap = 0; st = IONP_ERR_OOM; break; }
        }
        if (ntiles) {
            k_copy_map<<<(int)std::min<int64_t>(ceil_div(ntiles, 256), 4096), 256, 0, s>>>(b->d_one_map, ntiles, c.ntiles_one);
            count_launch();
        }
        void* part = nullptr;
        int64_t pstride = 0, astride = 0;
        if (c.kind != BK_BINARY && c.split > 1) {
            pstride = c.n * c.split * 8;
            astride = c.n;
            part = scratch_alloc((size_t)K * (size_t)(pstride + astride * 4), s);
            if (!part) { st = IONP_ERR_OOM; break; }
        }
        // template in slot KMAX, copies in slots 0..K-1
        if ((st = cuda_err(cudaMemcpyAsync(b->d_one + KMAX, &c, sizeof(BatchCall), cudaMemcpyHostToDevice, s), "time upload")))
            break;
        k_replicate<<<(int)ceil_div(K, 128), 128, 0, s>>>(b->d_one + KMAX, b->d_one, (int)K, b->d_pool, span_a, span_b, span_o,
                                                          lo_a * dt_size(c.dta), lo_b * dt_size(c.dtb), lo_o * dt_size(c.dto),
                                                          (char*)part, pstride,
                                                          part ? (uint32_t*)((char*)part + (size_t)K * pstride) : nullptr,
                                                          astride);
        count_launch();
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, slots));
        auto one = [&]() {
            cudaMemsetAsync(b->d_next, 0, 8, s);
            if (part) cudaMemsetAsync((char*)part + (size_t)K * pstride, 0, (size_t)K * astride * 4, s);
            if (ntiles) k_batch<<<grid, BT_THREADS, smem, s>>>(b->d_one, b->d_one_map, ntiles, b->d_next);
            count_launch();
        };
        one();
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; ++r) one();
        cudaEventRecord(e1, s);
        // the host template and the split scratch stay alive until the runs
        // are done
        st = cuda_err(cudaEventSynchronize(e1), "time sync");
        if (part) scratch_free(part, s);
        if (st) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        us_out[k] = ms * 1000.0f / ((float)reps * (float)K);
        if ((st = cuda_err(cudaGetLastError(), "time launch"))) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

}  // extern "C"
