// Host planning of ufunc.reduce and argmin/argmax: mirrors reduce_axis
// (ionp-core/src/ufunc.rs:7634-7825) and argext (8131-8206) to decide the
// fold order, then picks the kernel that realises that order fastest.
#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <vector>
#include "ionp_host.h"
#include "ionp_reduce_launch.cuh"
#include "ionp_reduce_rowst.cuh"

namespace ionp {
namespace {

constexpr int64_t SEG_MAX = 65536;  // longest run one CTA reduces

int pw_depth(int64_t n, std::map<int64_t, int>& memo) {
    if (n <= PW_BLOCK) return 0;
    auto it = memo.find(n);
    if (it != memo.end()) return it->second;
    int64_t n2 = pw_split(n);
    int d = 1 + std::max(pw_depth(n2, memo), pw_depth(n - n2, memo));
    memo[n] = d;
    return d;
}
// distinct node lengths at depth K of the split tree of n
std::set<int64_t> seg_lengths(int64_t n, int K) {
    std::set<int64_t> cur{n};
    for (int k = 0; k < K; ++k) {
        std::set<int64_t> nx;
        for (int64_t l : cur) { int64_t n2 = pw_split(l); nx.insert(n2); nx.insert(l - n2); }
        cur.swap(nx);
    }
    return cur;
}
// threads per run: one thread sums a run of one leaf block, a warp a run of
// up to 16 blocks, a whole CTA anything longer
int tpr_for(int64_t w) { return w <= PW_BLOCK ? 1 : w <= 2048 ? 32 : 256; }

struct Dim { int64_t n, st, ost, mst; };

// kept dims in output order; size-1 dims dropped, C-adjacent dims merged
int kept_dims(const std::vector<Dim>& in, RedDesc& d, bool with_mask) {
    std::vector<Dim> v;
    for (const Dim& x : in) {
        if (x.n == 1) continue;
        if (!v.empty()) {
            Dim& p = v.back();
            if (p.st == x.st * x.n && p.ost == x.ost * x.n && (!with_mask || p.mst == x.mst * x.n)) {
                p.n *= x.n; p.st = x.st; p.ost = x.ost; p.mst = x.mst;
                continue;
            }
        }
        v.push_back(x);
    }
    if ((int)v.size() > RD_MAXD) return set_err(IONP_ERR_UNSUPPORTED, "too many non-mergeable kept dims for the reduction kernels");
    d.nk = (int)v.size();
    d.nout = 1;
    for (int i = 0; i < d.nk; ++i) {
        d.kshape[i] = v[i].n; d.kst[i] = v[i].st; d.kost[i] = v[i].ost; d.mkst[i] = v[i].mst;
        d.nout *= v[i].n;
    }
    return IONP_OK;
}

bool identity_bits(int op, int cd, uint64_t* out) {
    *out = 0;
    if (cd == DT_BOOL) {
        if (op == OP_ADD || op == OP_LOGICAL_OR || op == OP_BITWISE_OR || op == OP_LOGICAL_XOR || op == OP_BITWISE_XOR) return true;
        if (op == OP_MULTIPLY || op == OP_LOGICAL_AND || op == OP_BITWISE_AND) { *out = 1; return true; }
        return false;
    }
    if (!dt_is_float(cd)) {
        if (op == OP_ADD || op == OP_BITWISE_OR || op == OP_BITWISE_XOR) return true;
        if (op == OP_MULTIPLY) { *out = 1; return true; }
        if (op == OP_BITWISE_AND) { *out = dt_bytes(cd) == 8 ? ~0ull : ((1ull << (8 * dt_bytes(cd))) - 1); return true; }
        return false;
    }
    if (op == OP_ADD) return true;
    if (op == OP_MULTIPLY) {
        if (cd == DT_F16) *out = 0x3C00;
        else if (cd == DT_F32) { float one = 1.0f; memcpy(out, &one, 4); }
        else { double one = 1.0; memcpy(out, &one, 8); }
        return true;
    }
    return false;
}

int32_t run_row(RedDesc& d, cudaStream_t s) {
    const int64_t w = d.w;
    int K = 0;
    if (w > SEG_MAX) {
        while (*seg_lengths(w, K).rbegin() > SEG_MAX) ++K;
        // the top pass folds at most 2^(2 TOP_CHUNK_LOG) partials per output
        // (runs of up to 2^38 elements; only zero-stride views get longer)
        if (K > 2 * TOP_CHUNK_LOG)
            return set_err(IONP_ERR_VALUE, "reduction run of " + std::to_string(w) + " elements is longer than the 2^38 this engine folds");
    }
    // more parallel units when there are few outputs and long runs: the
    // wide-row kernels take a warp (float add) or a CTA per unit
    int64_t want = sm_count() * 2;
    if (row_wide_ok(d, dt_bytes(d.cd))) {
        if (rowst_type_ok(d.op, d.cd)) want = sm_count() * 16;
        else if (rowco_type_ok(d.op, d.cd)) want = sm_count() * RCO_CTAS;
    }
    while ((d.nout << K) < want && *seg_lengths(w, K + 1).begin() >= 4096 && K < 20 && K < 2 * TOP_CHUNK_LOG) ++K;
    // float32 add over a power-of-two run: one 4096-element window per unit
    // (the window kernel then balances evenly over all warps, and the top
    // pass folds the window sums as the perfect tree they form)
    {
        RedDesc t = d;
        t.K = 0;
        if (pw32_ok(t)) {
            // units of 2^p windows spread round-robin over the resident
            // warps: the smallest split whose units give every warp an
            // equal share to within 3 % (else the most even one)
            int kw = 0;
            while ((w >> kw) > PW32_WIN) ++kw;
            const int64_t gw = pw32_resident_warps();
            int pick = 0;
            double best = -1.0;
            for (int kk = 0; kk <= std::min(kw, 2 * TOP_CHUNK_LOG); ++kk) {
                const int64_t units = d.nout << kk;
                const int64_t per = (units + gw - 1) / gw;
                const double eff = (double)units / ((double)gw * (double)per);
                if (eff >= 0.97) { pick = kk; break; }
                if (eff > best + 1e-9) { best = eff; pick = kk; }
            }
            K = pick;
        }
    }
    auto lens = seg_lengths(w, K);
    int64_t maxlen = *lens.rbegin();
    std::map<int64_t, int> memo;
    int D = 0;
    for (int64_t l : lens) D = std::max(D, pw_depth(l, memo));
    int tpr = tpr_for(maxlen);
    size_t acc = (d.cd == DT_F16 && d.op == OP_ADD) ? 4 : (size_t)dt_bytes(d.cd);
    int groups = RED_THREADS / tpr;
    size_t nslots = tpr >= 32 ? ((size_t)1 << D) : 1;
    size_t smem = (size_t)groups * nslots * (acc + 1) + 16;
    d.K = K;
    d.D = D;
    const int64_t ntasks = d.nout << K;
    int64_t g = (ntasks + groups - 1) / groups;
    int64_t cap = (int64_t)sm_count() * (tpr == 256 ? 8 : 8);
    int grid = (int)std::max<int64_t>(1, std::min(g, cap));
    void* scratch = nullptr;
    if (K > 0) {
        scratch = scratch_alloc((size_t)ntasks * acc, s);
        if (!scratch) return IONP_ERR_OOM;
        d.scratch = scratch;
    }
    d.err = async_error_word();
    int32_t st = cuda_err(launch_reduce_row(d, tpr, smem, grid, s), "reduce row launch");
    if (!st && K > 0) st = cuda_err(launch_reduce_row_top(d, s), "reduce top launch");
    if (scratch) scratch_free(scratch, s);
    return st;
}

int32_t fill_seed(IonpArr* out, int cd, uint64_t seed, cudaStream_t s) {
    void* dev = scratch_alloc(16, s);
    if (!dev) return IONP_ERR_OOM;
    int32_t st = cuda_err(cudaMemcpyAsync(dev, &seed, 8, cudaMemcpyHostToDevice, s), "seed upload");
    if (!st) {
        IonpArr src;
        memset(&src, 0, sizeof(src));
        src.dtype = cd;
        src.ndim = 0;
        src.data = dev;
        st = cast_impl(&src, out, nullptr, s);
    }
    cudaStreamSynchronize(s);  // the host seed copy must stay valid until the upload ran
    scratch_free(dev, s);
    return st;
}

}  // namespace
}  // namespace ionp

using namespace ionp;

extern "C" {

int32_t ionp_cast_scalar(const void* src, int32_t sd, void* dst, int32_t dd) {
    if (!src || !dst || !dt_valid(sd) || !dt_valid(dd)) return set_err(IONP_ERR_INVALID, "bad arguments");
    host_cast_scalar(src, sd, dst, dd);
    return IONP_OK;
}

int32_t ionp_reduce(int32_t op, const IonpArr* a_in, const int32_t* axes, int32_t naxes, int32_t keepdims,
                    int32_t compute_dtype, const void* initial, const IonpArr* where, IonpArr* out, IonpStream stream) {
    NvtxRange nvtx_("ionp_reduce");
    int32_t st;
    if ((st = check_arr(a_in, "a")) || (st = check_arr(out, "out"))) return st;
    if (where && (st = check_arr(where, "where"))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nd = a_in->ndim;
    bool red[IONP_MAX_DIMS] = {false};
    for (int k = 0; k < naxes; ++k) {
        if (axes[k] < 0 || axes[k] >= std::max(nd, 1) || (k > 0 && axes[k] <= axes[k - 1]))
            return set_err(IONP_ERR_AXIS, "axes must be normalized, sorted and unique");
        if (nd > 0) red[axes[k]] = true;
    }
    const char* name = op_name(op);
    // supports_reduce_family (ufunc.rs:106) before the reorderable check
    if (op_is_compare(op) && a_in->dtype != DT_BOOL)
        return set_err(IONP_ERR_NO_LOOP, std::string("ufunc '") + name + "' did not contain a loop with signature matching types");
    bool reorderable = !(op == OP_SUBTRACT || op == OP_DIVIDE || op == OP_FLOOR_DIVIDE || op == OP_LEFT_SHIFT || op == OP_RIGHT_SHIFT);
    if (naxes > 1 && !reorderable)
        return set_err(IONP_ERR_VALUE, std::string("reduction operation '") + name + "' is not reorderable, so at most one axis may be specified");
    int cd = compute_dtype;
    if (cd < 0) { if ((st = reduce_cd(op, a_in->dtype, &cd))) return st; }
    if (!dt_valid(cd)) return set_err(IONP_ERR_INVALID, "bad compute dtype");
    if (!red_any_valid(op, cd))
        return set_err(IONP_ERR_TYPE, std::string("ufunc '") + name + "' has no reduce loop for dtype " + dt_name(cd));
    // output shape check
    int kept_nd = 0;
    for (int i = 0; i < nd; ++i) if (!red[i]) kept_nd++;
    int want_nd = keepdims ? nd : kept_nd;
    if (out->ndim != want_nd) return set_err(IONP_ERR_VALUE, "out has the wrong number of dimensions");
    std::vector<int> out_dim_of(nd, -1);
    {
        int j = 0;
        for (int i = 0; i < nd; ++i) {
            if (keepdims) {
                out_dim_of[i] = i;
                if (out->shape[i] != (red[i] ? 1 : a_in->shape[i])) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
            } else if (!red[i]) {
                out_dim_of[i] = j;
                if (out->shape[j] != a_in->shape[i]) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
                j++;
            }
        }
    }
    const bool pw_family = (op == OP_ADD && (cd == DT_F32 || cd == DT_F64)) ||
                           (cd == DT_F16 && (op == OP_ADD || op == OP_MULTIPLY || op == OP_SUBTRACT || op == OP_DIVIDE));
    // seed = initial.or(identity)
    uint64_t seed = 0;
    bool has_seed = false;
    if (initial) { memcpy(&seed, initial, dt_bytes(cd)); has_seed = true; }
    else has_seed = identity_bits(op, cd, &seed);

    int64_t group = 1;
    for (int i = 0; i < nd; ++i) if (red[i]) group *= a_in->shape[i];
    if (numel(out) == 0) return IONP_OK;

    // temporaries: float compute in another dtype is materialised C-contiguous
    // (the reference folds the cast copy, whose strides decide the plan); a
    // non-bool mask is cast to bool.
    IonpArr acast, mcast;
    const IonpArr* a = a_in;
    void* tmp_a = nullptr;
    void* tmp_m = nullptr;
    auto cleanup = [&]() {
        if (tmp_a) scratch_free(tmp_a, s);
        if (tmp_m) scratch_free(tmp_m, s);
    };
    auto c_contig = [](IonpArr& t, const IonpArr* src, int dt) {
        memset(&t, 0, sizeof(t));
        t.dtype = dt;
        t.ndim = src->ndim;
        int64_t acc = 1;
        for (int i = src->ndim - 1; i >= 0; --i) { t.shape[i] = src->shape[i]; t.strides[i] = acc; acc *= std::max<int64_t>(src->shape[i], 1); }
        return acc;
    };
    // the kernels cast on load only for add/multiply widening integers to
    // int64/uint64; every other cast is materialised first
    const bool castld_ok = (op == OP_ADD || op == OP_MULTIPLY) && (cd == DT_I64 || cd == DT_U64) && !dt_is_float(a_in->dtype);
    if (group > 0 && a_in->dtype != cd && (where || !castld_ok)) {
        int64_t n = c_contig(acast, a_in, cd);
        tmp_a = scratch_alloc((size_t)n * dt_bytes(cd), s);
        if (!tmp_a) return IONP_ERR_OOM;
        acast.data = tmp_a;
        if ((st = cast_impl(a_in, &acast, nullptr, s))) { cleanup(); return st; }
        a = &acast;
    }
    const IonpArr* m = nullptr;
    if (where) {
        if (!has_seed) {
            cleanup();
            return set_err(IONP_ERR_VALUE, std::string("reduction operation '") + name +
                                               "' does not have an identity, so to use a where mask one has to specify 'initial'");
        }
        int64_t mb[IONP_MAX_DIMS];
        if (!bcast_strides(where, nd, a_in->shape, mb)) {
            cleanup();
            return set_err(IONP_ERR_BROADCAST, "operands could not be broadcast together with shapes " + fmt_shape(where->shape, where->ndim) + " " + fmt_shape(a_in->shape, nd) + " ");
        }
        if (where->dtype != DT_BOOL) {
            int64_t n = c_contig(mcast, where, DT_BOOL);
            tmp_m = scratch_alloc((size_t)std::max<int64_t>(n, 1), s);
            if (!tmp_m) { cleanup(); return IONP_ERR_OOM; }
            mcast.data = tmp_m;
            if ((st = cast_impl(where, &mcast, nullptr, s))) { cleanup(); return st; }
            m = &mcast;
        } else {
            m = where;
        }
    }
    if (group == 0) {
        if (!has_seed) {
            cleanup();
            return set_err(IONP_ERR_VALUE, std::string("zero-size array to reduction operation ") + name + " which has no identity");
        }
        st = fill_seed(out, cd, seed, s);
        cleanup();
        return st;
    }

    RedDesc d;
    memset(&d, 0, sizeof(d));
    d.a = elem_ptr(a);
    d.adt = a->dtype;
    d.cd = cd;
    d.op = op;
    d.o = (void*)elem_ptr(out);
    d.odt = out->dtype;
    d.has_seed = has_seed;
    d.seed = seed;
    int64_t mstr[IONP_MAX_DIMS] = {0};
    if (m) {
        bcast_strides(m, nd, a->shape, mstr);
        d.m = (const uint8_t*)elem_ptr(m);
    }
    std::vector<Dim> kd;
    for (int i = 0; i < nd; ++i)
        if (!red[i]) kd.push_back({a->shape[i], a->strides[i], out->strides[out_dim_of[i]], mstr[i]});
    if ((st = kept_dims(kd, d, m != nullptr))) { cleanup(); return st; }

    // wide / narrow classification (ufunc.rs:6679-6700)
    std::vector<int> by_stride;
    for (int i = 0; i < nd; ++i) if (a->shape[i] > 1) by_stride.push_back(i);
    std::stable_sort(by_stride.begin(), by_stride.end(), [&](int x, int y) { return std::llabs(a->strides[x]) < std::llabs(a->strides[y]); });
    std::vector<int> wide;
    for (int ax : by_stride) { if (red[ax]) wide.push_back(ax); else break; }
    auto mem_order = [&](std::vector<int> v) {
        std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return std::llabs(a->strides[x]) > std::llabs(a->strides[y]); });
        return v;
    };
    std::vector<int> narrow;
    for (int i = 0; i < nd; ++i) if (red[i] && std::find(wide.begin(), wide.end(), i) == wide.end()) narrow.push_back(i);
    narrow = mem_order(narrow);
    // coalesce_runs over the wide axes (innermost last), innermost-first runs
    std::vector<std::pair<int64_t, int64_t>> runs;
    for (int k = 0; k < (int)wide.size(); ++k) {  // wide[0] is the innermost
        int ax = wide[k];
        if (!runs.empty() && a->strides[ax] == runs.back().second * runs.back().first) runs.back().first *= a->shape[ax];
        else runs.push_back({a->shape[ax], a->strides[ax]});
    }
    auto set_narrow = [&](const std::vector<int>& axs) -> int32_t {
        if ((int)axs.size() > RD_MAXD) return set_err(IONP_ERR_UNSUPPORTED, "too many reduced dims");
        d.nr = (int)axs.size();
        for (int i = 0; i < d.nr; ++i) { d.rshape[i] = a->shape[axs[i]]; d.rst[i] = a->strides[axs[i]]; d.mrst[i] = mstr[axs[i]]; }
        return IONP_OK;
    };

    if (m) {
        // masked paths (ufunc.rs:7213-7548)
        d.pairwise = (op == OP_ADD && (cd == DT_F32 || cd == DT_F64));
        if (pw_family) {
            if ((st = set_narrow(narrow))) { cleanup(); return st; }
            if ((int)wide.size() > RD_MAXD) { cleanup(); return set_err(IONP_ERR_UNSUPPORTED, "too many reduced dims"); }
            d.nwr = (int)wide.size();
            for (int i = 0; i < d.nwr; ++i) {  // innermost last
                int ax = wide[d.nwr - 1 - i];
                d.wrshape[i] = a->shape[ax]; d.wrst[i] = a->strides[ax]; d.mwst_raw[i] = mstr[ax];
            }
        } else {
            std::vector<int> all;
            for (int i = 0; i < nd; ++i) if (red[i]) all.push_back(i);
            if ((st = set_narrow(mem_order(all)))) { cleanup(); return st; }
        }
        st = cuda_err(launch_reduce_masked(d, s), "masked reduce launch");
        cleanup();
        return st;
    }

    if (pw_family) {
        if (narrow.empty() && runs.size() == 1 && op == OP_ADD) {
            d.w = runs[0].first;
            d.ws = runs[0].second;
            st = run_row(d, s);
        } else if (wide.empty()) {
            if ((st = set_narrow(narrow))) { cleanup(); return st; }
            st = cuda_err(launch_reduce_col(d, s), "reduce col launch");
        } else {
            if ((st = set_narrow(narrow))) { cleanup(); return st; }
            if ((int)runs.size() > RD_MAXD) { cleanup(); return set_err(IONP_ERR_UNSUPPORTED, "too many wide runs"); }
            d.nw = (int)runs.size();
            for (int i = 0; i < d.nw; ++i) { d.wshape[i] = runs[i].first; d.wst[i] = runs[i].second; }
            st = cuda_err(launch_reduce_gen(d, s), "reduce gen launch");
        }
        cleanup();
        return st;
    }
    // sequential_group order: reduced axes ascending, C order; float multiply
    // folds in memory order (sequential_group_ordered)
    std::vector<int> fold_axes;
    for (int i = 0; i < nd; ++i) if (red[i] && a->shape[i] != 1) fold_axes.push_back(i);
    if (op == OP_MULTIPLY && dt_is_float(cd)) fold_axes = mem_order(fold_axes);
    if (red_assoc(op, cd)) {
        // one run in fold order?
        std::vector<std::pair<int64_t, int64_t>> fr;
        for (int k = (int)fold_axes.size() - 1; k >= 0; --k) {
            int ax = fold_axes[k];
            if (!fr.empty() && a->strides[ax] == fr.back().second * fr.back().first) fr.back().first *= a->shape[ax];
            else fr.push_back({a->shape[ax], a->strides[ax]});
        }
        int64_t min_kept = INT64_MAX;
        for (int i = 0; i < nd; ++i) if (!red[i] && a->shape[i] > 1) min_kept = std::min<int64_t>(min_kept, std::llabs(a->strides[i]));
        if (fr.size() == 1 && std::llabs(fr[0].second) <= min_kept) {
            d.w = fr[0].first;
            d.ws = fr[0].second;
            st = run_row(d, s);
            cleanup();
            return st;
        }
    }
    if ((st = set_narrow(fold_axes))) { cleanup(); return st; }
    if (red_assoc(op, cd) && d.nr == 1 && d.adt == d.cd) {
        // too few outputs for one thread each to keep HBM busy: cut the
        // axis into 2^K parts and fold the parts in order on top
        int K = 0;
        while (d.nout < 65536 && (d.nout << K) < sm_count() * 2048 && (d.rshape[0] >> (K + 1)) >= 256 && K < 10) ++K;
        if (K > 0) {
            d.K = K;
            void* scratch = scratch_alloc((size_t)(d.nout << K) * dt_bytes(cd), s);
            if (!scratch) { cleanup(); return IONP_ERR_OOM; }
            d.scratch = scratch;
            st = cuda_err(launch_reduce_col_split(d, s), "reduce col split launch");
            if (!st) st = cuda_err(launch_reduce_row_top(d, s), "reduce col top launch");
            scratch_free(scratch, s);
            cleanup();
            return st;
        }
    }
    st = cuda_err(launch_reduce_col(d, s), "reduce col launch");
    cleanup();
    return st;
}

int32_t ionp_argext(int32_t is_max, const IonpArr* a, int32_t axis, int32_t keepdims, IonpArr* out, IonpStream stream) {
    NvtxRange nvtx_("ionp_argext");
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    if (out->dtype != DT_I64) return set_err(IONP_ERR_TYPE, "argmin/argmax output must be int64");
    cudaStream_t s = (cudaStream_t)stream;
    const int nd = a->ndim;
    const char* name = is_max ? "argmax" : "argmin";
    if (axis < -1 || axis >= std::max(nd, 1)) return set_err(IONP_ERR_AXIS, "axis out of bounds");
    if (numel(a) == 0 && (axis == -1 || nd == 0 || a->shape[axis] == 0))
        return set_err(IONP_ERR_VALUE, std::string("attempt to get ") + name + " of an empty sequence");
    if (numel(out) == 0) return IONP_OK;
    if (nd == 0) return cuda_err(cudaMemsetAsync((void*)elem_ptr(out), 0, 8, s), "argext 0-d");
    RedDesc d;
    memset(&d, 0, sizeof(d));
    d.a = elem_ptr(a);
    d.adt = d.cd = a->dtype;
    d.o = (void*)elem_ptr(out);
    d.odt = DT_I64;
    int mode = 0, tpr = 256;
    if (axis == -1) {
        // C-order ravel: flat index over all dims (unit dims dropped, C-adjacent merged)
        std::vector<Dim> g;
        for (int i = 0; i < nd; ++i) {
            if (a->shape[i] == 1) continue;
            if (!g.empty() && g.back().st == a->strides[i] * a->shape[i]) { g.back().n *= a->shape[i]; g.back().st = a->strides[i]; continue; }
            g.push_back({a->shape[i], a->strides[i], 0, 0});
        }
        if (g.empty()) g.push_back({1, 0, 0, 0});
        if ((int)g.size() > RD_MAXD) return set_err(IONP_ERR_UNSUPPORTED, "too many non-mergeable dims for argext");
        d.nr = (int)g.size();
        d.w = 1;
        for (int i = 0; i < d.nr; ++i) { d.rshape[i] = g[i].n; d.rst[i] = g[i].st; d.w *= g[i].n; }
        d.nk = 0;
        d.nout = 1;
    } else {
        std::vector<Dim> kd;
        int j = 0;
        for (int i = 0; i < nd; ++i) {
            if (i == axis) { if (keepdims) j++; continue; }
            kd.push_back({a->shape[i], a->strides[i], out->strides[j], 0});
            j++;
        }
        if ((st = kept_dims(kd, d, false))) return st;
        d.nr = 1;
        d.rshape[0] = d.w = a->shape[axis];
        d.rst[0] = d.ws = a->strides[axis];
        int64_t min_kept = INT64_MAX;
        for (int i = 0; i < nd; ++i) if (i != axis && a->shape[i] > 1) min_kept = std::min<int64_t>(min_kept, std::llabs(a->strides[i]));
        if (std::llabs(d.ws) > min_kept && d.nout >= sm_count() * 32) mode = 1;  // column scan
    }
    if (mode == 0 && axis != -1 && d.nr == 1 && d.ws == 1 && d.nk == 1 && d.kst[0] == d.w && d.nout >= sm_count() * 256 &&
        (d.w * dt_bytes(d.cd)) % 16 == 0 && d.w * dt_bytes(d.cd) <= 256 && reinterpret_cast<uintptr_t>(d.a) % 16 == 0)
        return cuda_err(launch_argext(d, is_max, 3, tpr, s), "argext narrow launch");
    if (mode == 0) {
        tpr = d.w < 64 ? 1 : d.w <= 4096 ? 32 : 256;
        int K = 0;
        while ((d.nout << K) < sm_count() * 4 && (d.w >> (K + 1)) >= 8192 && K < 16) ++K;
        d.K = K;
        void* scratch = nullptr;
        if (K > 0) {
            int64_t nt = d.nout << K;
            scratch = scratch_alloc((size_t)nt * (dt_bytes(d.cd) + 8) + 64, s);
            if (!scratch) return IONP_ERR_OOM;
            d.scratch = scratch;
        }
        st = cuda_err(launch_argext(d, is_max, 0, tpr, s), "argext launch");
        if (!st && K > 0) st = cuda_err(launch_argext(d, is_max, 2, tpr, s), "argext top launch");
        if (scratch) scratch_free(scratch, s);
        return st;
    }
    // column scan; split the axis when the outputs alone leave HBM idle
    int K = 0;
    while ((d.nout << K) < sm_count() * 2048 && (d.w >> (K + 1)) >= 256 && K < 10) ++K;
    d.K = K;
    void* scratch = nullptr;
    if (K > 0) {
        scratch = scratch_alloc((size_t)(d.nout << K) * (dt_bytes(d.cd) + 8) + 64, s);
        if (!scratch) return IONP_ERR_OOM;
        d.scratch = scratch;
    }
    st = cuda_err(launch_argext(d, is_max, 1, tpr, s), "argext col launch");
    if (!st && K > 0) st = cuda_err(launch_argext(d, is_max, 2, tpr, s), "argext top launch");
    if (scratch) scratch_free(scratch, s);
    return st;
}

}  // extern "C"
