// ionp_reduce_noalloc: ufunc.reduce for callers that may not allocate device
// memory.
//
// Some hosts of this library cannot let it call cudaMalloc: a serving process
// that reserves its whole device-memory budget at start-up and forbids later
// allocations, a host runtime that owns every device byte through its own
// arena and hands the library only its own input and output buffers, or a
// latency-critical loop where a cudaMalloc (which may synchronise the device)
// is not acceptable. ionp_reduce draws its scratch from the caching allocator,
// which calls cudaMalloc on a cache miss. This entry point runs the same row
// (pairwise-tree) reduction kernels, but keeps the per-segment partial results
// of long runs in a fixed, file-scope device array instead, and calls no
// allocating routine at all.
//
// Scope: the reductions whose fold the row kernels realise without a
// temporary -- the reduced axes form one run that holds the smallest strides
// of the array (float add: the pairwise "wide" run with no narrow axis; the
// associative ops: one run in fold order), input already in the compute
// dtype (or an integer add/multiply widened on load), no where= mask, and a
// non-empty reduced extent. Anything else returns IONP_ERR_UNSUPPORTED and
// should go through ionp_reduce.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>
#include "ionp_host.h"
#include "ionp_reduce_launch.cuh"

namespace ionp {
namespace {

// The partial sums of split runs. Every GPU that loads the library holds this
// array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_partials[IONP_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 256;
std::mutex g_addr_mu;
void* g_addr[MAX_DEVICES] = {nullptr};

// Device address of g_noalloc_partials on the current device. In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
int32_t partials_address(void** out) {
    int dev = 0;
    int32_t st = cuda_err(cudaGetDevice(&dev), "ionp_reduce_noalloc: cudaGetDevice");
    if (st) return st;
    if (dev < 0 || dev >= MAX_DEVICES) return set_err(IONP_ERR_INVALID, "ionp_reduce_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> g(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        st = cuda_err(cudaGetSymbolAddress(&p, g_noalloc_partials), "ionp_reduce_noalloc: cudaGetSymbolAddress");
        if (st) return st;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return IONP_OK;
}

constexpr int64_t SEG_LIMIT = 65536;  // longest run one CTA reduces

int tree_depth(int64_t n) {
    if (n <= PW_BLOCK) return 0;
    int64_t n2 = pw_split(n);
    return 1 + std::max(tree_depth(n2), tree_depth(n - n2));
}
std::set<int64_t> lengths_at(int64_t n, int K) {
    std::set<int64_t> cur{n};
    for (int k = 0; k < K; ++k) {
        std::set<int64_t> nx;
        for (int64_t l : cur) { int64_t n2 = pw_split(l); nx.insert(n2); nx.insert(l - n2); }
        cur.swap(nx);
    }
    return cur;
}
int threads_per_run(int64_t w) { return w <= PW_BLOCK ? 1 : w <= 2048 ? 32 : 256; }

bool identity_of(int op, int cd, uint64_t* out) {
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

int32_t unsupported(const char* why) {
    return set_err(IONP_ERR_UNSUPPORTED, std::string("ionp_reduce_noalloc: ") + why + "; use ionp_reduce");
}

}  // namespace
}  // namespace ionp

using namespace ionp;

extern "C" int32_t ionp_reduce_noalloc(int32_t op, const IonpArr* a, const int32_t* axes, int32_t naxes,
                                       int32_t keepdims, const void* initial, IonpArr* out, IonpStream stream) {
    int32_t st;
    if ((st = check_arr(a, "a")) || (st = check_arr(out, "out"))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nd = a->ndim;
    bool red[IONP_MAX_DIMS] = {false};
    for (int k = 0; k < naxes; ++k) {
        if (!axes || axes[k] < 0 || axes[k] >= std::max(nd, 1) || (k > 0 && axes[k] <= axes[k - 1]))
            return set_err(IONP_ERR_AXIS, "axes must be normalized, sorted and unique");
        if (nd > 0) red[axes[k]] = true;
    }
    int cd;
    if ((st = reduce_cd(op, a->dtype, &cd))) return st;
    if (!red_row_valid(op, cd)) return unsupported("this op's fold needs the sequential column kernel");
    const bool castld = a->dtype != cd;
    if (castld && !((op == OP_ADD || op == OP_MULTIPLY) && (cd == DT_I64 || cd == DT_U64) && !dt_is_float(a->dtype)))
        return unsupported("the input would need a converted temporary copy");
    // output shape
    int kept_nd = 0;
    for (int i = 0; i < nd; ++i) if (!red[i]) kept_nd++;
    if (out->ndim != (keepdims ? nd : kept_nd)) return set_err(IONP_ERR_VALUE, "out has the wrong number of dimensions");
    std::vector<int> out_dim_of(nd, -1);
    for (int i = 0, j = 0; i < nd; ++i) {
        if (keepdims) {
            out_dim_of[i] = i;
            if (out->shape[i] != (red[i] ? 1 : a->shape[i])) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
        } else if (!red[i]) {
            out_dim_of[i] = j;
            if (out->shape[j] != a->shape[i]) return set_err(IONP_ERR_VALUE, "out has the wrong shape");
            j++;
        }
    }
    if (numel(out) == 0) return IONP_OK;
    int64_t group = 1;
    for (int i = 0; i < nd; ++i) if (red[i]) group *= a->shape[i];
    if (group == 0) return unsupported("an empty reduced extent fills the output from a host value");

    // The reduced axes must form one run in fold order holding the smallest
    // strides (reduce_axis_pairwise_narrow_wide, ufunc.rs:6679-6700, for
    // float add; sequential_group, ufunc.rs:6546, for the associative ops).
    int64_t w = 1, ws = 1;
    std::vector<std::pair<int64_t, int64_t>> runs;  // (extent, stride), innermost first
    if (dt_is_float(cd) && op == OP_ADD) {
        // wide axes: the reduced axes that are the smallest-stride axes of
        // the whole array; any other reduced axis is narrow
        std::vector<int> by_stride;
        for (int i = 0; i < nd; ++i) if (a->shape[i] > 1) by_stride.push_back(i);
        std::stable_sort(by_stride.begin(), by_stride.end(),
                         [&](int x, int y) { return std::llabs(a->strides[x]) < std::llabs(a->strides[y]); });
        size_t nwide = 0;
        while (nwide < by_stride.size() && red[by_stride[nwide]]) ++nwide;
        for (size_t k = nwide; k < by_stride.size(); ++k)
            if (red[by_stride[k]]) return unsupported("a narrow reduced axis folds sequentially in the column kernel");
        for (size_t k = 0; k < nwide; ++k) {
            int ax = by_stride[k];
            if (!runs.empty() && a->strides[ax] == runs.back().second * runs.back().first) runs.back().first *= a->shape[ax];
            else runs.push_back({a->shape[ax], a->strides[ax]});
        }
        if (runs.size() > 1) return unsupported("the wide axes do not coalesce into one run");
    } else {
        // associative ops: one run in fold order (reduced axes ascending)
        // with no kept axis inside it
        std::vector<int> fold;
        for (int i = 0; i < nd; ++i) if (red[i] && a->shape[i] != 1) fold.push_back(i);
        for (int k = (int)fold.size() - 1; k >= 0; --k) {
            int ax = fold[k];
            if (!runs.empty() && a->strides[ax] == runs.back().second * runs.back().first) runs.back().first *= a->shape[ax];
            else runs.push_back({a->shape[ax], a->strides[ax]});
        }
        if (runs.size() > 1) return unsupported("the reduced axes do not form one strided run");
        int64_t min_kept = INT64_MAX;
        for (int i = 0; i < nd; ++i)
            if (!red[i] && a->shape[i] > 1) min_kept = std::min<int64_t>(min_kept, std::llabs(a->strides[i]));
        if (!runs.empty() && std::llabs(runs[0].second) > min_kept)
            return unsupported("a kept axis has a smaller stride than the reduced run");
    }
    if (runs.size() == 1) { w = runs[0].first; ws = runs[0].second; }

    RedDesc d;
    memset(&d, 0, sizeof(d));
    d.a = elem_ptr(a);
    d.adt = a->dtype;
    d.cd = cd;
    d.op = op;
    d.o = (void*)elem_ptr(out);
    d.odt = out->dtype;
    if (initial) { memcpy(&d.seed, initial, dt_bytes(cd)); d.has_seed = 1; }
    else d.has_seed = identity_of(op, cd, &d.seed) ? 1 : 0;
    {
        // kept dims in output order; unit dims dropped, C-adjacent dims merged
        struct KD { int64_t n, st, ost; };
        std::vector<KD> v;
        for (int i = 0; i < nd; ++i) {
            if (red[i] || a->shape[i] == 1) continue;
            KD x{a->shape[i], a->strides[i], out->strides[out_dim_of[i]]};
            if (!v.empty() && v.back().st == x.st * x.n && v.back().ost == x.ost * x.n) {
                v.back().n *= x.n; v.back().st = x.st; v.back().ost = x.ost;
                continue;
            }
            v.push_back(x);
        }
        if ((int)v.size() > RD_MAXD) return unsupported("too many non-mergeable kept dims");
        d.nk = (int)v.size();
        d.nout = 1;
        for (int i = 0; i < d.nk; ++i) {
            d.kshape[i] = v[i].n; d.kst[i] = v[i].st; d.kost[i] = v[i].ost;
            d.nout *= v[i].n;
        }
    }
    d.w = w;
    d.ws = ws;

    // Split depth: the runs longer than one CTA's segment must split; a few
    // more levels spread few long runs over the SMs, as long as the partials
    // still fit the fixed array.
    const size_t acc = (cd == DT_F16 && op == OP_ADD) ? 4 : (size_t)dt_bytes(cd);
    int K = 0;
    if (w > SEG_LIMIT)
        while (*lengths_at(w, K).rbegin() > SEG_LIMIT && K <= 2 * TOP_CHUNK_LOG) ++K;
    auto fits = [&](int k) { return k == 0 || (size_t)(d.nout << k) * acc <= (size_t)IONP_NOALLOC_SCRATCH_BYTES; };
    if (!fits(K))
        return set_err(IONP_ERR_VALUE, "ionp_reduce_noalloc: the partial results of this reduction (" +
                                           std::to_string((size_t)(d.nout << K) * acc) + " bytes) exceed the " +
                                           std::to_string((size_t)IONP_NOALLOC_SCRATCH_BYTES) +
                                           "-byte static scratch; use ionp_reduce");
    while ((d.nout << K) < sm_count() * 2 && *lengths_at(w, K + 1).begin() >= 4096 && K < 20 && fits(K + 1)) ++K;
    auto lens = lengths_at(w, K);
    int D = 0;
    for (int64_t l : lens) D = std::max(D, tree_depth(l));
    const int tpr = threads_per_run(*lens.rbegin());
    const int groups = RED_THREADS / tpr;
    const size_t nslots = tpr >= 32 ? ((size_t)1 << D) : 1;
    const size_t smem = (size_t)groups * nslots * (acc + 1) + 16;
    d.K = K;
    d.D = D;
    const int64_t ntasks = d.nout << K;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntasks + groups - 1) / groups, (int64_t)sm_count() * 8));
    if (K > 0) {
        // Every partial the top pass reads is written by the row pass of the
        // same call, so the array needs no clearing between calls.
        if ((st = partials_address(&d.scratch))) return st;
    }
    st = cuda_err(launch_reduce_row(d, tpr, smem, grid, s), "ionp_reduce_noalloc: row launch");
    if (!st && K > 0) st = cuda_err(launch_reduce_row_top(d, s), "ionp_reduce_noalloc: top launch");
    return st;
}
