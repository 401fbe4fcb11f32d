// libngpu: host runtime and C ABI (include/ngpu.h) of the B200 simulation core.
//
// Builds the per-node layout (state rows, parameter rows, junction slots)
// from the morphology and channel placement once per model, owns the device
// buffers of each resident simulation, and launches the kernels of
// sim_kernels.cuh.  No call exits, aborts or traps; every error is a negative
// return code plus a thread-local message.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/ngpu.h"
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled
#include "explore.cuh"
#include "features.cuh"
#include "ga.cuh"
#include "gemm_tc.cuh"
#include "ngpu_jit.h"
#include "sim_kernels.cuh"

using namespace ngpu;

namespace {

thread_local std::string g_err;
std::atomic<int64_t> g_launches{0};

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define NGPU_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(NGPU_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Mechanism-set tables: per mechanism, the reference parameter indices it
// reads (in the order the channel code consumes them) and its state rows.
struct MechDesc {
    std::vector<int> params;
    int state_rows;
    int cost;  // rough instruction weight, for balancing node ranges over warps
};
struct SetDesc {
    int n_params;
    std::vector<MechDesc> mechs;
    // bits that require a calcium-dynamics mechanism on the same node
    uint32_t needs_ca_dyn;
    uint32_t ca_dyn_bit;
};

// Mechanism sets generated from NMODL files (ngpu_mechset_define): their
// layout tables and device source; ids from NGPU_MECHSET_GENERATED on.
struct GenSet {
    SetDesc desc;
    std::string name, source;
};
std::mutex g_gen_mu;
std::vector<std::unique_ptr<GenSet>> g_gen;  // never shrinks: references stay valid

const GenSet* gen_set(int ms) {
    std::lock_guard<std::mutex> lock(g_gen_mu);
    const int k = ms - NGPU_MECHSET_GENERATED;
    return (k >= 0 && k < (int)g_gen.size()) ? g_gen[k].get() : nullptr;
}

bool mechset_known(int ms) {
    return ms == NGPU_MECHSET_TTPC || ms == NGPU_MECHSET_MAINEN || gen_set(ms) != nullptr;
}

const SetDesc& set_desc(int ms) {
    if (ms >= NGPU_MECHSET_GENERATED) return gen_set(ms)->desc;
    // TTPC: GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/CudaStuff.cu:220 call list.
    static const SetDesc ttpc = {
        19,
        {{{0}, 2, 40}, {{1}, 2, 40}, {{2, 3, 4, 5}, 2, 15}, {{6, 7}, 1, 20}, {{8}, 1, 20},
         {{9}, 2, 40}, {{10}, 2, 40}, {{11}, 2, 50}, {{12}, 2, 50}, {{13}, 2, 50}, {{14, 15}, 0, 4},
         {{16, 17}, 1, 20}, {{18}, 1, 20}},
        TTPC::kCaHVA | TTPC::kCaLVA, TTPC::kCaDyn};
    // Mainen: Figures/FigureS4_mainen/CParsed/AllModels.cuh:63 call list
    // (ca's cao argument is never read by the channel code).
    static const SetDesc mainen = {
        34,
        {{{0}, 2, 40}, {{}, 2, 15}, {{2, 3, 4, 5}, 1, 25}, {{6, 7, 8, 9, 10}, 1, 25},
         {{11, 12, 13, 14, 15}, 1, 25}, {{16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27}, 2, 55},
         {{28, 29}, 0, 4}, {{30, 31}, 0, 4}, {{32, 33}, 0, 4}},
        Mainen::kCa, Mainen::kCad};
    return ms == NGPU_MECHSET_TTPC ? ttpc : mainen;
}

void* dmalloc(size_t bytes, int* rc) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        *rc = fail(NGPU_E_NOMEM, std::string("cudaMalloc(") + std::to_string(bytes) +
                                     "): " + cudaGetErrorString(e));
        return nullptr;
    }
    return p;
}

// Host-side per-node layout of a model.
struct HostNode {
    int32_t parent;
    uint32_t mask;
    int32_t srow;  // first channel-state row
    int32_t prow;  // first parameter row
};

}  // namespace

struct ngpu_sim;
struct ngpu_model {
    // ngpu_run's last simulation, reused by the next call of the same shape
    ngpu_sim* run_cache = nullptr;
    std::mutex run_mu;
    int n = 0, n_sections = 0, mechset = 0, n_mech = 0, n_params = 0;
    std::vector<int> parent, section;
    std::vector<double> a, b, cm;
    std::vector<uint32_t> mask;
    std::vector<HostNode> info;
    std::vector<int> row_param, row_sec;
    int slab_rows = 0, ptab_rows = 0;
    int64_t state_vars = 0, param_reads = 0;
    std::vector<int> weight;        // per-node channel cost
    std::vector<int2> rows;         // (state rows, parameter rows) per node
    std::vector<int> perm, inv;     // internal node -> caller's node (group representative), group -> internal
    // stiff-edge contraction (see contract_stiff_edges)
    int n_caller = 0;                    // nodes in the caller's numbering
    std::vector<int> node_internal;      // caller node -> internal node
    std::vector<double> density_scale;   // caller node -> area(node) / area(its internal node)
};

namespace {

// Stiff-edge contraction.
//
// Exports of NEURON models can hold compartments of near-zero area, whose
// per-area axial couplings reach 1e21 while ordinary ones are 1e-4 .. 10.
// Such compartments are tied to their neighbours so tightly that their
// voltages agree far below FP32 (or FP64) resolution, yet each step's
// right-hand side multiplies their voltage differences, rounding included,
// by those couplings, and the rounding noise leaks into the rest of the
// cell.  Nodes joined by such edges are therefore merged into one node
// before anything else (the voltage difference across a merged edge is the
// edge current over a conductance >= 1e7 times the median one).
//
// Rows are per unit membrane area, so the relative areas follow from the
// coefficients themselves: row i holds a_i = -G_i / area_i, its parent's row
// b_i = -G_i / area_parent, hence area_i / area_parent = b_i / a_i and the
// edge's absolute conductance G_i = |a_i| area_i.  A merged group keeps one
// row, normalised to the area of its representative (the member with
// channels, or else the largest); the others contribute capacitance only
// (sum of cm area) and their couplings are rescaled to the representative's
// area.  Two members with channels are never merged, since the kernel
// computes one channel set per node.
struct Contraction {
    std::vector<int> group;        // caller node -> group (groups numbered by first member)
    std::vector<int> rep, top;     // group -> representative / top member (caller numbering)
    std::vector<double> area;      // caller node -> area relative to the root
    int n_groups = 0;
};

constexpr double kStiffRatio = 1e7;

static Contraction contract_stiff_edges(int n, const int32_t* parent, const double* a, const double* b,
                                        const std::vector<uint32_t>& mask, bool enabled) {
    Contraction C;
    C.area.assign(n, 1.0);
    std::vector<double> G(n, 0.0);
    std::vector<char> ok(n, 0);
    for (int i = 1; i < n; ++i) {
        const double r = b[i] / a[i];
        if (std::isfinite(r) && r > 0.0 && std::isfinite(C.area[parent[i]] * r)) {
            C.area[i] = C.area[parent[i]] * r;
            G[i] = std::fabs(a[i]) * C.area[i];
            ok[i] = G[i] > 0.0 && std::isfinite(G[i]);
        } else {
            C.area[i] = C.area[parent[i]];
        }
    }
    std::vector<int> up(n);
    for (int i = 0; i < n; ++i) up[i] = i;
    std::vector<int> chan(n, -1);  // per set root: its member with channels
    for (int i = 0; i < n; ++i)
        if (mask[i]) chan[i] = i;
    auto find = [&](int x) {
        while (up[x] != x) x = up[x] = up[up[x]];
        return x;
    };
    if (enabled && n > 2) {
        std::vector<double> gs;
        for (int i = 1; i < n; ++i)
            if (ok[i]) gs.push_back(G[i]);
        if (!gs.empty()) {
            std::nth_element(gs.begin(), gs.begin() + gs.size() / 2, gs.end());
            const double thr = kStiffRatio * gs[gs.size() / 2];
            std::vector<int> stiff;
            for (int i = 1; i < n; ++i)
                if (ok[i] && G[i] > thr) stiff.push_back(i);
            std::stable_sort(stiff.begin(), stiff.end(), [&](int x, int y) { return G[x] > G[y]; });
            for (int i : stiff) {
                int x = find(i), y = find(parent[i]);
                if (x == y || (chan[x] >= 0 && chan[y] >= 0)) continue;
                if (y > x) std::swap(x, y);  // keep the smaller caller index as the set root
                up[x] = y;
                if (chan[y] < 0) chan[y] = chan[x];
            }
        }
    }
    C.group.assign(n, -1);
    std::vector<int> gid_of_root(n, -1);
    for (int i = 0; i < n; ++i) {
        const int r = find(i);
        if (gid_of_root[r] < 0) {
            gid_of_root[r] = C.n_groups++;
            C.top.push_back(i);  // first member in a parent-before-child order is the top
            C.rep.push_back(-1);
        }
        C.group[i] = gid_of_root[r];
    }
    for (int i = 0; i < n; ++i) {
        const int g = C.group[i];
        const int r = find(i);
        if (chan[r] >= 0) {
            C.rep[g] = chan[r];
        } else if (C.rep[g] < 0 || C.area[i] > C.area[C.rep[g]]) {
            C.rep[g] = i;
        }
    }
    return C;
}

}  // namespace

// Split of the tree for one CTA of W warps (see sim_kernels.cuh).  Nodes are
// already in heavy-first depth-first order (model creation reorders them), so
// every heavy path is a run of consecutive nodes.  Separator nodes cut the
// tree into work items ("components") of at most ~1/W of the channel cost:
//   plain component    a whole subtree [r, r + size(r)) hanging off separator u
//   segment component  a heavy-path piece r..l-1 (the spine) ending just above
//                      a lower separator l, plus the light subtrees of the
//                      spine nodes, which occupy [l + size(l), r + size(r))
// The separators form a small tree (the skeleton) that warp 0 solves.
struct Comp {
    int r, u, l;          // root, upper separator, lower separator (-1: plain)
    int lk;               // index of l in the separator list (-1: plain)
    int light_lo, light_hi;
    int64_t weight;
};

struct Partition {
    std::vector<Comp> comps;        // by decreasing weight (the dynamic schedule order)
    std::vector<int> seps;          // separator nodes, ascending
    std::vector<int> sep_par;       // skeleton parent (index into seps), -1 for the root
    std::vector<int> sep_comp;      // segment component whose lower separator this is, or -1
    std::vector<int> jslot, pslot;
    int n_jslots = 0;
};

static Partition make_partition(const ngpu_model* m, int W, int items_per_warp = 2) {
    const int N = m->n;
    const std::vector<int>& par = m->parent;
    Partition P;
    std::vector<std::vector<int>> kids(N);
    for (int i = 1; i < N; ++i) kids[par[i]].push_back(i);
    std::vector<int64_t> subw(N, 0);
    std::vector<int> subn(N, 1);
    for (int i = N - 1; i >= 0; --i) {
        subw[i] += m->weight[i];
        if (i > 0) {
            subw[par[i]] += subw[i];
            subn[par[i]] += subn[i];
        }
    }
    auto heavy = [&](int i) { return (i + 1 < N && par[i + 1] == i) ? i + 1 : -1; };
    // items of at most ~1/(k W) of the cost: k items per warp balance the dynamic queue
    // better than one, at a few more separators (the simulation chooses k per model)
    const int64_t parts = W > 1 ? (int64_t)std::max(1, items_per_warp) * W : 1;
    const int64_t target = std::max<int64_t>(1, (subw[0] + parts - 1) / parts);
    std::vector<char> is_sep(N, 0);
    is_sep[0] = 1;
    struct Raw { int r, l; };
    std::vector<Raw> raw;
    auto cweight = [&](const Raw& c) { return subw[c.r] - (c.l >= 0 ? subw[c.l] : 0); };
    for (int c : kids[0]) raw.push_back({c, -1});
    for (;;) {
        int best = -1;
        for (size_t k = 0; k < raw.size(); ++k)
            if (W > 1 && cweight(raw[k]) > target && (best < 0 || cweight(raw[k]) > cweight(raw[best])))
                best = (int)k;
        if (best < 0) break;
        Raw C = raw[best];
        raw.erase(raw.begin() + best);
        // walk the spine from r; cut at the first node whose own cost (itself
        // plus its light subtrees) would take the part above over the target
        int64_t acc = 0;
        int s = C.r;
        for (int i = C.r;; i = heavy(i)) {
            int64_t own = m->weight[i];
            for (int c : kids[i])
                if (c != heavy(i)) own += subw[c];
            const int h = heavy(i);
            if (acc + own > target || h < 0 || h == C.l) { s = i; break; }
            acc += own;
        }
        is_sep[s] = 1;
        if (s > C.r) raw.push_back({C.r, s});
        const int h = heavy(s);
        if (h >= 0 && h != C.l) raw.push_back({h, C.l});
        for (int c : kids[s])
            if (c != h) raw.push_back({c, -1});
    }
    for (int i = 0; i < N; ++i)
        if (is_sep[i]) P.seps.push_back(i);
    std::vector<int> sep_index(N, -1);
    for (size_t k = 0; k < P.seps.size(); ++k) sep_index[P.seps[k]] = (int)k;
    for (const Raw& c : raw) {
        Comp q;
        q.r = c.r;
        q.u = par[c.r];
        q.l = c.l;
        q.lk = c.l >= 0 ? sep_index[c.l] : -1;
        if (c.l >= 0) {
            q.light_lo = c.l + subn[c.l];
            q.light_hi = c.r + subn[c.r];
        } else {
            q.light_lo = c.r;
            q.light_hi = c.r + subn[c.r];
        }
        q.weight = cweight(c);
        P.comps.push_back(q);
    }
    std::sort(P.comps.begin(), P.comps.end(), [](const Comp& x, const Comp& y) {
        return x.weight != y.weight ? x.weight > y.weight : x.r < y.r;
    });
    // skeleton links
    std::vector<int> seg_of_lower(N, -1);
    for (size_t k = 0; k < P.comps.size(); ++k)
        if (P.comps[k].l >= 0) seg_of_lower[P.comps[k].l] = (int)k;
    P.sep_par.assign(P.seps.size(), -1);
    P.sep_comp.assign(P.seps.size(), -1);
    for (size_t k = 1; k < P.seps.size(); ++k) {
        const int sn = P.seps[k];
        if (is_sep[par[sn]]) {
            P.sep_par[k] = sep_index[par[sn]];
        } else {
            const int ci = seg_of_lower[sn];
            P.sep_comp[k] = ci;
            P.sep_par[k] = sep_index[P.comps[ci].u];
        }
    }
    // junction slots: every separator; every parent of a child that is not
    // node+1 or that roots a component
    std::vector<char> comp_root(N, 0);
    for (const Comp& c : P.comps) comp_root[c.r] = 1;
    std::vector<char> need(N, 0);
    for (int i = 0; i < N; ++i)
        if (is_sep[i]) need[i] = 1;
    for (int i = 1; i < N; ++i)
        if (!is_sep[i] && (par[i] != i - 1 || comp_root[i])) need[par[i]] = 1;
    P.jslot.assign(N, -1);
    P.pslot.assign(N, -1);
    for (int i = 0; i < N; ++i)
        if (need[i]) P.jslot[i] = P.n_jslots++;
    for (int i = 1; i < N; ++i)
        if (!is_sep[i] && (par[i] != i - 1 || comp_root[i])) P.pslot[i] = P.jslot[par[i]];
    return P;
}

struct ngpu_batch;
struct ngpu_sim {
    ngpu_model* m = nullptr;
    int n_sets = 0, n_stim = 0, n_inst = 0, n_groups = 0, n_pad = 0, precision = 0;
    // device buffers
    void* d_nodes = nullptr;
    void* d_vbuf = nullptr;
    void* d_slab = nullptr;
    float* d_ptab = nullptr;
    void* d_scr = nullptr;
    DevComp* d_comps = nullptr;
    DevSep* d_seps = nullptr;
    void* d_sepv = nullptr;
    int n_warps = 1;
    Partition part;
    double* d_jacc = nullptr;
    void* d_jx = nullptr;
    int* d_inst_stim = nullptr;
    int* d_bad = nullptr;
    int* d_row_param = nullptr;
    int* d_row_sec = nullptr;
    float* d_amps = nullptr;
    float* d_dts = nullptr;
    float* d_trace = nullptr;
    size_t trace_bytes = 0;
    float* d_tmp_out = nullptr;
    size_t tmp_out_bytes = 0;
    float* d_params_in = nullptr;  // the caller's [set][param][section] table, uploaded
    size_t params_in_bytes = 0;
    void* h_stage = nullptr;       // pinned host staging for host-buffer copies
    size_t stage_bytes = 0;
    // stimulus / recording (internal node numbering)
    int nt = 0, stim_node = 0;
    double stim_scale = 0.0;
    std::vector<int> rec_nodes;       // per requested site
    std::vector<int> rec_cols;        // column of each requested site
    int n_rec_unique = 0, rec_every = 1, n_samples = 0;
    float v_init = -65.f;
    bool has_params = false, has_stim = false, initialized = false;
    // runtime-specialised kernels the node records' classes refer to
    // (nullptr: the ahead-of-time kernels, every node generic)
    const ngpu_jit::Module* jit = nullptr;
    ngpu_batch* batch = nullptr;  // the batch whose kernels this simulation's records follow
    int s2_stage = 0;             // skeleton solved from shared memory (see sim_kernels.cuh)
    int items_per_warp = 2;       // work items per warp in the tree split
    ngpu_jit::Folds folds;        // parameters the runtime-specialised kernel compiles in
    uint2* d_prange = nullptr;    // [ptab_rows] bit-pattern range of each parameter row
    unsigned long long* d_phash = nullptr;  // [ptab_rows] hash of each parameter row
    std::vector<int32_t> prow_canon;  // parameter block start -> the block it reads (identical values)
    bool ch_prefetch = true;      // the runtime-specialised kernel compiles the channel-pass L2 prefetch in
    int layout = NGPU_LAYOUT_LANE_INSTANCE;  // lane = instance, or one warp per instance (thread-item)
    int ti_warps = 4;             // thread-item layout: instances (warps) per CTA
    int ti_items = 32;            // thread-item layout: work items per instance's tree
};

// Rows (state and parameter) a node's channel update reads, on average; the
// channel-pass prefetch is compiled in from kPrefetchRowsPerNode on.  Measured
// on B200: the HH-type cells (~30 rows per node) run 7-13 % faster with it,
// the TTPC-like cell (~12) 7 % faster without it.
constexpr double kPrefetchRowsPerNode = 20.0;

// Thread-item layout: work items per instance at most / by default, and the
// SM count the default CTA shape spreads a small batch over.
constexpr int kMaxTiItems = 512;
// Lane-instance CTAs of up to 16 warps (runtime-compiled kernels bounded for
// 3 CTAs per SM; the ahead-of-time kernels take up to kMaxWarps).
constexpr int kMaxWideWarps = 16;
constexpr int kDefaultTiItems = 32;
constexpr int kSmCount = 148;

static double rows_per_node(const ngpu_model* m) {
    return m->n > 0 ? (double)(m->state_vars + m->param_reads) / m->n : 0.0;
}

// CTAs per SM that `smem` bytes of dynamic shared memory and W warps of 80
// registers allow (228 KB per SM, 1 KB of it reserved per CTA).
// CTAs per SM a wide (more than 8 warps) lane-instance kernel is compiled
// for: 1 when the batch has at most one group per SM (registers are then
// plentiful: 16 warps get 128), else 3 (one wave for large batches).
static int wide_ctas_per_sm(int n_groups) { return n_groups <= kSmCount ? 1 : 3; }

static int ctas_per_sm(size_t smem, int W, int n_groups) {
    // kernels of up to 8 warps use 80 registers; wider ones are compiled for wide_ctas_per_sm
    const int by_regs = W > kMaxWarps ? wide_ctas_per_sm(n_groups) : 65536 / (kLanes * W * 80);
    const int by_smem = (int)((228 * 1024) / (smem + 1024));
    return std::max(1, std::min(std::min(by_regs, by_smem), 64 / W));
}

// Stage the skeleton in shared memory when that costs no occupancy.
template <typename R>
static int choose_s2_stage(int n_nodes, int n_seps, int W, int n_groups) {
    if (W < 2 || n_seps < 2) return 0;
    const size_t plain = SmemPlan<R>::bytes(n_nodes), staged = SmemPlan<R>::bytes(n_nodes, n_seps, 1);
    return staged <= 227 * 1024 && ctas_per_sm(staged, W, n_groups) >= ctas_per_sm(plain, W, n_groups) ? 1 : 0;
}

template <typename R>
static SimArgs<R> make_args(ngpu_sim* s) {
    SimArgs<R> A;
    const ngpu_model* m = s->m;
    A.nodes = (const NodeRec<R>*)s->d_nodes;
    A.n_nodes = m->n;
    A.vbuf = (R*)s->d_vbuf;
    A.slab = (R*)s->d_slab;
    A.slab_rows = m->slab_rows;
    A.ptab = s->d_ptab;
    A.ptab_rows = m->ptab_rows;
    A.scr = (R*)s->d_scr;
    A.jacc = s->d_jacc;
    A.jx = (R*)s->d_jx;
    A.n_jslots = s->part.n_jslots;
    A.amps = s->d_amps;
    A.dts = s->d_dts;
    A.nt = s->nt;
    A.stim_node = s->stim_node;
    A.stim_scale = s->stim_scale;
    A.inst_stim = s->d_inst_stim;
    A.trace = s->d_trace;
    A.n_rec = s->n_rec_unique;
    A.rec_every = s->rec_every;
    A.n_inst_pad = s->n_pad;
    A.n_inst = s->n_inst;
    A.v_init = s->v_init;
    A.bad = s->d_bad;
    A.n_warps = s->n_warps;
    A.comps = s->d_comps;
    A.n_comps = (int)s->part.comps.size();
    A.seps = s->d_seps;
    A.n_seps = (int)s->part.seps.size();
    A.sepv = (R*)s->d_sepv;
    A.s2_stage = s->s2_stage;
    return A;
}

template <typename R>
static cudaError_t launch_init(ngpu_sim* s, cudaStream_t st) {
    SimArgs<R> A = make_args<R>(s);
    const int threads = kLanes * std::min(s->n_warps, kMaxWarps);  // any warp count serves the init
    if (s->jit) {
        void* args[] = {(void*)&A};
        const cudaError_t e = cudaLaunchKernel((const void*)s->jit->init, dim3(s->n_groups), dim3(threads), args, 0, st);
        g_launches++;
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (s->m->mechset == NGPU_MECHSET_TTPC) k_sim_init<R, 0><<<s->n_groups, threads, 0, st>>>(A);
    else k_sim_init<R, 1><<<s->n_groups, threads, 0, st>>>(A);
    g_launches++;
    return cudaGetLastError();
}

// Thread-item layout: one warp per instance, ti_warps instances per CTA.
template <typename R>
static cudaError_t launch_advance_ti(ngpu_sim* s, int t0, int n, cudaStream_t st) {
    SimArgs<R> A = make_args<R>(s);
    const int W = s->ti_warps;
    const int ctas = (s->n_inst + W - 1) / W;
    const size_t smem = SmemPlan<R>::ti_bytes(s->m->n, (int)s->part.seps.size(), W);
    cudaError_t e;
    const void* k;
    if (s->jit) k = (const void*)s->jit->advance_ti;
    else if (s->m->mechset == NGPU_MECHSET_TTPC) k = (const void*)k_sim_advance_ti<R, 0>;
    else k = (const void*)k_sim_advance_ti<R, 1>;
    if (!k) return cudaErrorInvalidDeviceFunction;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&A, (void*)&t0, (void*)&n};
    e = cudaLaunchKernel(k, dim3(ctas), dim3(kLanes * W), args, smem, st);
    g_launches++;
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename R>
static cudaError_t launch_advance(ngpu_sim* s, int t0, int n, cudaStream_t st) {
    if (s->layout == NGPU_LAYOUT_WARP_INSTANCE) return launch_advance_ti<R>(s, t0, n, st);
    SimArgs<R> A = make_args<R>(s);
    const int threads = kLanes * s->n_warps;
    const size_t smem = SmemPlan<R>::bytes(s->m->n, (int)s->part.seps.size(), s->s2_stage);
    cudaError_t e;
    if (s->jit) {
        const void* k = (const void*)s->jit->advance;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        void* args[] = {(void*)&A, (void*)&t0, (void*)&n};
        e = cudaLaunchKernel(k, dim3(s->n_groups), dim3(threads), args, smem, st);
        g_launches++;
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (s->m->mechset == NGPU_MECHSET_TTPC) {
        e = cudaFuncSetAttribute(k_sim_advance<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_sim_advance<R, 0><<<s->n_groups, threads, smem, st>>>(A, t0, n);
    } else {
        e = cudaFuncSetAttribute(k_sim_advance<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_sim_advance<R, 1><<<s->n_groups, threads, smem, st>>>(A, t0, n);
    }
    g_launches++;
    return cudaGetLastError();
}

extern "C" {

const char* ngpu_last_error(void) { return g_err.c_str(); }
int ngpu_abi_version(void) { return NGPU_ABI_VERSION; }
int64_t ngpu_launch_count(int32_t reset) {
    return reset ? g_launches.exchange(0) : g_launches.load();
}

int ngpu_device_count(int32_t* n) {
    int c = 0;
    const cudaError_t e = cudaGetDeviceCount(&c);
    if (n) *n = e == cudaSuccess ? c : 0;
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    return NGPU_OK;
}

int ngpu_set_device(int32_t device) {
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return NGPU_OK;
}

int ngpu_mechset_info(int32_t mechset, int32_t* n_mech, int32_t* n_params) {
    if (!mechset_known(mechset)) return fail(NGPU_E_INVALID, "unknown mechanism set");
    const SetDesc& sd = set_desc(mechset);
    if (n_mech) *n_mech = (int32_t)sd.mechs.size();
    if (n_params) *n_params = sd.n_params;
    return NGPU_OK;
}

int ngpu_mechset_define(const char* name, const char* source, int32_t n_mech, const int32_t* state_rows,
                        const int32_t* n_mech_params, const int32_t* mech_param_index, int32_t n_params,
                        const int32_t* cost, int32_t* mechset) {
    if (!name || !source || !state_rows || !n_mech_params || !cost || !mechset)
        return fail(NGPU_E_INVALID, "null argument");
    if (n_mech < 1 || n_mech > 16) return fail(NGPU_E_INVALID, "a mechanism set holds 1..16 mechanisms");
    if (n_params < 0 || n_params > 4096) return fail(NGPU_E_INVALID, "n_params out of range");
    auto g = std::make_unique<GenSet>();
    g->name = name;
    g->source = source;
    g->desc.n_params = n_params;
    g->desc.needs_ca_dyn = 0;
    g->desc.ca_dyn_bit = 0;
    int off = 0;
    for (int k = 0; k < n_mech; ++k) {
        if (state_rows[k] < 0 || state_rows[k] > 64 || n_mech_params[k] < 0 || n_mech_params[k] > 64 || cost[k] < 0)
            return fail(NGPU_E_INVALID, "mechanism " + std::to_string(k) + ": bad row counts or cost");
        MechDesc md;
        md.state_rows = state_rows[k];
        md.cost = cost[k];
        for (int j = 0; j < n_mech_params[k]; ++j) {
            const int pi = mech_param_index ? mech_param_index[off + j] : -1;
            if (pi < 0 || pi >= n_params) return fail(NGPU_E_INVALID, "parameter index out of range");
            md.params.push_back(pi);
        }
        off += n_mech_params[k];
        g->desc.mechs.push_back(md);
    }
    std::lock_guard<std::mutex> lock(g_gen_mu);
    if (g_gen.size() >= 1000) return fail(NGPU_E_INVALID, "too many mechanism sets defined");
    g_gen.push_back(std::move(g));
    *mechset = NGPU_MECHSET_GENERATED + (int32_t)g_gen.size() - 1;
    return NGPU_OK;
}

int ngpu_model_create(int32_t n_nodes, const int32_t* parent, const double* a, const double* b,
                      const double* cm, const int32_t* section, int32_t n_sections,
                      int32_t mechset, const uint8_t* mech_mask, ngpu_model** out) {
    if (!out) return fail(NGPU_E_INVALID, "out is null");
    *out = nullptr;
    if (n_nodes < 1 || !parent || !a || !b || !cm || !section || !mech_mask || n_sections < 1)
        return fail(NGPU_E_INVALID, "model arrays missing or empty");
    if (!mechset_known(mechset)) return fail(NGPU_E_INVALID, "unknown mechanism set");
    const SetDesc& sd = set_desc(mechset);
    const int NM = (int)sd.mechs.size();
    if (parent[0] != -1) return fail(NGPU_E_INVALID, "parent[0] must be -1 (node 0 is the root)");
    for (int i = 1; i < n_nodes; ++i)
        if (parent[i] < 0 || parent[i] >= i)
            return fail(NGPU_E_INVALID, "parent[" + std::to_string(i) + "] = " +
                                            std::to_string(parent[i]) +
                                            " is not an earlier node (Hines order required)");
    for (int i = 0; i < n_nodes; ++i) {
        if (section[i] < 0 || section[i] >= n_sections)
            return fail(NGPU_E_INVALID, "section index out of range at node " + std::to_string(i));
        if (!std::isfinite(a[i]) || !std::isfinite(b[i]) || !std::isfinite(cm[i]) || cm[i] < 0)
            return fail(NGPU_E_INVALID, "non-finite coefficient at node " + std::to_string(i));
    }
    if (n_nodes > 32767) return fail(NGPU_E_INVALID, "at most 32767 nodes per morphology");
    if (NM > 16) return fail(NGPU_E_INVALID, "at most 16 mechanisms per set");
    std::vector<uint32_t> maskc(n_nodes, 0u);
    for (int k = 0; k < NM; ++k)
        for (int i = 0; i < n_nodes; ++i)
            if (mech_mask[(size_t)k * n_nodes + i]) maskc[i] |= (1u << k);
    // Stiff edges merged first; the tree below is the merged one (groups,
    // numbered parent-before-child), with rows normalised to each group's
    // representative.  NGPU_CONTRACT=0 keeps every node (diagnostics).
    const char* cev = getenv("NGPU_CONTRACT");
    const Contraction Ct = contract_stiff_edges(n_nodes, parent, a, b, maskc, !(cev && cev[0] == '0'));
    const int n_caller = n_nodes;
    n_nodes = Ct.n_groups;
    std::vector<int32_t> parent_g(n_nodes), section_g(n_nodes);
    std::vector<double> a_g(n_nodes), b_g(n_nodes), cm_g(n_nodes, 0.0);
    std::vector<uint32_t> mask0(n_nodes);
    for (int g = 0; g < n_nodes; ++g) {
        const int t = Ct.top[g], r = Ct.rep[g];
        const double ar = Ct.area[r];
        parent_g[g] = g == 0 ? -1 : Ct.group[parent[t]];
        section_g[g] = section[r];
        mask0[g] = maskc[r];
        // row g's coupling to its parent, per the representative's area; the
        // parent row's entry, per the parent group's representative's area
        a_g[g] = g == 0 ? a[0] : a[t] * (Ct.area[t] / ar);
        b_g[g] = g == 0 ? b[0] : b[t] * (Ct.area[parent[t]] / Ct.area[Ct.rep[parent_g[g]]]);
    }
    for (int i = 0; i < n_caller; ++i) cm_g[Ct.group[i]] += cm[i] * (Ct.area[i] / Ct.area[Ct.rep[Ct.group[i]]]);
    parent = parent_g.data();
    a = a_g.data();
    b = b_g.data();
    cm = cm_g.data();
    section = section_g.data();
    // Internal node order: heavy-first depth-first (children by decreasing
    // channel-cost subtree weight), so heavy paths are runs of consecutive
    // nodes.  Any Hines order the caller gives is accepted; stimulus and
    // recording nodes are mapped through the permutation.
    std::vector<int64_t> subw(n_nodes, 0);
    for (int i = n_nodes - 1; i >= 0; --i) {
        int wt = 12;
        for (int k = 0; k < NM; ++k)
            if (mask0[i] & (1u << k)) wt += sd.mechs[k].cost;
        subw[i] += wt;
        if (i > 0) subw[parent[i]] += subw[i];
    }
    std::vector<std::vector<int>> kids(n_nodes);
    for (int i = 1; i < n_nodes; ++i) kids[parent[i]].push_back(i);
    std::vector<int> order;
    order.reserve(n_nodes);
    {
        std::vector<int> stack{0};
        while (!stack.empty()) {
            const int v = stack.back();
            stack.pop_back();
            order.push_back(v);
            std::vector<int> ks = kids[v];
            std::stable_sort(ks.begin(), ks.end(), [&](int x, int y) { return subw[x] > subw[y]; });
            for (auto it = ks.rbegin(); it != ks.rend(); ++it) stack.push_back(*it);
        }
    }
    ngpu_model* m = new (std::nothrow) ngpu_model();
    if (!m) return fail(NGPU_E_NOMEM, "host allocation failed");
    m->perm.assign(n_nodes, 0);
    for (int i = 0; i < n_nodes; ++i) m->perm[i] = Ct.rep[order[i]];
    m->inv.assign(n_nodes, 0);
    for (int i = 0; i < n_nodes; ++i) m->inv[order[i]] = i;
    m->n_caller = n_caller;
    m->node_internal.assign(n_caller, 0);
    m->density_scale.assign(n_caller, 1.0);
    for (int j = 0; j < n_caller; ++j) {
        const int g = Ct.group[j];
        m->node_internal[j] = m->inv[g];
        m->density_scale[j] = Ct.area[j] / Ct.area[Ct.rep[g]];
    }
    m->n = n_nodes;
    m->n_sections = n_sections;
    m->mechset = mechset;
    m->n_mech = NM;
    m->n_params = sd.n_params;
    m->parent.resize(n_nodes);
    m->section.resize(n_nodes);
    m->a.resize(n_nodes);
    m->b.resize(n_nodes);
    m->cm.resize(n_nodes);
    m->mask.resize(n_nodes);
    for (int i = 0; i < n_nodes; ++i) {
        const int o = order[i];
        m->parent[i] = i == 0 ? -1 : m->inv[parent[o]];
        m->section[i] = section[o];
        m->a[i] = a[o];
        m->b[i] = b[o];
        m->cm[i] = cm[o];
        m->mask[i] = mask0[o];
    }
    for (int i = 0; i < n_nodes; ++i) {
        if ((m->mask[i] & sd.needs_ca_dyn) && !(m->mask[i] & sd.ca_dyn_bit)) {
            const int o = m->perm[i];
            delete m;
            return fail(NGPU_E_INVALID, "node " + std::to_string(o) +
                                            " has a calcium current without calcium dynamics "
                                            "(its reversal potential would be infinite)");
        }
    }
    // state and parameter rows
    std::map<std::pair<int, uint32_t>, int> prow_of;
    m->info.resize(n_nodes);
    int srow = 0;
    for (int i = 0; i < n_nodes; ++i) {
        HostNode& ni = m->info[i];
        ni.parent = m->parent[i];
        ni.mask = m->mask[i];
        ni.srow = srow;
        int srows = 0, wt = 12;
        std::vector<int> plist;
        for (int k = 0; k < NM; ++k)
            if (ni.mask & (1u << k)) {
                srows += sd.mechs[k].state_rows;
                wt += sd.mechs[k].cost;
                plist.insert(plist.end(), sd.mechs[k].params.begin(), sd.mechs[k].params.end());
            }
        srow += srows;
        m->weight.push_back(wt);
        m->state_vars += srows;
        m->param_reads += (int64_t)plist.size();
        auto key = std::make_pair(m->section[i], ni.mask);
        auto it = prow_of.find(key);
        if (it == prow_of.end()) {
            int first = (int)m->row_param.size();
            for (int p : plist) {
                m->row_param.push_back(p);
                m->row_sec.push_back(m->section[i]);
            }
            it = prow_of.emplace(key, first).first;
        }
        ni.prow = it->second;
        m->rows.push_back(make_int2(srows, (int)plist.size()));
    }
    m->slab_rows = std::max(1, srow);
    if (m->row_param.size() > 65535) {
        delete m;
        return fail(NGPU_E_INVALID, "too many distinct parameter rows (more than 65535)");
    }
    m->ptab_rows = std::max(1, (int)m->row_param.size());
    if (m->row_param.empty()) {
        m->row_param.push_back(0);
        m->row_sec.push_back(0);
    }
    *out = m;
    return NGPU_OK;
}

static void sim_free(ngpu_sim* s);

int ngpu_model_destroy(ngpu_model* m) {
    if (m && m->run_cache) sim_free(m->run_cache);
    delete m;
    return NGPU_OK;
}

int ngpu_model_layout(const ngpu_model* m, int32_t* state_rows, int32_t* param_rows,
                      int32_t* n_jslots, int64_t* state_vars, int64_t* param_reads) {
    if (!m) return fail(NGPU_E_INVALID, "null model");
    if (state_rows) *state_rows = m->slab_rows;
    if (param_rows) *param_rows = m->ptab_rows;
    if (n_jslots) *n_jslots = make_partition(m, 1).n_jslots;
    if (state_vars) *state_vars = m->state_vars;
    if (param_reads) *param_reads = m->param_reads;
    return NGPU_OK;
}

int ngpu_model_nodes(const ngpu_model* m, int32_t* n_internal, int32_t* n_caller, int32_t* node_internal,
                     double* density_scale) {
    if (!m) return fail(NGPU_E_INVALID, "null model");
    if (n_internal) *n_internal = m->n;
    if (n_caller) *n_caller = m->n_caller;
    for (int j = 0; j < m->n_caller; ++j) {
        if (node_internal) node_internal[j] = m->node_internal[j];
        if (density_scale) density_scale[j] = m->density_scale[j];
    }
    return NGPU_OK;
}

int ngpu_model_arrays(const ngpu_model* m, int32_t* parent, double* a, double* b, double* cm) {
    if (!m) return fail(NGPU_E_INVALID, "null model");
    for (int i = 0; i < m->n; ++i) {
        if (parent) parent[i] = m->parent[i];
        if (a) a[i] = m->a[i];
        if (b) b[i] = m->b[i];
        if (cm) cm[i] = m->cm[i];
    }
    return NGPU_OK;
}

int ngpu_model_partition(const ngpu_model* m, int32_t n_warps, int32_t* sep_flag, int32_t* item,
                         int32_t* jslot, int32_t* pslot, int32_t* n_jslots) {
    if (!m) return fail(NGPU_E_INVALID, "null model");
    // warps of a CTA, or (up to kMaxTiItems) the lanes of one instance's warp
    if (n_warps < 1 || n_warps > kMaxTiItems) return fail(NGPU_E_INVALID, "n_warps out of range");
    Partition P = make_partition(m, n_warps);
    std::vector<int> owner(m->n, -1), sep(m->n, 0);
    for (int i : P.seps) sep[i] = 1;
    for (size_t k = 0; k < P.comps.size(); ++k) {
        const Comp& c = P.comps[k];
        if (c.l >= 0)
            for (int i = c.r; i < c.l; ++i) owner[i] = (int)k;
        for (int i = c.light_lo; i < c.light_hi; ++i) owner[i] = (int)k;
    }
    for (int j = 0; j < m->n_caller; ++j) {  // j: node in the caller's numbering
        const int i = m->node_internal[j];
        if (sep_flag) sep_flag[j] = sep[i];
        if (item) item[j] = owner[i];
        if (jslot) jslot[j] = P.jslot[i];
        if (pslot) pslot[j] = P.pslot[i];
    }
    if (n_jslots) *n_jslots = P.n_jslots;
    return NGPU_OK;
}

int ngpu_model_split_info(const ngpu_model* m, int32_t n_warps, int32_t* perm, int32_t* n_comps,
                          int32_t* comps, int32_t max_comps, int32_t* n_seps, int32_t* seps,
                          int32_t max_seps, int32_t* jslot, int32_t* pslot) {
    if (!m) return fail(NGPU_E_INVALID, "null model");
    // warps of a CTA, or (up to kMaxTiItems) the lanes of one instance's warp
    if (n_warps < 1 || n_warps > kMaxTiItems) return fail(NGPU_E_INVALID, "n_warps out of range");
    Partition P = make_partition(m, n_warps);
    if (perm)
        for (int i = 0; i < m->n; ++i) perm[i] = m->perm[i];
    if (n_comps) *n_comps = (int32_t)P.comps.size();
    if (n_seps) *n_seps = (int32_t)P.seps.size();
    if (comps)
        for (int k = 0; k < (int)P.comps.size() && k < max_comps; ++k) {
            const Comp& c = P.comps[k];
            const int32_t v[6] = {c.r, c.u, c.l, c.lk, c.light_lo, c.light_hi};
            for (int j = 0; j < 6; ++j) comps[6 * k + j] = v[j];
        }
    if (seps)
        for (int k = 0; k < (int)P.seps.size() && k < max_seps; ++k) {
            seps[3 * k] = P.seps[k];
            seps[3 * k + 1] = P.sep_par[k];
            seps[3 * k + 2] = P.sep_comp[k];
        }
    for (int i = 0; i < m->n; ++i) {
        if (jslot) jslot[i] = P.jslot[i];
        if (pslot) pslot[i] = P.pslot[i];
    }
    return NGPU_OK;
}

static void sim_free(ngpu_sim* s) {
    if (!s) return;
    void* ptrs[] = {s->d_nodes, s->d_vbuf, s->d_slab, s->d_ptab, s->d_scr, s->d_jacc, s->d_jx,
                    s->d_inst_stim, s->d_bad, s->d_row_param, s->d_row_sec, s->d_amps,
                    s->d_dts, s->d_trace, s->d_tmp_out, s->d_comps, s->d_seps, s->d_sepv, s->d_prange,
                    s->d_phash, s->d_params_in};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->h_stage) cudaFreeHost(s->h_stage);
    delete s;
}

// Host-buffer copies.  A copy between pageable host memory and the device
// runs at a few GB/s: the driver stages it through its own pinned buffer,
// one page at a time on one thread, and a fresh destination (a new numpy
// array) also takes its first-touch page faults on that thread.  The
// simulation's own pinned staging buffer (grown to the largest copy, kept
// for the next call) moves at full link speed, and the host side of the copy
// (pageable <-> pinned) is split over several threads.  Measured on B200 for
// the 98 MB trace of the TTPC-like batch: 25 ms through the driver's path.
static void* sim_stage(ngpu_sim* s, size_t bytes) {
    if (s->stage_bytes >= bytes) return s->h_stage;
    if (s->h_stage) cudaFreeHost(s->h_stage);
    s->h_stage = nullptr;
    s->stage_bytes = 0;
    if (cudaHostAlloc(&s->h_stage, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();  // no pinned memory: the caller takes the driver's path
        s->h_stage = nullptr;
        return nullptr;
    }
    s->stage_bytes = bytes;
    return s->h_stage;
}

static void host_copy_parallel(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPerThreadMin = size_t(4) << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t want = std::min<size_t>(std::min<size_t>(16, std::max(1u, hw / 2)), bytes / kPerThreadMin);
    const size_t T = std::max<size_t>(1, want);
    if (T == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t part = (bytes / T + 4095) / 4096 * 4096;
    std::vector<std::thread> th;
    th.reserve(T - 1);
    for (size_t k = 1; k < T; ++k) {
        const size_t lo = std::min(bytes, k * part), hi = std::min(bytes, lo + part);
        if (hi > lo) th.emplace_back([=] { std::memcpy((char*)dst + lo, (const char*)src + lo, hi - lo); });
    }
    std::memcpy(dst, src, std::min(bytes, part));
    for (auto& t : th) t.join();
}

// The device side of the simulation's tree split (s->part): junction
// accumulators and dV slots, work items, separators and segment links,
// (re)allocated for the split and its items and separators uploaded.
static int sim_upload_split(ngpu_sim* s) {
    void** old[] = {(void**)&s->d_jacc, (void**)&s->d_jx, (void**)&s->d_comps, (void**)&s->d_seps, &s->d_sepv};
    for (void** p : old)
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    const size_t G = (size_t)s->n_groups, L = kLanes, esz = s->precision == NGPU_FP64 ? 8 : 4;
    const size_t nj = std::max(1, s->part.n_jslots), ns = std::max<size_t>(1, s->part.seps.size());
    int rc = NGPU_OK;
    if (!(s->d_jacc = (double*)dmalloc(G * 2 * nj * L * sizeof(double), &rc))) return rc;
    if (!(s->d_jx = dmalloc(G * nj * L * esz, &rc))) return rc;
    if (!(s->d_comps = (DevComp*)dmalloc(sizeof(DevComp) * std::max<size_t>(1, s->part.comps.size()), &rc))) return rc;
    if (!(s->d_seps = (DevSep*)dmalloc(sizeof(DevSep) * ns, &rc))) return rc;
    if (!(s->d_sepv = dmalloc(G * 4 * ns * L * esz, &rc))) return rc;
    std::vector<DevComp> dc;
    for (const Comp& c : s->part.comps) dc.push_back({c.r, c.u, c.l, c.lk, c.light_lo, c.light_hi});
    std::vector<DevSep> ds;
    for (size_t k = 0; k < s->part.seps.size(); ++k)
        ds.push_back({s->part.seps[k], s->part.sep_par[k], s->part.sep_comp[k], 0});
    if (!dc.empty()) NGPU_CUDA(cudaMemcpy(s->d_comps, dc.data(), sizeof(DevComp) * dc.size(), cudaMemcpyHostToDevice));
    NGPU_CUDA(cudaMemcpy(s->d_seps, ds.data(), sizeof(DevSep) * ds.size(), cudaMemcpyHostToDevice));
    return NGPU_OK;
}

int ngpu_sim_create(ngpu_model* m, int32_t n_sets, int32_t n_stim, int32_t precision,
                    ngpu_sim** out) {
    return ngpu_sim_create_ex(m, n_sets, n_stim, precision, 0, out);
}

int ngpu_sim_create_ex(ngpu_model* m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t n_warps,
                       ngpu_sim** out) {
    return ngpu_sim_create_shaped(m, n_sets, n_stim, precision, n_warps, 0, out);
}

int ngpu_sim_create_shaped(ngpu_model* m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t n_warps,
                           int32_t items_per_warp, ngpu_sim** out) {
    if (n_warps < 0 || n_warps > kMaxWarps)
        return fail(NGPU_E_INVALID, "n_warps must be 0 (automatic) or 1.." + std::to_string(kMaxWarps));
    return ngpu_sim_create_layout(m, n_sets, n_stim, precision, NGPU_LAYOUT_LANE_INSTANCE, n_warps, items_per_warp,
                                  out);
}

int ngpu_sim_create_layout(ngpu_model* m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t layout,
                           int32_t cta_warps, int32_t items, ngpu_sim** out) {
    if (!out) return fail(NGPU_E_INVALID, "out is null");
    *out = nullptr;
    if (layout != NGPU_LAYOUT_LANE_INSTANCE && layout != NGPU_LAYOUT_WARP_INSTANCE)
        return fail(NGPU_E_INVALID, "layout must be NGPU_LAYOUT_LANE_INSTANCE or NGPU_LAYOUT_WARP_INSTANCE");
    const bool ti = layout == NGPU_LAYOUT_WARP_INSTANCE;
    const int32_t n_warps = cta_warps, items_per_warp = ti ? 0 : items;
    if (ti ? (items < 0 || items > kMaxTiItems) : (items < 0 || items > 8))
        return fail(NGPU_E_INVALID, ti ? "items must be 0 (automatic) or 1.." + std::to_string(kMaxTiItems)
                                       : std::string("items_per_warp must be 0 (automatic) or 1..8"));
    const int max_w = ti ? kMaxWarps : kMaxWideWarps;
    if (n_warps < 0 || n_warps > max_w)
        return fail(NGPU_E_INVALID, "n_warps must be 0 (automatic) or 1.." + std::to_string(max_w));
    if (!m) return fail(NGPU_E_INVALID, "null model");
    if (n_sets < 1 || n_stim < 1) return fail(NGPU_E_INVALID, "need n_sets >= 1 and n_stim >= 1");
    if (precision != NGPU_FP32 && precision != NGPU_FP64)
        return fail(NGPU_E_INVALID, "precision must be NGPU_FP32 or NGPU_FP64");
    if ((int64_t)n_sets * n_stim > (int64_t)1 << 30) return fail(NGPU_E_INVALID, "too many instances");
    {
        const size_t need = precision == NGPU_FP64 ? SmemPlan<double>::bytes(m->n) : SmemPlan<float>::bytes(m->n);
        if (need > 227 * 1024)
            return fail(NGPU_E_INVALID, "morphology too large for the shared-memory solve plan (" +
                                            std::to_string(m->n) + " nodes)");
    }
    ngpu_sim* s = new (std::nothrow) ngpu_sim();
    if (!s) return fail(NGPU_E_NOMEM, "host allocation failed");
    s->m = m;
    s->n_sets = n_sets;
    s->n_stim = n_stim;
    s->n_inst = n_sets * n_stim;
    s->n_groups = (s->n_inst + kLanes - 1) / kLanes;
    s->n_pad = s->n_groups * kLanes;
    s->precision = precision;
    const size_t esz = precision == NGPU_FP64 ? 8 : 4;
    const size_t G = (size_t)s->n_groups, L = kLanes;
    int rc = NGPU_OK;
    // warps per CTA and the tree split over them
    // warps per CTA: a batch of at most one 32-instance group per SM leaves SMs
    // idle, so its CTAs get up to 16 warps (a finer split of the tree, the
    // runtime-compiled kernel at one CTA per SM: the HH cell at 2457
    // instances runs 1.4x faster, the TTPC-like cell at 33 instances 1.5x);
    // larger batches up to 8 (three CTAs per SM at 80 registers)
    int W = std::min(8, std::max(1, m->n / 48));
    if (s->n_groups <= kSmCount && !ti && ngpu_jit::enabled() && ngpu_jit::nvrtc().ok)
        W = std::min(kMaxWideWarps, std::max(1, m->n / 32));
    if (const char* ev = getenv("NGPU_WARPS")) W = std::max(1, std::min(kMaxWideWarps, atoi(ev)));
    if (n_warps > 0) W = n_warps;
    W = std::min(W, m->n);
    s->n_warps = W;
    s->ch_prefetch = rows_per_node(m) >= kPrefetchRowsPerNode;
    if (const char* ev = getenv("NGPU_CH_PREFETCH")) s->ch_prefetch = atoi(ev) != 0;
    // without the prefetch, finer items balance better (TTPC-like: +4 % from 2 to 3 per warp);
    // the autotuner searches this per morphology
    s->items_per_warp = s->ch_prefetch ? 2 : 3;
    if (const char* ev = getenv("NGPU_ITEMS_PER_WARP")) s->items_per_warp = std::max(1, std::min(8, atoi(ev)));
    if (items_per_warp > 0) s->items_per_warp = items_per_warp;
    if (ti) {
        // one warp per instance: the tree split into ti_items items for the
        // warp's lanes; CTAs of ti_warps instances, enough CTAs for every SM
        // first (the layout serves batches too small to fill the GPU)
        s->layout = NGPU_LAYOUT_WARP_INSTANCE;
        s->n_warps = kMaxWarps;  // the initialisation kernel's warps (any count serves it)
        s->ti_items = items > 0 ? items : kDefaultTiItems;
        s->ti_items = std::min(s->ti_items, m->n);
        s->ti_warps = n_warps > 0 ? n_warps
                                  : std::min(kMaxWarps, std::max(1, (s->n_inst + kSmCount - 1) / kSmCount));
        s->part = make_partition(m, s->ti_items, 1);
        s->s2_stage = 0;
        const size_t need = precision == NGPU_FP64
                                ? SmemPlan<double>::ti_bytes(m->n, (int)s->part.seps.size(), s->ti_warps)
                                : SmemPlan<float>::ti_bytes(m->n, (int)s->part.seps.size(), s->ti_warps);
        if (need > 227 * 1024) {
            sim_free(s);
            return fail(NGPU_E_INVALID, "thread-item layout: " + std::to_string(need) +
                                            " bytes of shared memory per CTA; use fewer instances per CTA or items");
        }
    } else {
        s->part = make_partition(m, W, s->items_per_warp);
        s->s2_stage = precision == NGPU_FP64 ? choose_s2_stage<double>(m->n, (int)s->part.seps.size(), W, s->n_groups)
                                             : choose_s2_stage<float>(m->n, (int)s->part.seps.size(), W, s->n_groups);
    }
#define ALLOC(field, type, bytes)                              \
    s->field = (type)dmalloc((bytes), &rc);                    \
    if (!s->field) {                                           \
        sim_free(s);                                           \
        return rc;                                             \
    }
    ALLOC(d_nodes, void*, (precision == NGPU_FP64 ? sizeof(NodeRec<double>) : sizeof(NodeRec<float>)) * m->n);
    ALLOC(d_vbuf, void*, G * 2 * m->n * L * esz);
    ALLOC(d_slab, void*, G * m->slab_rows * L * esz);
    ALLOC(d_ptab, float*, G * m->ptab_rows * L * sizeof(float));
    ALLOC(d_scr, void*, G * 3 * m->n * L * esz);
    ALLOC(d_inst_stim, int*, sizeof(int) * s->n_pad);
    ALLOC(d_bad, int*, sizeof(int) * s->n_pad);
    ALLOC(d_row_param, int*, sizeof(int) * m->row_param.size());
    ALLOC(d_row_sec, int*, sizeof(int) * m->row_sec.size());
#undef ALLOC
    if ((rc = sim_upload_split(s)) != NGPU_OK) {
        sim_free(s);
        return rc;
    }
    std::vector<int> inst_stim(s->n_pad);
    for (int k = 0; k < s->n_pad; ++k) inst_stim[k] = std::min(k, s->n_inst - 1) % n_stim;
    cudaMemcpy(s->d_inst_stim, inst_stim.data(), sizeof(int) * s->n_pad, cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_row_param, m->row_param.data(), sizeof(int) * m->row_param.size(),
               cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_row_sec, m->row_sec.data(), sizeof(int) * m->row_sec.size(),
               cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemset(s->d_bad, 0, sizeof(int) * s->n_pad);
    if (e != cudaSuccess) {
        sim_free(s);
        return fail(NGPU_E_CUDA, std::string("sim create: ") + cudaGetErrorString(e));
    }
    // default recording: the root, every step
    s->rec_nodes = {0};
    s->rec_cols = {0};
    s->n_rec_unique = 1;
    *out = s;
    return NGPU_OK;
}

int ngpu_sim_destroy(ngpu_sim* s) {
    sim_free(s);
    return NGPU_OK;
}

int ngpu_sim_layout(const ngpu_sim* s, int32_t* layout, int32_t* cta_warps, int32_t* items) {
    if (!s) return fail(NGPU_E_INVALID, "null sim");
    const bool ti = s->layout == NGPU_LAYOUT_WARP_INSTANCE;
    if (layout) *layout = s->layout;
    if (cta_warps) *cta_warps = ti ? s->ti_warps : s->n_warps;
    if (items) *items = ti ? s->ti_items : s->items_per_warp;
    return NGPU_OK;
}

static int sim_upload_nodes(ngpu_sim* s);

// Parameters with one value (the same bits) in every parameter set and every
// section whose nodes use them: the runtime-specialised kernel compiles them
// in (param_fold.cuh).  Wherever that kernel runs (either precision), with
// runtime compilation on and NGPU_PARAM_FOLD not 0.  New values
// after initialisation re-select the kernel before the next launch.
// Parameter blocks (the rows of one section and mechanism combination) that
// hold the same values at every instance as another block of the same
// combination: their nodes read that block's rows instead.  A fit gives its
// parameters per region, so most sections repeat another section's values;
// sharing shrinks the parameter rows the kernels touch (TTPC-like cell: 1788
// rows per group of 32 instances) to the distinct ones, which stay in cache.
// The values read are the same bits, so results are unchanged.  Candidates
// are grouped by a hash of each row and confirmed by an exact comparison on
// the device.  NGPU_PARAM_DEDUP=0 turns it off.
static int sim_share_param_blocks(ngpu_sim* s, std::vector<int32_t>* canon_out) {
    const ngpu_model* m = s->m;
    canon_out->clear();
    const char* ev = getenv("NGPU_PARAM_DEDUP");
    if ((ev && ev[0] == '0') || m->ptab_rows < 2) return NGPU_OK;
    int rc = NGPU_OK;
    if (!s->d_phash) {
        s->d_phash = (unsigned long long*)dmalloc(sizeof(unsigned long long) * m->ptab_rows, &rc);
        if (!s->d_phash) return rc;
    }
    k_ptab_hash<<<m->ptab_rows, 256>>>(s->d_ptab, m->ptab_rows, s->n_groups, s->d_phash);
    g_launches++;
    std::vector<unsigned long long> h(m->ptab_rows);
    NGPU_CUDA(cudaMemcpy(h.data(), s->d_phash, sizeof(h[0]) * m->ptab_rows, cudaMemcpyDeviceToHost));
    // blocks: first row -> (rows, mask), from the nodes that read them
    std::map<int, std::pair<int, uint32_t>> blocks;
    for (int i = 0; i < m->n; ++i)
        if (m->rows[i].y > 0) blocks[m->info[i].prow] = {m->rows[i].y, m->mask[i]};
    std::map<std::vector<unsigned long long>, int> first;   // (mask, rows, row hashes) -> first block
    std::vector<int3> pairs;
    for (const auto& b : blocks) {
        std::vector<unsigned long long> key = {b.second.second, (unsigned long long)b.second.first};
        key.insert(key.end(), h.begin() + b.first, h.begin() + b.first + b.second.first);
        auto it = first.find(key);
        if (it == first.end()) first.emplace(std::move(key), b.first);
        else pairs.push_back(make_int3(it->second, b.first, b.second.first));
    }
    if (pairs.empty()) return NGPU_OK;
    int3* d_pairs = (int3*)dmalloc(sizeof(int3) * pairs.size(), &rc);
    if (!d_pairs) return rc;
    int* d_same = (int*)dmalloc(sizeof(int) * pairs.size(), &rc);
    if (!d_same) {
        cudaFree(d_pairs);
        return rc;
    }
    std::vector<int> same(pairs.size(), 0);
    cudaError_t e = cudaMemcpy(d_pairs, pairs.data(), sizeof(int3) * pairs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_ptab_blocks_equal<<<(unsigned)pairs.size(), 256>>>(s->d_ptab, m->ptab_rows, s->n_groups, d_pairs, d_same);
        g_launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(same.data(), d_same, sizeof(int) * pairs.size(), cudaMemcpyDeviceToHost);
    cudaFree(d_pairs);
    cudaFree(d_same);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("parameter blocks: ") + cudaGetErrorString(e));
    std::vector<int32_t> canon(m->ptab_rows);
    for (int r = 0; r < m->ptab_rows; ++r) canon[r] = r;
    bool any = false;
    for (size_t k = 0; k < pairs.size(); ++k)
        if (same[k]) {
            canon[pairs[k].y] = pairs[k].x;
            any = true;
        }
    if (any) *canon_out = std::move(canon);
    return NGPU_OK;
}

extern "C++" {  // defined with the batch, outside this C-linkage block
static const ngpu_jit::Folds& batch_folds(const ngpu_batch* b);
static int batch_refold(ngpu_batch* b);
}

static int sim_find_folds(ngpu_sim* s) {
    const ngpu_model* m = s->m;
    ngpu_jit::Folds folds;
    const char* ev = getenv("NGPU_PARAM_FOLD");
    const bool on = ngpu_jit::enabled() &&
                    !(ev && ev[0] == '0') && m->ptab_rows > 0;
    if (on) {
        if (!s->d_prange) {
            int rc = NGPU_OK;
            s->d_prange = (uint2*)dmalloc(sizeof(uint2) * m->ptab_rows, &rc);
            if (!s->d_prange) return rc;
        }
        k_ptab_range<<<m->ptab_rows, 256>>>(s->d_ptab, m->ptab_rows, s->n_groups, s->d_prange);
        g_launches++;
        std::vector<uint2> rng(m->ptab_rows);
        NGPU_CUDA(cudaMemcpy(rng.data(), s->d_prange, sizeof(uint2) * m->ptab_rows, cudaMemcpyDeviceToHost));
        std::vector<int> state(m->n_params, 0);        // 0 unseen, 1 one value so far, 2 varies
        std::vector<unsigned> bits(m->n_params, 0);
        for (int r = 0; r < m->ptab_rows; ++r) {
            const int p = m->row_param[r];
            const uint2 b = rng[r];
            const bool finite = (b.x & 0x7F800000u) != 0x7F800000u;
            if (b.x != b.y || !finite || (state[p] == 1 && bits[p] != b.x)) state[p] = 2;
            else if (state[p] == 0) {
                state[p] = 1;
                bits[p] = b.x;
            }
        }
        for (int p = 0; p < m->n_params; ++p)
            if (state[p] == 1) {
                float v;
                std::memcpy(&v, &bits[p], 4);
                folds.emplace_back(p, v);
            }
    }
    std::vector<int32_t> canon;
    const int rc = sim_share_param_blocks(s, &canon);
    if (rc != NGPU_OK) return rc;
    const bool changed = folds != s->folds || canon != s->prow_canon;
    s->folds = std::move(folds);
    s->prow_canon = std::move(canon);
    if (s->batch) {  // the batch's kernel folds what its members share: still true for this member?
        bool holds = true;
        for (const auto& x : batch_folds(s->batch))
            if (std::find(s->folds.begin(), s->folds.end(), x) == s->folds.end()) holds = false;
        if (!holds) return batch_refold(s->batch);
    }
    if (changed && s->initialized) return sim_upload_nodes(s);
    return NGPU_OK;
}

int ngpu_sim_set_params(ngpu_sim* s, const float* params, int32_t on_device) {
    if (!s || !params) return fail(NGPU_E_INVALID, "null sim or params");
    const ngpu_model* m = s->m;
    const size_t n = (size_t)s->n_sets * m->n_params * m->n_sections;
    const float* src = params;
    if (!on_device) {
        // the upload buffer stays with the simulation for the next call
        const size_t bytes = n * sizeof(float);
        if (s->params_in_bytes < bytes) {
            if (s->d_params_in) cudaFree(s->d_params_in);
            s->d_params_in = nullptr;
            s->params_in_bytes = 0;
            int rc = NGPU_OK;
            s->d_params_in = (float*)dmalloc(bytes, &rc);
            if (!s->d_params_in) return rc;
            s->params_in_bytes = bytes;
        }
        cudaError_t e;
        if (void* stg = sim_stage(s, bytes)) {
            host_copy_parallel(stg, params, bytes);
            e = cudaMemcpyAsync(s->d_params_in, stg, bytes, cudaMemcpyHostToDevice, 0);
            if (e == cudaSuccess) e = cudaStreamSynchronize(0);  // the staging buffer is free again
        } else {
            e = cudaMemcpy(s->d_params_in, params, bytes, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("params upload: ") + cudaGetErrorString(e));
        src = s->d_params_in;
    }
    const size_t total = (size_t)s->n_groups * m->ptab_rows * kLanes;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    k_gather_params<<<blocks, 256>>>(src, s->d_row_param, s->d_row_sec, m->ptab_rows, m->n_params,
                                     m->n_sections, s->n_stim, s->n_inst, s->n_groups, s->d_ptab);
    g_launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("param gather: ") + cudaGetErrorString(e));
    s->has_params = true;
    return sim_find_folds(s);
}

int ngpu_sim_set_stimulus(ngpu_sim* s, int32_t nt, const float* amps, const float* dts,
                          int32_t stim_node, float stim_area_um2, int32_t on_device) {
    if (!s || !amps || !dts) return fail(NGPU_E_INVALID, "null sim or stimulus arrays");
    if (nt < 1) return fail(NGPU_E_INVALID, "nt must be >= 1");
    if (stim_node < 0 || stim_node >= s->m->n_caller) return fail(NGPU_E_INVALID, "stim_node out of range");
    if (!(stim_area_um2 > 0.f) || !std::isfinite(stim_area_um2))
        return fail(NGPU_E_INVALID, "stimulus area must be positive");
    if (!on_device) {
        for (int t = 0; t < nt; ++t)
            if (!(dts[t] > 0.f) || !std::isfinite(dts[t]))
                return fail(NGPU_E_INVALID, "dt must be positive and finite at step " + std::to_string(t));
    }
    if (s->d_amps) cudaFree(s->d_amps);
    if (s->d_dts) cudaFree(s->d_dts);
    s->d_amps = nullptr;
    s->d_dts = nullptr;
    int rc = NGPU_OK;
    s->d_amps = (float*)dmalloc(sizeof(float) * (size_t)nt * s->n_stim, &rc);
    if (!s->d_amps) return rc;
    s->d_dts = (float*)dmalloc(sizeof(float) * (size_t)nt, &rc);
    if (!s->d_dts) return rc;
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    NGPU_CUDA(cudaMemcpy(s->d_amps, amps, sizeof(float) * (size_t)nt * s->n_stim, kind));
    NGPU_CUDA(cudaMemcpy(s->d_dts, dts, sizeof(float) * (size_t)nt, kind));
    s->nt = nt;
    s->stim_node = s->m->node_internal[stim_node];
    // density over the internal node's area (differs only for a merged node)
    s->stim_scale = 100.0 / (double)stim_area_um2 * s->m->density_scale[stim_node];
    s->has_stim = true;
    s->initialized = false;
    return NGPU_OK;
}

int ngpu_sim_set_recording(ngpu_sim* s, int32_t n_rec, const int32_t* rec_nodes, int32_t rec_every) {
    if (!s) return fail(NGPU_E_INVALID, "null sim");
    if (n_rec < 1 || !rec_nodes) return fail(NGPU_E_INVALID, "need at least one recording site");
    if (rec_every < 1) return fail(NGPU_E_INVALID, "rec_every must be >= 1");
    std::vector<int> uniq;
    std::vector<int> cols(n_rec);
    for (int r = 0; r < n_rec; ++r) {
        if (rec_nodes[r] < 0 || rec_nodes[r] >= s->m->n_caller)
            return fail(NGPU_E_INVALID, "recording node out of range");
        const int node = s->m->node_internal[rec_nodes[r]];  // merged nodes share one column
        auto it = std::find(uniq.begin(), uniq.end(), node);
        if (it == uniq.end()) {
            cols[r] = (int)uniq.size();
            uniq.push_back(node);
        } else {
            cols[r] = (int)(it - uniq.begin());
        }
    }
    s->rec_nodes.assign(n_rec, 0);
    for (int r = 0; r < n_rec; ++r) s->rec_nodes[r] = s->m->node_internal[rec_nodes[r]];
    s->rec_cols = cols;
    s->n_rec_unique = (int)uniq.size();
    s->rec_every = rec_every;
    s->initialized = false;
    return NGPU_OK;
}

// The mechanism masks a simulation's (or batch's) kernel is compiled for.
// Whether the kernel is compiled without the generic channel path: only
// when the compiled classes hold every mask in `all` (no node takes it), and
// only for kernels without the channel-pass prefetch.  Measured on B200:
// without the path the TTPC-like cell runs 6 % faster and the TTPC set
// generated from its .mod files 16 % (its generic path alone made it spill);
// the HH-type cells, compiled with the prefetch, run 2-4 % slower.
static bool masks_cover(const std::vector<uint32_t>& picked, const std::vector<uint32_t>& all, bool prefetch) {
    if (prefetch) return false;
    for (uint32_t x : all)
        if (std::find(picked.begin(), picked.end(), x) == picked.end()) return false;
    return true;
}

static std::vector<uint32_t> model_masks(const ngpu_model* m) {
    std::vector<uint32_t> v(m->mask.begin(), m->mask.end());
    return v;
}

// Node records with this run's split, recording columns and mechanism
// classes, uploaded to the device.  The classes follow the
// runtime-specialised kernels of the simulation's batch, or its own.

// Host side of an initialisation: node records, the trace buffer (kept when
// its size is unchanged, so the device addresses a captured graph holds stay
// valid), the error flags.
static int sim_prepare_init(ngpu_sim* s, float v_init, cudaStream_t st) {
    if (!s) return fail(NGPU_E_INVALID, "null sim");
    if (!s->has_params) return fail(NGPU_E_STATE, "set_params must precede init");
    if (!s->has_stim) return fail(NGPU_E_STATE, "set_stimulus must precede init");
    if (!std::isfinite(v_init)) return fail(NGPU_E_INVALID, "v_init must be finite");
    const int rc = sim_upload_nodes(s);
    if (rc != NGPU_OK) return rc;
    s->n_samples = (s->nt + s->rec_every - 1) / s->rec_every;
    const size_t tbytes = sizeof(float) * (size_t)s->n_samples * s->n_rec_unique * s->n_pad;
    if (!s->d_trace || s->trace_bytes != tbytes) {
        if (s->d_trace) cudaFree(s->d_trace);
        s->d_trace = nullptr;
        int rc = NGPU_OK;
        s->d_trace = (float*)dmalloc(tbytes, &rc);
        if (!s->d_trace) return rc;
        s->trace_bytes = tbytes;
    }
    NGPU_CUDA(cudaMemsetAsync(s->d_bad, 0, sizeof(int) * s->n_pad, st));
    s->v_init = v_init;
    return NGPU_OK;
}

int ngpu_sim_init(ngpu_sim* s, float v_init, void* cuda_stream) {
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const int rc = sim_prepare_init(s, v_init, st);
    if (rc != NGPU_OK) return rc;
    cudaError_t e = s->precision == NGPU_FP64 ? launch_init<double>(s, st) : launch_init<float>(s, st);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("init launch: ") + cudaGetErrorString(e));
    s->initialized = true;
    return NGPU_OK;
}

int ngpu_sim_advance(ngpu_sim* s, int32_t t0, int32_t n_steps, void* cuda_stream) {
    if (!s) return fail(NGPU_E_INVALID, "null sim");
    if (!s->initialized) return fail(NGPU_E_STATE, "init must precede advance");
    if (t0 < 0 || n_steps < 0 || (int64_t)t0 + n_steps > s->nt)
        return fail(NGPU_E_INVALID, "step range outside the stimulus");
    if (n_steps == 0) return NGPU_OK;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    cudaError_t e = s->precision == NGPU_FP64 ? launch_advance<double>(s, t0, n_steps, st)
                                              : launch_advance<float>(s, t0, n_steps, st);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("advance launch: ") + cudaGetErrorString(e));
    return NGPU_OK;
}

}  // extern "C"

// ---- several simulations in one launch ------------------------------------
struct ngpu_batch {
    std::vector<ngpu_sim*> sims;
    int precision = 0, mechset = 0, threads = 0, total_ctas = 0;
    size_t smem = 0;
    // a captured run (init + chunked advances), reused while its arguments hold
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> graph_key;
    int graph_kernels = 0;  // kernels one replay launches
    // runtime-specialised kernels over the members' masks (nullptr: ahead of time)
    const ngpu_jit::Module* jit = nullptr;
    ngpu_jit::Folds folds;  // parameters every member holds at one, the same, value
};

// The folds that hold for every member (same parameter, same value).
static ngpu_jit::Folds batch_common_folds(const ngpu_batch* b) {
    if (b->sims.empty()) return {};
    ngpu_jit::Folds out = b->sims[0]->folds;
    for (size_t k = 1; k < b->sims.size(); ++k) {
        const ngpu_jit::Folds& f = b->sims[k]->folds;
        ngpu_jit::Folds keep;
        for (const auto& x : out)
            if (std::find(f.begin(), f.end(), x) != f.end()) keep.push_back(x);
        out.swap(keep);
    }
    return out;
}

static const ngpu_jit::Folds& batch_folds(const ngpu_batch* b) { return b->folds; }
static void batch_drop_graph(ngpu_batch* b);
static int batch_select_kernels(ngpu_batch* b);

// A member's new parameter values break a fold of the batch's kernel: fold
// what every member still shares, select that kernel, drop the captured run
// (it holds the old kernel) and re-upload the initialised members' records.
static int batch_refold(ngpu_batch* b) {
    b->folds = batch_common_folds(b);
    batch_drop_graph(b);
    const int rc = batch_select_kernels(b);
    if (rc != NGPU_OK) return rc;
    for (ngpu_sim* t : b->sims)
        if (t->initialized) {
            const int r2 = sim_upload_nodes(t);
            if (r2 != NGPU_OK) return r2;
        }
    return NGPU_OK;
}

static int sim_upload_nodes(ngpu_sim* s) {
    const ngpu_model* m = s->m;
    s->jit = nullptr;
    const GenSet* gs = gen_set(m->mechset);
    {  // FP32 and FP64 alike (generated sets have no other kernel)
        if (s->batch) {
            s->jit = s->batch->jit;
        } else {
            const std::vector<uint32_t> all = model_masks(m), picked = ngpu_jit::pick_masks(all, kMaxClasses);
            s->jit = ngpu_jit::module(m->mechset, s->precision == NGPU_FP64, picked, gs ? &gs->source : nullptr,
                                      s->ch_prefetch, s->folds, masks_cover(picked, all, s->ch_prefetch),
                                      s->layout == NGPU_LAYOUT_WARP_INSTANCE,
                                      s->layout == NGPU_LAYOUT_LANE_INSTANCE ? std::max(8, s->n_warps) : 8,
                                      wide_ctas_per_sm(s->n_groups));
        }
        if (gs && !s->jit)
            return fail(NGPU_E_CUDA, "mechanism set '" + gs->name +
                                         "' runs only through runtime compilation: " + ngpu_jit::last_log());
        if (!s->jit && s->layout == NGPU_LAYOUT_LANE_INSTANCE && s->n_warps > kMaxWarps)
            return fail(NGPU_E_CUDA, "CTAs of more than " + std::to_string(kMaxWarps) +
                                         " warps run only through runtime compilation: " + ngpu_jit::last_log());
    }
    std::vector<int> uniq(s->n_rec_unique, -1);
    for (size_t r = 0; r < s->rec_nodes.size(); ++r) uniq[s->rec_cols[r]] = s->rec_nodes[r];
    std::vector<int> rec(m->n, -1);
    for (int c = 0; c < s->n_rec_unique; ++c) rec[uniq[c]] = c;
    auto fill = [&](auto* recs) {
        for (int i = 0; i < m->n; ++i) {
            auto& q = recs[i];
            using RT = std::remove_reference_t<decltype(q.a)>;
            q.a = (RT)m->a[i];
            q.b = (RT)m->b[i];
            q.cm = (RT)(m->cm[i] / 1000.0);
            q.srow = m->info[i].srow;
            q.parent = (int16_t)m->parent[i];
            q.jslot = (int16_t)s->part.jslot[i];
            q.pslot = (int16_t)s->part.pslot[i];
            q.rec = (int16_t)rec[i];
            q.mask = (uint16_t)m->mask[i];
            q.prow = (uint16_t)(s->prow_canon.empty() ? m->info[i].prow : s->prow_canon[m->info[i].prow]);
            q.srows = (uint8_t)m->rows[i].x;
            q.prows = (uint8_t)m->rows[i].y;
            q.cls = (uint8_t)ngpu_jit::class_of(s->jit, (uint32_t)m->mask[i], kGenericClass);
            q.pad_ = 0;
        }
    };
    if (s->precision == NGPU_FP64) {
        std::vector<NodeRec<double>> recs(m->n);
        fill(recs.data());
        NGPU_CUDA(cudaMemcpy(s->d_nodes, recs.data(), sizeof(recs[0]) * m->n, cudaMemcpyHostToDevice));
    } else {
        std::vector<NodeRec<float>> recs(m->n);
        fill(recs.data());
        NGPU_CUDA(cudaMemcpy(s->d_nodes, recs.data(), sizeof(recs[0]) * m->n, cudaMemcpyHostToDevice));
    }
    return NGPU_OK;
}

template <typename R>
static BatchArgs<R> make_batch_args(ngpu_batch* b) {
    BatchArgs<R> B;
    memset((void*)&B, 0, sizeof(B));
    B.n = (int)b->sims.size();
    // CTAs are dealt to the members in order of decreasing cost per CTA (the
    // tree's channel weight): the GPU starts the longest CTAs first and fills
    // in with the short ones, instead of ending on a tail of long CTAs
    std::vector<int> order(B.n);
    std::vector<int64_t> cost(B.n, 0);
    for (int k = 0; k < B.n; ++k) {
        order[k] = k;
        for (int64_t w : b->sims[k]->m->weight) cost[k] += w;
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    int c = 0;
    for (int j = 0; j < B.n; ++j) {
        const int k = order[j];
        B.sim[j] = make_args<R>(b->sims[k]);
        B.cta0[j] = c;
        c += b->sims[k]->n_groups;
    }
    B.cta0[B.n] = c;
    return B;
}

template <typename R>
static cudaError_t launch_batch(ngpu_batch* b, bool init, int t0, int n, cudaStream_t st) {
    const BatchArgs<R> B = make_batch_args<R>(b);
    cudaError_t e;
    if (b->jit) {
        if (init) {
            void* args[] = {(void*)&B};
            e = cudaLaunchKernel((const void*)b->jit->batch_init, dim3(b->total_ctas), dim3(b->threads), args, 0, st);
        } else {
            const void* k = (const void*)b->jit->batch_advance;
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
            if (e != cudaSuccess) return e;
            void* args[] = {(void*)&B, (void*)&t0, (void*)&n};
            e = cudaLaunchKernel(k, dim3(b->total_ctas), dim3(b->threads), args, b->smem, st);
        }
        g_launches++;
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    if (b->mechset == NGPU_MECHSET_TTPC) {
        if (init) {
            k_batch_init<R, 0><<<b->total_ctas, b->threads, 0, st>>>(B);
        } else {
            e = cudaFuncSetAttribute(k_batch_advance<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
            if (e != cudaSuccess) return e;
            k_batch_advance<R, 0><<<b->total_ctas, b->threads, b->smem, st>>>(B, t0, n);
        }
    } else {
        if (init) {
            k_batch_init<R, 1><<<b->total_ctas, b->threads, 0, st>>>(B);
        } else {
            e = cudaFuncSetAttribute(k_batch_advance<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
            if (e != cudaSuccess) return e;
            k_batch_advance<R, 1><<<b->total_ctas, b->threads, b->smem, st>>>(B, t0, n);
        }
    }
    g_launches++;
    return cudaGetLastError();
}

static cudaError_t launch_batch_any(ngpu_batch* b, bool init, int t0, int n, cudaStream_t st) {
    return b->precision == NGPU_FP64 ? launch_batch<double>(b, init, t0, n, st)
                                     : launch_batch<float>(b, init, t0, n, st);
}

static void batch_drop_graph(ngpu_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_key.clear();
}

// One specialised kernel over every member's masks, with the parameters all
// members share compiled in.
static int batch_select_kernels(ngpu_batch* b) {
    b->jit = nullptr;
    const GenSet* gs = gen_set(b->mechset);
    std::vector<uint32_t> all;
    int64_t pf_ctas = 0;  // the prefetch follows the members that hold most of the CTAs
    for (ngpu_sim* s : b->sims) {
        const std::vector<uint32_t> mm = model_masks(s->m);
        all.insert(all.end(), mm.begin(), mm.end());
        pf_ctas += s->ch_prefetch ? s->n_groups : -s->n_groups;
    }
    const std::vector<uint32_t> picked = ngpu_jit::pick_masks(all, kMaxClasses);
    b->jit = ngpu_jit::module(b->mechset, b->precision == NGPU_FP64, picked, gs ? &gs->source : nullptr,
                              pf_ctas >= 0, b->folds, masks_cover(picked, all, pf_ctas >= 0));
    if (gs && !b->jit)
        return fail(NGPU_E_CUDA, "mechanism set '" + gs->name +
                                     "' runs only through runtime compilation: " + ngpu_jit::last_log());
    return NGPU_OK;
}

extern "C" {

int ngpu_batch_create(ngpu_sim* const* sims, int32_t n, ngpu_batch** out) {
    if (!out) return fail(NGPU_E_INVALID, "out is null");
    *out = nullptr;
    if (!sims || n < 1 || n > kMaxBatch)
        return fail(NGPU_E_INVALID, "a batch holds 1.." + std::to_string(kMaxBatch) + " simulations");
    for (int k = 0; k < n; ++k) {
        if (!sims[k]) return fail(NGPU_E_INVALID, "null simulation in the batch");
        for (int j = 0; j < k; ++j)
            if (sims[j] == sims[k]) return fail(NGPU_E_INVALID, "a simulation appears twice in the batch");
        if (sims[k]->precision != sims[0]->precision)
            return fail(NGPU_E_INVALID, "a batch needs one precision");
        if (sims[k]->m->mechset != sims[0]->m->mechset)
            return fail(NGPU_E_INVALID, "a batch needs one mechanism set");
        if (sims[k]->batch) return fail(NGPU_E_INVALID, "a simulation belongs to one batch at a time");
        if (sims[k]->layout != NGPU_LAYOUT_LANE_INSTANCE)
            return fail(NGPU_E_INVALID, "a batch holds lane-instance simulations only");
    }
    // the batch kernel runs CTAs of up to kMaxWarps warps: a member created
    // with wider CTAs (a small batch of its own) is split again for them
    // and must be initialised again (through the batch)
    for (int k = 0; k < n; ++k) {
        ngpu_sim* s = sims[k];
        if (s->n_warps <= kMaxWarps) continue;
        const int W = std::min(kMaxWarps, std::max(1, s->m->n / 48));
        s->n_warps = W;
        s->part = make_partition(s->m, W, s->items_per_warp);
        s->s2_stage = s->precision == NGPU_FP64
                          ? choose_s2_stage<double>(s->m->n, (int)s->part.seps.size(), W, s->n_groups)
                          : choose_s2_stage<float>(s->m->n, (int)s->part.seps.size(), W, s->n_groups);
        const int rc = sim_upload_split(s);
        if (rc != NGPU_OK) return rc;
        s->initialized = false;
    }
    ngpu_batch* b = new (std::nothrow) ngpu_batch();
    if (!b) return fail(NGPU_E_NOMEM, "host allocation failed");
    b->sims.assign(sims, sims + n);
    b->precision = sims[0]->precision;
    b->mechset = sims[0]->m->mechset;
    int W = 1;
    for (ngpu_sim* s : b->sims) {
        W = std::max(W, s->n_warps);
        b->total_ctas += s->n_groups;
        const int ns = (int)s->part.seps.size();
        b->smem = std::max(b->smem, b->precision == NGPU_FP64 ? SmemPlan<double>::bytes(s->m->n, ns, s->s2_stage)
                                                             : SmemPlan<float>::bytes(s->m->n, ns, s->s2_stage));
    }
    b->threads = kLanes * W;
    b->folds = batch_common_folds(b);
    {
        const int rc = batch_select_kernels(b);
        if (rc != NGPU_OK) {
            delete b;
            return rc;
        }
    }
    for (ngpu_sim* s : b->sims) {
        s->batch = b;
        if (s->initialized) {  // its records still carry its own classes
            const int rc = sim_upload_nodes(s);
            if (rc != NGPU_OK) {
                for (ngpu_sim* t : b->sims) t->batch = nullptr;
                delete b;
                return rc;
            }
        }
    }
    *out = b;
    return NGPU_OK;
}

int ngpu_batch_destroy(ngpu_batch* b) {
    if (b) {
        batch_drop_graph(b);
        // members keep the batch's kernels until their next initialisation
        for (ngpu_sim* s : b->sims)
            if (s->batch == b) s->batch = nullptr;
    }
    delete b;
    return NGPU_OK;
}

static int batch_check_steps(ngpu_batch* b, int t0, int n) {
    for (ngpu_sim* s : b->sims) {
        if (!s->initialized) return fail(NGPU_E_STATE, "init must precede advance");
        if (t0 < 0 || n < 0 || (int64_t)t0 + n > s->nt)
            return fail(NGPU_E_INVALID, "step range outside a member's stimulus");
    }
    return NGPU_OK;
}

int ngpu_batch_init(ngpu_batch* b, float v_init, void* cuda_stream) {
    if (!b) return fail(NGPU_E_INVALID, "null batch");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    for (ngpu_sim* s : b->sims) {
        const int rc = sim_prepare_init(s, v_init, st);
        if (rc != NGPU_OK) return rc;
    }
    const cudaError_t e = launch_batch_any(b, true, 0, 0, st);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("batch init launch: ") + cudaGetErrorString(e));
    for (ngpu_sim* s : b->sims) s->initialized = true;
    return NGPU_OK;
}

int ngpu_batch_advance(ngpu_batch* b, int32_t t0, int32_t n_steps, void* cuda_stream) {
    if (!b) return fail(NGPU_E_INVALID, "null batch");
    const int rc = batch_check_steps(b, t0, n_steps);
    if (rc != NGPU_OK) return rc;
    if (n_steps == 0) return NGPU_OK;
    const cudaError_t e = launch_batch_any(b, false, t0, n_steps, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("batch advance launch: ") + cudaGetErrorString(e));
    return NGPU_OK;
}

int ngpu_batch_run_graph(ngpu_batch* b, float v_init, int32_t nt, int32_t chunk, void* cuda_stream) {
    if (!b) return fail(NGPU_E_INVALID, "null batch");
    if (nt < 1 || chunk < 1) return fail(NGPU_E_INVALID, "need nt >= 1 and chunk >= 1");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    for (ngpu_sim* s : b->sims) {
        const int rc = sim_prepare_init(s, v_init, st);
        if (rc != NGPU_OK) return rc;
        if (nt > s->nt) return fail(NGPU_E_INVALID, "nt beyond a member's stimulus");
    }
    // the graph bakes in every launch argument: reuse it only for the same ones
    std::vector<unsigned char> key;
    auto add = [&](const void* p, size_t bytes) {
        const unsigned char* c = (const unsigned char*)p;
        key.insert(key.end(), c, c + bytes);
    };
    if (b->precision == NGPU_FP64) {
        const BatchArgs<double> B = make_batch_args<double>(b);
        add(&B, sizeof(B));
    } else {
        const BatchArgs<float> B = make_batch_args<float>(b);
        add(&B, sizeof(B));
    }
    add(&nt, sizeof(nt));
    add(&chunk, sizeof(chunk));
    add(&st, sizeof(st));
    if (!b->exec || key != b->graph_key) {
        batch_drop_graph(b);
        // set the shared-memory attribute outside the capture
        cudaError_t e = cudaSuccess;
        if (b->jit)
            e = cudaFuncSetAttribute((const void*)b->jit->batch_advance, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)b->smem);
        else if (b->precision == NGPU_FP64)
            e = b->mechset == NGPU_MECHSET_TTPC
                    ? cudaFuncSetAttribute(k_batch_advance<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem)
                    : cudaFuncSetAttribute(k_batch_advance<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
        else
            e = b->mechset == NGPU_MECHSET_TTPC
                    ? cudaFuncSetAttribute(k_batch_advance<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem)
                    : cudaFuncSetAttribute(k_batch_advance<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
        if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("batch attribute: ") + cudaGetErrorString(e));
        if (!st) return fail(NGPU_E_INVALID, "graph capture needs a non-default stream");
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
        const auto before = g_launches.load();
        cudaError_t le = launch_batch_any(b, true, 0, 0, st);
        for (int t0 = 0; le == cudaSuccess && t0 < nt; t0 += chunk)
            le = launch_batch_any(b, false, t0, std::min(chunk, nt - t0), st);
        b->graph_kernels = (int)(g_launches.load() - before);
        g_launches -= b->graph_kernels;  // captured, not run
        e = cudaStreamEndCapture(st, &b->graph);
        if (le != cudaSuccess || e != cudaSuccess) {
            batch_drop_graph(b);
            return fail(NGPU_E_CUDA, std::string("graph capture: ") +
                                         cudaGetErrorString(le != cudaSuccess ? le : e));
        }
        e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) {
            batch_drop_graph(b);
            return fail(NGPU_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        b->graph_key = key;
    }
    const cudaError_t e = cudaGraphLaunch(b->exec, st);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    g_launches += b->graph_kernels;
    for (ngpu_sim* s : b->sims) s->initialized = true;
    return NGPU_OK;
}

int ngpu_sim_n_samples(const ngpu_sim* s) { return s ? s->n_samples : 0; }

// Window bounds as features.py computes them (Python's round: half to even).
static int feature_args(int32_t n_samples, double dt, double stim_on, double stim_off, FeatureArgs* a) {
    if (n_samples < 2 || !(dt > 0) || !std::isfinite(dt) || !std::isfinite(stim_on) || !std::isfinite(stim_off))
        return fail(NGPU_E_INVALID, "features: need >= 2 samples, dt > 0 and finite window bounds");
    const int T = n_samples;
    auto rnd = [](double x) { return (int)std::nearbyint(x); };
    a->i_on = std::max(0, rnd(stim_on / dt));
    a->i_off = std::min(T, rnd(stim_off / dt));
    if (a->i_off - a->i_on < 2) return fail(NGPU_E_INVALID, "features: the stimulus window holds < 2 samples");
    a->dur = (float)((a->i_off - a->i_on) * dt);
    auto win = [&](double lo, double hi, int* ia, int* ib) {
        const int r = rnd(lo / dt);
        *ia = std::max(0, r);
        *ib = std::min(T, std::max(r + 1, rnd(hi / dt)));
    };
    win(std::max(0.0, stim_on - 10.0), stim_on, &a->vb_lo, &a->vb_hi);
    win(std::max(stim_on, stim_off - 50.0), stim_off, &a->ss_lo, &a->ss_hi);
    if (stim_off + 10.0 < T * dt) win(stim_off + 10.0, T * dt, &a->af_lo, &a->af_hi);
    else a->af_lo = a->af_hi = -1;
    a->dt = (float)dt;
    a->n_samples = T;
    return NGPU_OK;
}

static int launch_features(FeatureArgs a, cudaStream_t st) {
    if (a.n_traces < 1) return NGPU_OK;
    k_trace_features<<<(a.n_traces + 127) / 128, 128, 0, st>>>(a);
    g_launches++;
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}

int ngpu_trace_features(const float* v_dev, int64_t stride_trace, int64_t stride_sample, int32_t n_traces,
                        int32_t n_samples, double dt, double stim_on, double stim_off, float threshold, float* out_dev,
                        void* cuda_stream) {
    if (!v_dev || !out_dev) return fail(NGPU_E_INVALID, "features: null pointer");
    if (n_traces < 0 || stride_trace < 0 || stride_sample < 1) return fail(NGPU_E_INVALID, "features: bad strides");
    FeatureArgs a;
    const int rc = feature_args(n_samples, dt, stim_on, stim_off, &a);
    if (rc != NGPU_OK) return rc;
    a.v = v_dev;
    a.stride_trace = stride_trace;
    a.stride_sample = stride_sample;
    a.n_traces = n_traces;
    a.threshold = threshold;
    a.out = out_dev;
    return launch_features(a, (cudaStream_t)cuda_stream);
}

int ngpu_sim_features(ngpu_sim* s, int32_t site, double dt, double stim_on, double stim_off, float threshold,
                      float* out_dev, void* cuda_stream) {
    if (!s || !out_dev) return fail(NGPU_E_INVALID, "null argument");
    if (!s->initialized || !s->d_trace) return fail(NGPU_E_STATE, "run the simulation first");
    if (site < 0 || site >= (int)s->rec_cols.size()) return fail(NGPU_E_INVALID, "recording site out of range");
    FeatureArgs a;
    const int rc = feature_args(s->n_samples, dt, stim_on, stim_off, &a);
    if (rc != NGPU_OK) return rc;
    a.v = s->d_trace + (size_t)s->rec_cols[site] * s->n_pad;   // [sample][column][instance]
    a.stride_trace = 1;
    a.stride_sample = (int64_t)s->n_rec_unique * s->n_pad;
    a.n_traces = s->n_inst;
    a.threshold = threshold;
    a.out = out_dev;
    return launch_features(a, (cudaStream_t)cuda_stream);
}

// ------------------------------------------------------------------ exploration score

int64_t ngpu_dvdt_peaks_scratch_bytes(int32_t n_traces, int32_t n_samples) {
    if (n_traces < 0 || n_samples < 0) return 0;
    return (int64_t)peak_scratch_cap(n_samples) * n_traces * (int64_t)sizeof(int32_t);
}

static int launch_dvdt_peaks(PeakArgs a, int64_t scratch_bytes, cudaStream_t st) {
    if (!(a.dt > 0) || !std::isfinite(a.dt) || std::isnan(a.height))
        return fail(NGPU_E_INVALID, "dvdt peaks: need dt > 0 (finite) and a height that is not NaN");
    if (a.distance < 1) return fail(NGPU_E_INVALID, "dvdt peaks: distance must be >= 1 sample");
    if (a.n_samples < 0 || a.n_samples >= (1 << 29) || a.n_traces < 0)
        return fail(NGPU_E_INVALID, "dvdt peaks: sample count out of range (< 2^29)");
    if (a.n_traces == 0) return NGPU_OK;
    a.cap = peak_scratch_cap(a.n_samples);
    const int64_t need = ngpu_dvdt_peaks_scratch_bytes(a.n_traces, a.n_samples);
    if (scratch_bytes < need)
        return fail(NGPU_E_INVALID, "dvdt peaks: scratch holds " + std::to_string(scratch_bytes) + " bytes, needs " +
                                        std::to_string(need));
    if (!a.v || !a.out || !a.pos) return fail(NGPU_E_INVALID, "dvdt peaks: null pointer");
    // 64 threads a CTA: the traces of an exploration (10,000) spread over every SM
    k_dvdt_peaks<<<(a.n_traces + 63) / 64, 64, 0, st>>>(a);
    g_launches++;
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}

int ngpu_trace_dvdt_peaks(const float* v_dev, int64_t stride_trace, int64_t stride_sample, int32_t n_traces,
                          int32_t n_samples, double dt, double height, int32_t distance, void* scratch_dev,
                          int64_t scratch_bytes, int32_t* out_dev, void* cuda_stream) {
    if (stride_trace < 0 || stride_sample < 1) return fail(NGPU_E_INVALID, "dvdt peaks: bad strides");
    PeakArgs a;
    a.v = v_dev;
    a.stride_trace = stride_trace;
    a.stride_sample = stride_sample;
    a.n_traces = n_traces;
    a.n_samples = n_samples;
    a.dt = dt;
    a.height = height;
    a.distance = distance;
    a.pos = (int32_t*)scratch_dev;
    a.out = out_dev;
    return launch_dvdt_peaks(a, scratch_bytes, (cudaStream_t)cuda_stream);
}

int ngpu_sim_dvdt_peaks(ngpu_sim* s, int32_t site, double dt, double height, int32_t distance, void* scratch_dev,
                        int64_t scratch_bytes, int32_t* out_dev, void* cuda_stream) {
    if (!s) return fail(NGPU_E_INVALID, "null simulation");
    if (!s->initialized || !s->d_trace) return fail(NGPU_E_STATE, "run the simulation first");
    if (site < 0 || site >= (int)s->rec_cols.size()) return fail(NGPU_E_INVALID, "recording site out of range");
    PeakArgs a;
    a.v = s->d_trace + (size_t)s->rec_cols[site] * s->n_pad;  // [sample][column][instance]
    a.stride_trace = 1;
    a.stride_sample = (int64_t)s->n_rec_unique * s->n_pad;
    a.n_traces = s->n_inst;
    a.n_samples = s->n_samples;
    a.dt = dt;
    a.height = height;
    a.distance = distance;
    a.pos = (int32_t*)scratch_dev;
    a.out = out_dev;
    return launch_dvdt_peaks(a, scratch_bytes, (cudaStream_t)cuda_stream);
}

int ngpu_sim_param_rows(const ngpu_sim* s, int32_t* rows_read, int32_t* rows_total) {
    if (!s || !rows_read || !rows_total) return fail(NGPU_E_INVALID, "null argument");
    const ngpu_model* m = s->m;
    std::map<int, int> used;   // block start the nodes read -> its rows
    for (int i = 0; i < m->n; ++i)
        if (m->rows[i].y > 0)
            used[s->prow_canon.empty() ? m->info[i].prow : s->prow_canon[m->info[i].prow]] = m->rows[i].y;
    int n = 0;
    for (const auto& u : used) n += u.second;
    *rows_read = n;
    *rows_total = m->ptab_rows;
    return NGPU_OK;
}

int ngpu_sim_param_folds(const ngpu_sim* s, int32_t* n_folds) {
    if (!s || !n_folds) return fail(NGPU_E_INVALID, "null argument");
    *n_folds = s->batch ? (int32_t)s->batch->folds.size() : (s->jit ? (int32_t)s->folds.size() : 0);
    return NGPU_OK;
}

int ngpu_sim_classes(const ngpu_sim* s, int32_t* n_classes) {
    if (!s || !n_classes) return fail(NGPU_E_INVALID, "null argument");
    *n_classes = s->jit ? (int32_t)s->jit->masks.size() : 0;
    return NGPU_OK;
}

int ngpu_jit_build(int32_t mechset, int32_t precision, const uint32_t* masks, int32_t n_masks, int32_t cc_major,
                   int32_t cc_minor, int64_t* cubin_bytes) {
    if (!cubin_bytes || (n_masks > 0 && !masks)) return fail(NGPU_E_INVALID, "null argument");
    if (!mechset_known(mechset)) return fail(NGPU_E_INVALID, "unknown mechset");
    if (precision != NGPU_FP32 && precision != NGPU_FP64) return fail(NGPU_E_INVALID, "precision must be FP32 or FP64");
    const GenSet* gs = gen_set(mechset);
    if (n_masks < (gs ? 0 : 1) || n_masks > kMaxClasses)
        return fail(NGPU_E_INVALID, "1.." + std::to_string(kMaxClasses) + " masks");
    std::vector<char> cubin;
    std::string err;
    const std::vector<uint32_t> mv(masks, masks + n_masks);
    std::lock_guard<std::mutex> lock(ngpu_jit::mu());
    if (!ngpu_jit::build_cubin(gs ? 2 : mechset, precision == NGPU_FP64, mv, gs ? &gs->source : nullptr,
                               std::to_string(cc_major) + std::to_string(cc_minor) + "a", &cubin, &err)) {
        ngpu_jit::last_log() = err;
        return fail(NGPU_E_CUDA, "runtime compilation failed: " + err);
    }
    *cubin_bytes = (int64_t)cubin.size();
    return NGPU_OK;
}

const char* ngpu_jit_log(void) {
    static thread_local std::string copy;
    std::lock_guard<std::mutex> lock(ngpu_jit::mu());
    copy = ngpu_jit::last_log();
    return copy.c_str();
}

int ngpu_sim_trace_device(ngpu_sim* s, const float** trace, int32_t* n_inst_padded) {
    if (!s || !trace) return fail(NGPU_E_INVALID, "null argument");
    *trace = s->d_trace;
    if (n_inst_padded) *n_inst_padded = s->n_pad;
    return NGPU_OK;
}

int ngpu_sim_get_trace(ngpu_sim* s, float* out, int32_t on_device, void* cuda_stream) {
    if (!s || !out) return fail(NGPU_E_INVALID, "null sim or out");
    if (!s->initialized) return fail(NGPU_E_STATE, "no run to read");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const int nr = s->n_rec_unique, ns = s->n_samples;
    const size_t per_inst_u = (size_t)nr * ns;
    const size_t bytes_u = sizeof(float) * per_inst_u * s->n_inst;
    if (s->tmp_out_bytes < bytes_u) {
        if (s->d_tmp_out) cudaFree(s->d_tmp_out);
        s->d_tmp_out = nullptr;
        s->tmp_out_bytes = 0;
        int rc = NGPU_OK;
        s->d_tmp_out = (float*)dmalloc(bytes_u, &rc);
        if (!s->d_tmp_out) return rc;
        s->tmp_out_bytes = bytes_u;
    }
    dim3 grid((s->n_pad + 31) / 32, (ns + 31) / 32, nr), block(32, 8);
    k_trace_transpose<<<grid, block, 0, st>>>(s->d_trace, ns, nr, s->n_pad, s->n_inst, s->d_tmp_out);
    g_launches++;
    NGPU_CUDA(cudaGetLastError());
    const int n_rec = (int)s->rec_nodes.size();
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    bool identity = (n_rec == nr);
    for (int r = 0; r < n_rec && identity; ++r) identity = s->rec_cols[r] == r;
    // a host destination is written through the pinned staging buffer
    const size_t bytes_out = sizeof(float) * (size_t)n_rec * ns * s->n_inst;
    float* stg = on_device ? nullptr : (float*)sim_stage(s, bytes_out);
    float* dst = stg ? stg : out;
    if (identity) {
        NGPU_CUDA(cudaMemcpyAsync(dst, s->d_tmp_out, bytes_u, kind, st));
    } else {
        // duplicated sites: strided copies of each requested column
        for (int r = 0; r < n_rec; ++r) {
            NGPU_CUDA(cudaMemcpy2DAsync(dst + (size_t)r * ns, sizeof(float) * n_rec * ns,
                                        s->d_tmp_out + (size_t)s->rec_cols[r] * ns, sizeof(float) * per_inst_u,
                                        sizeof(float) * ns, s->n_inst, kind, st));
        }
    }
    NGPU_CUDA(cudaStreamSynchronize(st));
    if (stg) host_copy_parallel(out, stg, bytes_out);
    return NGPU_OK;
}

int ngpu_sim_check(ngpu_sim* s, int32_t* n_bad, void* cuda_stream) {
    if (!s || !n_bad) return fail(NGPU_E_INVALID, "null argument");
    std::vector<int> bad(s->n_pad);
    NGPU_CUDA(cudaMemcpyAsync(bad.data(), s->d_bad, sizeof(int) * s->n_pad, cudaMemcpyDeviceToHost,
                              (cudaStream_t)cuda_stream));
    NGPU_CUDA(cudaStreamSynchronize((cudaStream_t)cuda_stream));
    int c = 0;
    for (int i = 0; i < s->n_inst; ++i) c += bad[i] != 0;
    *n_bad = c;
    return NGPU_OK;
}

int ngpu_run(ngpu_model* m, int32_t n_sets, const float* params, int32_t n_stim, int32_t nt,
             const float* amps, const float* dts, int32_t stim_node, float stim_area_um2,
             int32_t n_rec, const int32_t* rec_nodes, float v_init, int32_t precision, float* out) {
    if (!out) return fail(NGPU_E_INVALID, "out is null");
    if (!m) return fail(NGPU_E_INVALID, "null model");
    // The last run's simulation stays with the model and serves the next call
    // of the same shape (sets, stimuli, precision): no device allocation or
    // release per call.  A call that finds it in use by another thread runs
    // on a simulation of its own.
    std::unique_lock<std::mutex> lock(m->run_mu, std::try_to_lock);
    ngpu_sim* s = nullptr;
    int rc = NGPU_OK;
    ngpu_sim* c = lock.owns_lock() ? m->run_cache : nullptr;
    if (c && c->n_sets == n_sets && c->n_stim == n_stim && c->precision == precision) {
        s = c;
    } else {
        if (c) {
            sim_free(c);
            m->run_cache = nullptr;
        }
        rc = ngpu_sim_create(m, n_sets, n_stim, precision, &s);
        if (rc) return rc;
    }
    if (lock.owns_lock()) m->run_cache = nullptr;  // taken; kept again below on success
    // one pinned staging buffer for both host copies (parameters in, trace out;
    // pinning takes ~3 ms per MB, so it is sized once for the larger)
    sim_stage(s, std::max(sizeof(float) * (size_t)n_sets * m->n_params * m->n_sections,
                          sizeof(float) * (size_t)n_sets * n_stim * std::max(0, n_rec) * std::max(0, nt)));
    if ((rc = ngpu_sim_set_params(s, params, 0)) ||
        (rc = ngpu_sim_set_stimulus(s, nt, amps, dts, stim_node, stim_area_um2, 0)) ||
        (rc = ngpu_sim_set_recording(s, n_rec, rec_nodes, 1)) || (rc = ngpu_sim_init(s, v_init, nullptr)) ||
        (rc = ngpu_sim_advance(s, 0, nt, nullptr)) || (rc = ngpu_sim_get_trace(s, out, 0, nullptr))) {
        std::string msg = g_err;
        sim_free(s);
        g_err = msg;
        return rc;
    }
    int32_t nbad = 0;
    rc = ngpu_sim_check(s, &nbad, nullptr);
    if (rc == NGPU_OK && lock.owns_lock()) m->run_cache = s;
    else sim_free(s);
    if (rc) return rc;
    if (nbad) return fail(NGPU_E_NUMERIC, std::to_string(nbad) + " instance(s) produced non-finite voltage");
    return NGPU_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free entry point (ngpu_run_static).
//
// Some callers are not allowed to allocate device memory at all: an
// application that hands this library a region of its own pre-allocated
// device arena and runs under a fixed device-memory budget, or a host loop
// with latency limits that cannot afford cudaMalloc / cudaFree (both can
// synchronise the whole device and take unbounded time).  For them every
// buffer of one simulation run -- node records, channel states, parameters
// table, solver scratch, trace -- is carved out of the single file-scope
// array below instead of being allocated.  Inputs and outputs stay in the
// caller's own device memory.
//
// The array is a host-side stand-in in host code: its device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on the device.  Every call shares the
// array and leaves its contents behind; each call re-initialises what it
// relies on.  Two calls whose work overlaps on the GPU (different streams,
// or another thread) race on the array and must be serialised by the caller.
// ===========================================================================
namespace {
constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // held by every GPU that loads the library
constexpr int kStaticMaxNodes = 512;
constexpr int kStaticMaxInstances = 256;
constexpr int kStaticMaxRec = 16;
}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device, looked up on
// every call (it allocates nothing, and a device reset that reloads the
// module moves the array).  In host code the array's name is only a stand-in.
static int static_scratch_address(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
        return fail(NGPU_E_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    *out = (unsigned char*)p;
    return NGPU_OK;
}

extern "C" int ngpu_run_static(ngpu_model* m, int32_t n_sets, const float* params_dev, int32_t n_stim,
                               int32_t nt, const float* amps_dev, const float* dts_dev, int32_t stim_node,
                               float stim_area_um2, int32_t n_rec, const int32_t* rec_nodes, float v_init,
                               float* out_dev, void* cuda_stream) {
    if (!m || !params_dev || !amps_dev || !dts_dev || !rec_nodes || !out_dev)
        return fail(NGPU_E_INVALID, "ngpu_run_static: null argument");
    if (m->mechset >= NGPU_MECHSET_GENERATED)
        return fail(NGPU_E_INVALID, "ngpu_run_static: a mechanism set generated from NMODL files runs only "
                                    "through runtime compilation (ngpu_run / ngpu_sim_*)");
    const int N = m->n;
    if (N > kStaticMaxNodes)
        return fail(NGPU_E_INVALID, "ngpu_run_static: at most " + std::to_string(kStaticMaxNodes) +
                                        " nodes (model has " + std::to_string(N) + ")");
    if (n_sets < 1 || n_stim < 1 || (int64_t)n_sets * n_stim > kStaticMaxInstances)
        return fail(NGPU_E_INVALID, "ngpu_run_static: 1 to " + std::to_string(kStaticMaxInstances) +
                                        " instances (sets x stimuli)");
    if (nt < 1) return fail(NGPU_E_INVALID, "ngpu_run_static: nt must be >= 1");
    if (n_rec < 1 || n_rec > kStaticMaxRec)
        return fail(NGPU_E_INVALID, "ngpu_run_static: 1 to " + std::to_string(kStaticMaxRec) + " recording sites");
    if (stim_node < 0 || stim_node >= m->n_caller)
        return fail(NGPU_E_INVALID, "ngpu_run_static: stim_node out of range");
    if (!(stim_area_um2 > 0.f) || !std::isfinite(stim_area_um2))
        return fail(NGPU_E_INVALID, "ngpu_run_static: stimulus area must be positive");
    if (!std::isfinite(v_init)) return fail(NGPU_E_INVALID, "ngpu_run_static: v_init must be finite");
    for (int r = 0; r < n_rec; ++r)
        if (rec_nodes[r] < 0 || rec_nodes[r] >= m->n_caller)
            return fail(NGPU_E_INVALID, "ngpu_run_static: recording node out of range");

    // ---- host bookkeeping in fixed-size local arrays (one warp per group:
    // the root is the only separator, its child subtrees the work items)
    const int n_inst = n_sets * n_stim;
    const int n_groups = (n_inst + kLanes - 1) / kLanes;
    const int n_pad = n_groups * kLanes;
    NodeRec<float> recs[kStaticMaxNodes];  // ~38 KB of stack in all
    DevComp comps[kStaticMaxNodes];
    int subn[kStaticMaxNodes], jslot[kStaticMaxNodes], pslot[kStaticMaxNodes];
    int inst_stim[kStaticMaxInstances + kLanes];
    int rec_col_of_node[kStaticMaxRec], rec_cols[kStaticMaxRec], n_rec_u = 0;
    for (int r = 0; r < n_rec; ++r) {
        const int node = m->node_internal[rec_nodes[r]];
        int c = -1;
        for (int k = 0; k < n_rec_u; ++k)
            if (rec_col_of_node[k] == node) c = k;
        if (c < 0) {
            c = n_rec_u;
            rec_col_of_node[n_rec_u++] = node;
        }
        rec_cols[r] = c;
    }
    for (int i = 0; i < N; ++i) subn[i] = 1;
    for (int i = N - 1; i > 0; --i) subn[m->parent[i]] += subn[i];
    int n_comps = 0;
    for (int i = 1; i < N; ++i)
        if (m->parent[i] == 0) comps[n_comps++] = {i, 0, -1, -1, i, i + subn[i]};
    int nj = 0;
    for (int i = 0; i < N; ++i) jslot[i] = -1;
    jslot[0] = nj++;
    for (int i = 1; i < N; ++i) {
        const int p = m->parent[i];
        if ((p != i - 1 || p == 0) && jslot[p] < 0) jslot[p] = nj++;
    }
    for (int i = 0; i < N; ++i) {
        const int p = i > 0 ? m->parent[i] : -1;
        pslot[i] = (i > 0 && (p != i - 1 || p == 0)) ? jslot[p] : -1;
    }
    for (int i = 0; i < N; ++i) {
        NodeRec<float>& q = recs[i];
        q.a = (float)m->a[i];
        q.b = (float)m->b[i];
        q.cm = (float)(m->cm[i] / 1000.0);
        q.srow = m->info[i].srow;
        q.parent = (int16_t)m->parent[i];
        q.jslot = (int16_t)jslot[i];
        q.pslot = (int16_t)pslot[i];
        q.rec = -1;
        q.mask = (uint16_t)m->mask[i];
        q.prow = (uint16_t)m->info[i].prow;
        q.srows = (uint8_t)m->rows[i].x;
        q.prows = (uint8_t)m->rows[i].y;
        q.cls = (uint8_t)kGenericClass;
        q.pad_ = 0;
    }
    for (int k = 0; k < n_rec_u; ++k) recs[rec_col_of_node[k]].rec = (int16_t)k;
    for (int k = 0; k < n_pad; ++k) inst_stim[k] = std::min(k, n_inst - 1) % n_stim;
    const DevSep root_sep = {0, -1, -1, 0};

    // ---- carve the static array
    const size_t G = (size_t)n_groups, L = kLanes;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~size_t(255);
        return at;
    };
    const size_t o_recs = take(sizeof(NodeRec<float>) * N);
    const size_t o_comps = take(sizeof(DevComp) * std::max(1, n_comps));
    const size_t o_seps = take(sizeof(DevSep));
    const size_t o_istim = take(sizeof(int) * n_pad);
    const size_t o_bad = take(sizeof(int) * n_pad);
    const size_t o_rowp = take(sizeof(int) * m->row_param.size());
    const size_t o_rows = take(sizeof(int) * m->row_sec.size());
    const size_t o_vbuf = take(G * N * 2 * L * sizeof(float));
    const size_t o_slab = take(G * m->slab_rows * L * sizeof(float));
    const size_t o_ptab = take(G * m->ptab_rows * L * sizeof(float));
    const size_t o_scr = take(G * N * 3 * L * sizeof(float));
    const size_t o_jacc = take(G * 2 * nj * L * sizeof(double));
    const size_t o_jx = take(G * nj * L * sizeof(float));
    const size_t o_sepv = take(G * 4 * L * sizeof(float));
    const size_t o_trace = take((size_t)nt * n_rec_u * n_pad * sizeof(float));
    if (off > kStaticScratchBytes)
        return fail(NGPU_E_INVALID, "ngpu_run_static: this run needs " + std::to_string(off) +
                                        " bytes of device scratch; the static array holds " +
                                        std::to_string(kStaticScratchBytes));
    unsigned char* base = nullptr;
    int rc = static_scratch_address(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    NGPU_CUDA(cudaMemcpyAsync(base + o_recs, recs, sizeof(NodeRec<float>) * N, cudaMemcpyHostToDevice, st));
    if (n_comps)
        NGPU_CUDA(cudaMemcpyAsync(base + o_comps, comps, sizeof(DevComp) * n_comps, cudaMemcpyHostToDevice, st));
    NGPU_CUDA(cudaMemcpyAsync(base + o_seps, &root_sep, sizeof(DevSep), cudaMemcpyHostToDevice, st));
    NGPU_CUDA(cudaMemcpyAsync(base + o_istim, inst_stim, sizeof(int) * n_pad, cudaMemcpyHostToDevice, st));
    NGPU_CUDA(cudaMemcpyAsync(base + o_rowp, m->row_param.data(), sizeof(int) * m->row_param.size(),
                              cudaMemcpyHostToDevice, st));
    NGPU_CUDA(cudaMemcpyAsync(base + o_rows, m->row_sec.data(), sizeof(int) * m->row_sec.size(),
                              cudaMemcpyHostToDevice, st));
    // the copies above read host stack memory: make sure they are done before returning
    NGPU_CUDA(cudaStreamSynchronize(st));

    SimArgs<float> A;
    A.nodes = (const NodeRec<float>*)(base + o_recs);
    A.n_nodes = N;
    A.vbuf = (float*)(base + o_vbuf);
    A.slab = (float*)(base + o_slab);
    A.slab_rows = m->slab_rows;
    A.ptab = (const float*)(base + o_ptab);
    A.ptab_rows = m->ptab_rows;
    A.scr = (float*)(base + o_scr);
    A.jacc = (double*)(base + o_jacc);
    A.jx = (float*)(base + o_jx);
    A.n_jslots = nj;
    A.amps = amps_dev;
    A.dts = dts_dev;
    A.nt = nt;
    A.stim_node = m->node_internal[stim_node];
    A.stim_scale = 100.0 / (double)stim_area_um2 * m->density_scale[stim_node];
    A.inst_stim = (const int*)(base + o_istim);
    A.trace = (float*)(base + o_trace);
    A.n_rec = n_rec_u;
    A.rec_every = 1;
    A.n_inst_pad = n_pad;
    A.n_inst = n_inst;
    A.v_init = v_init;
    A.bad = (int*)(base + o_bad);
    A.n_warps = 1;
    A.comps = (const DevComp*)(base + o_comps);
    A.n_comps = n_comps;
    A.seps = (const DevSep*)(base + o_seps);
    A.n_seps = 1;
    A.sepv = (float*)(base + o_sepv);
    A.s2_stage = 0;

    const size_t total = G * m->ptab_rows * L;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    k_gather_params<<<blocks, 256, 0, st>>>(params_dev, (const int*)(base + o_rowp), (const int*)(base + o_rows),
                                              m->ptab_rows, m->n_params, m->n_sections, n_stim, n_inst, n_groups,
                                              (float*)(base + o_ptab));
    const size_t smem = SmemPlan<float>::bytes(N);
    if (m->mechset == NGPU_MECHSET_TTPC) {
        k_sim_init<float, 0><<<n_groups, kLanes, 0, st>>>(A);
        k_sim_advance<float, 0><<<n_groups, kLanes, smem, st>>>(A, 0, nt);
    } else {
        k_sim_init<float, 1><<<n_groups, kLanes, 0, st>>>(A);
        k_sim_advance<float, 1><<<n_groups, kLanes, smem, st>>>(A, 0, nt);
    }
    g_launches += 3;
    NGPU_CUDA(cudaGetLastError());
    // trace [sample][site][instance] -> out [instance][requested site][sample]
    for (int r = 0; r < n_rec; ++r) {
        dim3 grid((n_pad + 31) / 32, (nt + 31) / 32, 1), block(32, 8);
        k_trace_transpose_site<<<grid, block, 0, st>>>(A.trace, nt, n_rec_u, rec_cols[r], n_pad, n_inst, n_rec, r,
                                                       out_dev);
        g_launches++;
    }
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}

// ---- BF16 tensor-core GEMM (surrogate network) -------------------------------
static __device__ int g_gemm_err;

// The split of K over CTAs: the whole of K per CTA, except for the split-K
// epilogue, which spreads K over up to `slots` CTAs (the resident CTAs of
// one wave: two per SM for the cp.async kernel, one for the TMA kernel),
// each slice at least one 64-wide tile.
static int gemm_k_split(const GemmArgs& g, int bn, int epi, int slots, int* splits) {
    const int KT = g.K / kGemmBK;
    const int tiles = ((g.M + kGemmBM - 1) / kGemmBM) * ((g.N + bn - 1) / bn);
    int z = 1;
    if (epi == kEpiSplitAdd) z = std::max(1, std::min(KT, slots / tiles));
    const int per = (KT + z - 1) / z;
    *splits = (KT + per - 1) / per;
    return per;
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), looked up once
// through the runtime; nullptr where the driver does not offer it.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    return fn;
}

// Tensor map of a bf16 operand [rows][ld] read in boxes of 64 (K) x box_rows,
// 128-byte swizzle, zero fill past the edges.
static bool gemm_tensor_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int K, int ld, int box_rows) {
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(__nv_bfloat16)};
    const cuuint32_t box[2] = {(cuuint32_t)kGemmBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA kernel runs where the tensor maps can be built and every tile box
// fits its operand (M >= 128 rows, N >= BN); NGPU_GEMM_TMA=0 selects the
// cp.async kernel everywhere.
static bool gemm_use_tma(const GemmArgs& g, int bn) {
    const char* ev = getenv("NGPU_GEMM_TMA");
    if (ev && ev[0] == '0') return false;
    return g.M >= kGemmBM && g.N >= bn && tensor_map_encoder() != nullptr;
}

// More than two work units (tiles x K slices) per SM: the persistent
// kernel, one CTA per SM, unless NGPU_GEMM_PERSISTENT=0.  Measured on B200:
// 8192^3 0.809 ms against 0.889 one CTA per tile, 4096^3 0.115 against
// 0.123; at 1.7 tiles per SM (8192 x 512 x 512, 128-wide tiles) the overlap
// gains less than the one-CTA-per-tile kernel's 16-warp epilogue (0.029
// against 0.024 ms).
static bool gemm_use_persistent(int units) {
    const char* ev = getenv("NGPU_GEMM_PERSISTENT");
    if (ev && ev[0] == '0') return false;
    return units > 2 * kSmCount;
}

template <int BN, int EPI>
static cudaError_t launch_gemm_bn(GemmArgs g, cudaStream_t st) {
    if (gemm_use_tma(g, BN)) {
        CUtensorMap ta, tb;
        if (gemm_tensor_map(&ta, g.A, g.M, g.K, g.lda, kGemmBM) && gemm_tensor_map(&tb, g.B, g.N, g.K, g.ldb, BN)) {
            const int n_mt = (g.M + kGemmBM - 1) / kGemmBM, n_nt = (g.N + BN - 1) / BN;
            int splits = 1;
            const int per = gemm_k_split(g, BN, EPI, kSmCount, &splits);
            if (gemm_use_persistent(n_mt * n_nt * splits)) {
                const size_t smem = gemm_persist_smem_bytes<BN>();
                cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16_tma_persistent<BN, EPI>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess) return e;
                g.kt_split = per;
                if (EPI == kEpiSplitAdd) {
                    e = cudaMemsetAsync(g.out_f32, 0, sizeof(float) * ((size_t)(g.M - 1) * g.ldo + g.N), st);
                    if (e != cudaSuccess) return e;
                }
                const int units = n_mt * n_nt * splits;
                k_gemm_bf16_tma_persistent<BN, EPI><<<std::min(units, kSmCount), kPersistThreads, smem, st>>>(
                    ta, tb, g, units, n_mt, n_nt);
                g_launches++;
                return cudaGetLastError();
            }
            const size_t smem = gemm_tma_smem_bytes<BN>();
            cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16_tma<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
            g.kt_split = per;  // split-K: one CTA per SM, one wave
            if (EPI == kEpiSplitAdd) {
                e = cudaMemsetAsync(g.out_f32, 0, sizeof(float) * ((size_t)(g.M - 1) * g.ldo + g.N), st);
                if (e != cudaSuccess) return e;
            }
            dim3 grid(n_mt, n_nt, splits);
            k_gemm_bf16_tma<BN, EPI><<<grid, kTmaThreads, smem, st>>>(ta, tb, g);
            g_launches++;
            return cudaGetLastError();
        }
    }
    const size_t smem = gemm_smem_bytes<BN>();
    cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16_tn<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int splits = 1;
    g.kt_split = gemm_k_split(g, BN, EPI, 2 * kSmCount, &splits);
    if (EPI == kEpiSplitAdd) {  // the slices add into a zeroed output
        e = cudaMemsetAsync(g.out_f32, 0, sizeof(float) * ((size_t)(g.M - 1) * g.ldo + g.N), st);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((g.M + kGemmBM - 1) / kGemmBM, (g.N + BN - 1) / BN, splits);
    k_gemm_bf16_tn<BN, EPI><<<grid, kGemmThreads, smem, st>>>(g);
    g_launches++;
    return cudaGetLastError();
}

template <int EPI>
static cudaError_t launch_gemm_epi(GemmArgs g, int bn, cudaStream_t st) {
    switch (bn) {
        case 32: return launch_gemm_bn<32, EPI>(g, st);
        case 64: return launch_gemm_bn<64, EPI>(g, st);
        case 128: return launch_gemm_bn<128, EPI>(g, st);
        default: return launch_gemm_bn<256, EPI>(g, st);
    }
}

extern "C" int ngpu_gemm_bf16_tn(const void* A, const void* B, int32_t M, int32_t N, int32_t K, int32_t lda,
                                 int32_t ldb, int32_t epilogue, int32_t bn, float* out_f32, void* out_bf16,
                                 void* out_bf16_t, int32_t ldo, int32_t ldt, const float* bias, const float* zin,
                                 void* cuda_stream) {
    if (!A || !B) return fail(NGPU_E_INVALID, "gemm: null operand");
    if (M < 1 || N < 1 || K < kGemmBK || K % kGemmBK)
        return fail(NGPU_E_INVALID, "gemm: need M, N >= 1 and K a positive multiple of 64");
    if (lda < K || ldb < K || lda % 8 || ldb % 8)
        return fail(NGPU_E_INVALID, "gemm: leading dimensions must be >= K and multiples of 8");
    if (((uintptr_t)A | (uintptr_t)B) & 15) return fail(NGPU_E_INVALID, "gemm: operands must be 16-byte aligned");
    if (bn != 32 && bn != 64 && bn != 128 && bn != 256) return fail(NGPU_E_INVALID, "gemm: bn must be 32, 64, 128 or 256");
    const bool need_f32 = epilogue == kEpiStore || epilogue == kEpiBias || epilogue == kEpiBiasGelu ||
                          epilogue == kEpiSplitAdd;
    const bool need_bf16 = epilogue == kEpiBiasGelu || epilogue == kEpiGeluGrad;
    if ((need_f32 && !out_f32) || (need_bf16 && (!out_bf16 || !out_bf16_t)) ||
        ((epilogue == kEpiBias || epilogue == kEpiBiasGelu) && !bias) || (epilogue == kEpiGeluGrad && !zin))
        return fail(NGPU_E_INVALID, "gemm: missing output / bias / pre-activation for the epilogue");
    if (ldo < N || (need_bf16 && ldt < M)) return fail(NGPU_E_INVALID, "gemm: output leading dimension too small");
    int* err = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&err, g_gemm_err);
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("gemm: ") + cudaGetErrorString(e));
    GemmArgs g{(const __nv_bfloat16*)A, (const __nv_bfloat16*)B, M, N, K, lda, ldb, out_f32,
               (__nv_bfloat16*)out_bf16, (__nv_bfloat16*)out_bf16_t, ldo, ldt, bias, zin, err, K / kGemmBK};
    cudaStream_t st = (cudaStream_t)cuda_stream;
    switch (epilogue) {
        case kEpiStore: e = launch_gemm_epi<kEpiStore>(g, bn, st); break;
        case kEpiBiasGelu: e = launch_gemm_epi<kEpiBiasGelu>(g, bn, st); break;
        case kEpiBias: e = launch_gemm_epi<kEpiBias>(g, bn, st); break;
        case kEpiGeluGrad: e = launch_gemm_epi<kEpiGeluGrad>(g, bn, st); break;
        case kEpiSplitAdd: e = launch_gemm_epi<kEpiSplitAdd>(g, bn, st); break;
        default: return fail(NGPU_E_INVALID, "gemm: unknown epilogue");
    }
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("gemm launch: ") + cudaGetErrorString(e));
    return NGPU_OK;
}

extern "C" int ngpu_gemm_error(int32_t* flag) {
    int v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_gemm_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_gemm_err, &zero, sizeof(int));
    if (e != cudaSuccess) return fail(NGPU_E_CUDA, std::string("gemm error flag: ") + cudaGetErrorString(e));
    if (flag) *flag = v;
    return NGPU_OK;
}

// ------------------------------------------------------------------ GA
namespace {

uint32_t pow2_at_least(int n) {
    uint32_t p = 2;
    while (p < (uint32_t)n) p <<= 1;
    return p;
}

// Keep freed scratch in the current device's stream-ordered pool instead of
// returning it to the system at every synchronisation (the pool's default),
// so that repeated GA steps reuse it; set once per device, for this process.
void keep_pool_memory() {
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done.push_back(dev);
}

// stream-ordered scratch, freed on the same stream
struct StreamScratch {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit StreamScratch(cudaStream_t s) : st(s) { keep_pool_memory(); }
    ~StreamScratch() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T>
    T* get(size_t count, int* rc) {
        void* p = nullptr;
        const cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), st);
        if (e != cudaSuccess) {
            *rc = fail(NGPU_E_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
            return nullptr;
        }
        ptrs.push_back(p);
        return (T*)p;
    }
};

int grid_for(size_t n, int threads) { return (int)std::min<size_t>((n + threads - 1) / threads, 148 * 32); }

}  // namespace

int ngpu_ga_offspring(const double* pop_dev, const int32_t* rank_dev, const double* crowd_dev, int32_t mu,
                      int32_t n_genes, int32_t n_kids, double low, double up, double eta_c, double eta_m, double cx_prob,
                      double p_mut, uint64_t seed, uint64_t generation, double* kids_dev, void* cuda_stream) {
    if (!pop_dev || !rank_dev || !crowd_dev || !kids_dev) return fail(NGPU_E_INVALID, "ga_offspring: null pointer");
    if (mu < 1 || n_genes < 1 || n_kids < 0) return fail(NGPU_E_INVALID, "ga_offspring: mu, n_genes >= 1");
    if ((uint64_t)n_kids >= (1ull << 44) || kGaDrawsFixed + kGaDrawsPerGene * (uint64_t)n_genes >= (1u << 20))
        return fail(NGPU_E_INVALID, "ga_offspring: too many children or genes for the draw counter");
    if (!(up > low) || !(eta_c >= 0) || !(eta_m >= 0)) return fail(NGPU_E_INVALID, "ga_offspring: bad bounds or eta");
    if (n_kids == 0) return NGPU_OK;
    GaVariation a{pop_dev, rank_dev, crowd_dev, mu, n_genes, n_kids, low, up, eta_c, eta_m, cx_prob, p_mut,
                  ga_key(seed, generation), kids_dev};
    k_ga_offspring<<<(n_kids + 127) / 128, 128, 0, (cudaStream_t)cuda_stream>>>(a);
    g_launches++;
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}

int ngpu_ga_select_truncation(const double* score_dev, int32_t n, int32_t mu, int32_t* out_idx_dev,
                              void* cuda_stream) {
    if (!score_dev || !out_idx_dev) return fail(NGPU_E_INVALID, "ga_select_truncation: null pointer");
    if (n < 1 || n > (1 << 24) || mu < 1 || mu > n) return fail(NGPU_E_INVALID, "ga_select_truncation: 1 <= mu <= n <= 2^24");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int rc = NGPU_OK;
    StreamScratch ws(st);
    const uint32_t n2 = pow2_at_least(n);
    GaSortSlice s{ws.get<uint64_t>(n2, &rc), ws.get<uint64_t>(n2, &rc), ws.get<uint32_t>(n2, &rc)};
    if (rc != NGPU_OK) return rc;
    k_ga_truncation_keys<<<grid_for(n2, 256), 256, 0, st>>>(score_dev, n, n2, s);
    g_launches += ga_sort(s, n2, 1, st);
    k_ga_take<<<grid_for(mu, 256), 256, 0, st>>>(s.idx, mu, out_idx_dev);
    g_launches += 2;
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}

int ngpu_ga_select_nsga2(const double* obj_dev, int32_t n, int32_t m, int32_t mu, int32_t* out_idx_dev,
                         int32_t* rank_dev, double* crowd_dev, int32_t* n_fronts_dev, void* cuda_stream) {
    if (!obj_dev || !out_idx_dev || !rank_dev || !crowd_dev || !n_fronts_dev)
        return fail(NGPU_E_INVALID, "ga_select_nsga2: null pointer");
    if (n < 1 || n > 32 * kGaMaxWords || mu < 1 || mu > n)
        return fail(NGPU_E_INVALID, "ga_select_nsga2: 1 <= mu <= n <= " + std::to_string(32 * kGaMaxWords));
    if (m < 1 || m > 192) return fail(NGPU_E_INVALID, "ga_select_nsga2: 1..192 objectives");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int rc = NGPU_OK;
    StreamScratch ws(st);
    const int W = (n + 31) / 32;
    const uint32_t n2 = pow2_at_least(n);
    double* fT = ws.get<double>((size_t)n * m, &rc);
    uint32_t* dom = ws.get<uint32_t>((size_t)n * W, &rc);
    GaCrowdArgs c{fT, rank_dev, n, m, n2,
                  GaSortSlice{ws.get<uint64_t>((size_t)m * n2, &rc), ws.get<uint64_t>((size_t)m * n2, &rc),
                              ws.get<uint32_t>((size_t)m * n2, &rc)},
                  ws.get<int32_t>((size_t)m * n, &rc), ws.get<int32_t>((size_t)m * n, &rc),
                  ws.get<double>((size_t)m * n, &rc)};
    GaSortSlice s{ws.get<uint64_t>(n2, &rc), ws.get<uint64_t>(n2, &rc), ws.get<uint32_t>(n2, &rc)};
    if (rc != NGPU_OK) return rc;
    k_ga_transpose<<<grid_for((size_t)n * m, 256), 256, 0, st>>>(obj_dev, n, m, fT);
    k_ga_dominance<<<dim3((n + kGaDomThreads - 1) / kGaDomThreads, W), kGaDomThreads, (size_t)m * 32 * sizeof(double),
                     st>>>(fT, n, m, W, dom);
    {
        // cooperative: every CTA resident at once (the grid barrier needs it)
        int dev = 0, sms = 0, per_sm = 0;
        NGPU_CUDA(cudaGetDevice(&dev));
        NGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        NGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ga_fronts, kGaFrontThreads, 0));
        if (per_sm < 1) return fail(NGPU_E_CUDA, "ga_select_nsga2: the front kernel cannot be resident");
        const int blocks = std::max(1, std::min(sms * per_sm, (n + kGaFrontThreads - 1) / kGaFrontThreads));
        GaFrontArgs fa{dom, n, W, rank_dev, ws.get<uint32_t>(W, &rc), ws.get<uint32_t>(W, &rc), ws.get<int>(1, &rc),
                       n_fronts_dev};
        if (rc != NGPU_OK) return rc;
        void* args[] = {&fa};
        NGPU_CUDA(cudaLaunchCooperativeKernel((const void*)k_ga_fronts, dim3(blocks), dim3(kGaFrontThreads), args, 0,
                                              st));
    }
    k_ga_crowd_keys<<<grid_for((size_t)m * n2, 256), 256, 0, st>>>(c);
    g_launches += ga_sort(c.s, n2, m, st);
    k_ga_crowd_bounds<<<grid_for((size_t)m * n, 256), 256, 0, st>>>(c);
    k_ga_crowd_contrib<<<grid_for((size_t)m * n, 256), 256, 0, st>>>(c);
    k_ga_crowd_sum<<<grid_for(n2, 256), 256, 0, st>>>(c.contrib, rank_dev, n, m, n2, crowd_dev, s);
    g_launches += ga_sort(s, n2, 1, st);
    k_ga_take<<<grid_for(mu, 256), 256, 0, st>>>(s.idx, mu, out_idx_dev);
    g_launches += 8;
    NGPU_CUDA(cudaGetLastError());
    return NGPU_OK;
}
