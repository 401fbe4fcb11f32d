// Fused multi-compartment simulation kernels.
//
// One CTA advances one group of 32 instances (parameter set x stimulus; lane
// = instance) through every timestep of a launch.  All lanes of a warp always
// work on the same node, so the per-node mechanism branches are warp-uniform
// and every state / parameter / scratch access is one coalesced 128-byte row
// (structure of arrays, instance index innermost).
//
// Each timestep is the reference's per-step algorithm
// (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/CudaStuff.cu:227-330): Hines
// forward elimination leaf -> root (BeforeLU, :31-69), back-substitution root
// -> leaf (BkSub, :72-104), V += dV (:298-301), cnexp channel-state update at
// the new V (:324-326), channel currents (:262-267) and the assembly of the
// next step's diagonal and right-hand side (:268-291).
//
// The tree is split once on the host into a small "top tree" (containing the
// root) and subtrees hanging off it, bin-packed over the CTA's W warps by
// channel cost.  Subtrees are contiguous node ranges in Hines (depth-first)
// order and independent given their top-tree parent, so elimination and
// back-substitution of the subtrees run on all warps at once; warp 0 solves
// only the top tree in between (S1 / S2 / S3 below).  A chain child hands its
// elimination term to node i-1 in registers; any other child (branch
// junction, or a subtree root) adds it to an FP64 junction accumulator of
// its parent.
//
// Storage per group of 32 instances (rows of 32 elements, one per lane):
//   vbuf   [N][2]  V and its Kahan compensation
//   slab   channel state rows, per node in mechanism order
//   ptab   parameter rows per distinct (section, mechanism set) pair
//   scr    [N][3]  (d, rhs, e) after assembly, e = b_i (V_p - V_i) the
//                  parent-row axial term; (r, c, -) after elimination with
//                  dV_i = r_i - c_i dV_parent
//   jacc   [J][2]  FP64 (d, rhs) accumulators of junction parents
//   jx     [J]     dV of junction parents for their far children
#pragma once
#include "channels_mainen.cuh"
#include "channels_ttpc.cuh"
#include "ngpu_math.cuh"

namespace ngpu {

constexpr int kLanes = 32;
constexpr int kMaxWarps = 16;

struct NodeInfo {
    int32_t parent;  // -1 for the root
    uint32_t mask;   // mechanism bits
    int32_t srow;    // first channel-state row in slab
    int32_t prow;    // first parameter row
    int32_t jslot;   // junction slot if this node has a child other than node+1, else -1
    int32_t pslot;   // the parent's junction slot if parent != node-1, else -1
    int32_t rec;     // recording column or -1
    int32_t pad;
};

template <typename R>
struct NodeCoef {
    R a;       // row i, column parent(i)
    R b;       // row parent(i), column i
    R dconst;  // -a_i - sum over children c of b_c
    R cm;      // cm_i / 1000  (uF/cm2 -> mA/cm2/mV per 1/ms)
};

template <typename R>
struct SolveNode {  // phase-S topology, staged in shared memory
    R a, b;
    int32_t jslot, pslot;
};

template <typename R>
struct SimArgs {
    const NodeInfo* info;
    const NodeCoef<R>* coef;
    const SolveNode<R>* solve;
    int n_nodes;
    R* vbuf;
    R* slab;
    int slab_rows;
    const float* ptab;
    int ptab_rows;
    R* scr;
    double* jacc;
    R* jx;
    int n_jslots;
    const float* amps;     // [n_stim][nt]
    const float* dts;      // [nt]
    int nt;
    int stim_node;
    double stim_scale;     // 100 / area (nA/um2 -> mA/cm2)
    const int* inst_stim;  // [n_inst_pad]
    float* trace;          // [n_samples][n_rec][n_inst_pad]
    int n_rec;
    int rec_every;
    int n_inst_pad;
    float v_init;
    int* bad;              // [n_inst_pad] non-finite voltage flags
    int* err;              // device error word
    int n_warps;
    const int2* rows;      // [N] (state rows, parameter rows) per node, for prefetch
    const int2* seg;       // subtree node ranges [start, end), grouped by warp
    int seg_off[kMaxWarps + 1];
    const int* top;        // top-tree nodes, ascending
    int n_top;
    const int* tch;        // top nodes whose channels each warp updates
    int tch_off[kMaxWarps + 1];
};

template <typename R, int MS, bool INIT>
__device__ __forceinline__ void channels(uint32_t mk, R v, R dt, R* st, const float* pr, R& I, R& G) {
    if constexpr (MS == 0) ttpc_node<R, INIT>(mk, v, dt, st, pr, I, G);
    else mainen_node<R, INIT>(mk, v, dt, st, pr, I, G);
}

// v + x with running compensation c (Kahan); the round-to-nearest intrinsics
// keep the compiler from re-associating the correction away.
__device__ __forceinline__ void kahan_add(float& v, float& c, float x) {
    float y = __fsub_rn(x, c);
    float t = __fadd_rn(v, y);
    c = __fsub_rn(__fsub_rn(t, v), y);
    v = t;
}
__device__ __forceinline__ void kahan_add(double& v, double& c, double x) { v += x; (void)c; }

template <typename R>
struct Group {  // per-CTA pointers (lane offset included)
    R* vbuf;
    R* slab;
    const float* ptab;
    R* scr;
    double* jacc;
    R* jx;
    int inst;
};

template <typename R>
__device__ __forceinline__ Group<R> group_of(const SimArgs<R>& A) {
    const int g = blockIdx.x, lane = threadIdx.x & 31;
    const size_t N = (size_t)A.n_nodes;
    Group<R> p;
    p.vbuf = A.vbuf + (size_t)g * N * 2 * kLanes + lane;
    p.slab = A.slab + (size_t)g * A.slab_rows * kLanes + lane;
    p.ptab = A.ptab + (size_t)g * A.ptab_rows * kLanes + lane;
    p.scr = A.scr + (size_t)g * N * 3 * kLanes + lane;
    p.jacc = A.jacc + (size_t)g * 2 * A.n_jslots * kLanes + lane;
    p.jx = A.jx + (size_t)g * A.n_jslots * kLanes + lane;
    p.inst = g * kLanes + lane;
    return p;
}

// Shared memory: the solve topology of every node.
template <typename R>
struct SmemPlan {
    static size_t bytes(int n_nodes) { return sizeof(SolveNode<R>) * (size_t)n_nodes; }
};

// Bulk prefetch of a run of rows into L2 (one instruction per contiguous block).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename R>
__device__ __forceinline__ void prefetch_node(const SimArgs<R>& A, const Group<R>& G, int i, int lane) {
    if (lane == 0) {
        const NodeInfo ni = A.info[i];
        const int2 rows = A.rows[i];  // (state rows, parameter rows) of node i
        prefetch_l2(G.scr - lane + (size_t)i * 3 * kLanes, 3 * kLanes * sizeof(R));
        prefetch_l2(G.vbuf - lane + (size_t)i * 2 * kLanes, 2 * kLanes * sizeof(R));
        if (rows.x) prefetch_l2(G.slab - lane + (size_t)ni.srow * kLanes, rows.x * kLanes * sizeof(R));
        if (rows.y) prefetch_l2(G.ptab - lane + (size_t)ni.prow * kLanes, rows.y * kLanes * sizeof(float));
    }
}

// Elimination of node i given its (d, rhs, e) rows; updates the chain carry
// or the parent's junction accumulator, writes (r, c).
template <typename R>
__device__ __forceinline__ void eliminate_node(const Group<R>& G, const SolveNode<R>& s, int i, R d0,
                                               R r0, R e0, R& carry_d, R& carry_r) {
    using M = Math<R>;
    R d, r;
    if (s.jslot >= 0) {
        double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
        d = (R)((double)d0 + (double)carry_d + ja[0]);
        r = (R)((double)r0 + (double)carry_r + ja[kLanes]);
        ja[0] = 0.0;
        ja[kLanes] = 0.0;
    } else {
        d = d0 + carry_d;
        r = r0 + carry_r;
    }
    R* out = G.scr + (size_t)i * 3 * kLanes;
    if (i == 0) {  // root: dV_0 = rhs_0 / d_0
        out[0] = M::dv(r, d);
        out[kLanes] = 0;
        carry_d = carry_r = 0;
        return;
    }
    const R inv = M::rc(d);
    const R rr = r * inv, cc = s.a * inv;
    out[0] = rr;
    out[kLanes] = cc;
    const R cd = -s.b * cc, cr = e0 - s.b * rr;  // e0: parent-row axial term
    if (s.pslot < 0) {
        carry_d = cd;
        carry_r = cr;
    } else {
        double* ja = G.jacc + (size_t)(2 * s.pslot) * kLanes;
        atomicAdd(ja, (double)cd);
        atomicAdd(ja + kLanes, (double)cr);
        carry_d = 0;
        carry_r = 0;
    }
}

// Leaf -> root elimination over nodes [lo, hi), with the next rows loaded
// one node ahead.
template <typename R>
__device__ __forceinline__ void eliminate_range(const Group<R>& G, const SolveNode<R>* sn, int lo, int hi) {
    if (hi <= lo) return;
    R carry_d = 0, carry_r = 0;
    const R* row = G.scr + (size_t)(hi - 1) * 3 * kLanes;
    R d = row[0], r = row[kLanes], e = row[2 * kLanes];
    for (int i = hi - 1; i >= lo; --i) {
        R dn = 0, rn = 0, en = 0;
        if (i > lo) {
            const R* nx = G.scr + (size_t)(i - 1) * 3 * kLanes;
            dn = nx[0];
            rn = nx[kLanes];
            en = nx[2 * kLanes];
        }
        eliminate_node(G, sn[i], i, d, r, e, carry_d, carry_r);
        d = dn;
        r = rn;
        e = en;
    }
}

// One node of the fused root -> leaf pass: back-substitution, V update
// (BACKSUB), channel update at the new V, next-step assembly.
template <typename R, int MS, bool INIT, bool BACKSUB>
__device__ __forceinline__ void update_node(const SimArgs<R>& A, const Group<R>& G, const SolveNode<R>& s,
                                            int i, R dt, R dtn_inv, R istim_amp, bool rec_now,
                                            float* trace, R& x_prev) {
    const NodeInfo ni = A.info[i];
    const NodeCoef<R> c = A.coef[i];
    R* vo = G.vbuf + (size_t)i * 2 * kLanes;
    R* o = G.scr + (size_t)i * 3 * kLanes;
    R V;
    if (INIT) {
        V = (R)A.v_init;
        vo[0] = V;
        vo[kLanes] = 0;
    } else if (BACKSUB) {
        const R xp = (i == 0) ? (R)0 : (s.pslot < 0 ? x_prev : G.jx[(size_t)s.pslot * kLanes]);
        const R x = o[0] - o[kLanes] * xp;
        if (s.jslot >= 0) G.jx[(size_t)s.jslot * kLanes] = x;
        x_prev = x;
        V = vo[0];
        R vc = vo[kLanes];
        kahan_add(V, vc, x);
        vo[0] = V;
        vo[kLanes] = vc;
    } else {
        V = vo[0];
    }
    const R vp = INIT ? V : ((i == 0) ? V : G.vbuf[(size_t)ni.parent * 2 * kLanes]);
    R I, Gm;
    channels<R, MS, INIT>(ni.mask, V, dt, G.slab + (size_t)ni.srow * kLanes, G.ptab + (size_t)ni.prow * kLanes,
                          I, Gm);
    const R istim = (i == A.stim_node) ? istim_amp : (R)0;
    const R dvp = vp - V;
    o[0] = Gm + c.cm * dtn_inv + c.dconst;
    o[kLanes] = istim - I - c.a * dvp;
    o[2 * kLanes] = c.b * dvp;
    if (rec_now && ni.rec >= 0) trace[(size_t)ni.rec * A.n_inst_pad] = (float)V;
}

template <typename R>
__device__ __forceinline__ void step_inputs(const SimArgs<R>& A, const Group<R>& G, int t, bool init, R& dt,
                                            R& dtn_inv, R& istim_amp, bool& rec_now, float*& trace) {
    const int tn = init ? 0 : t + 1;
    const int tnc = tn < A.nt ? tn : A.nt - 1;
    dt = init ? (R)0 : (R)A.dts[t];
    dtn_inv = (R)1 / (R)A.dts[tnc];
    const int stim = A.inst_stim[G.inst];
    istim_amp = (R)A.stim_scale * (R)A.amps[(size_t)stim * A.nt + tnc];
    rec_now = tn < A.nt && (tn % A.rec_every) == 0;
    trace = A.trace + (size_t)(tn / A.rec_every) * A.n_rec * A.n_inst_pad + G.inst;
}

template <typename R>
__device__ __forceinline__ void stage_solve_topology(const SimArgs<R>& A, char* smem) {
    SolveNode<R>* sn = (SolveNode<R>*)smem;
    for (int i = threadIdx.x; i < A.n_nodes; i += blockDim.x) sn[i] = A.solve[i];
    __syncthreads();
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps) k_sim_init(SimArgs<R> A) {
    const Group<R> G = group_of(A);
    const int w = threadIdx.x >> 5;
    if (w == 0)
        for (int j = 0; j < 2 * A.n_jslots; ++j) G.jacc[(size_t)j * kLanes] = 0.0;
    R dt, dtn_inv, istim_amp;
    bool rec_now;
    float* trace;
    step_inputs(A, G, 0, true, dt, dtn_inv, istim_amp, rec_now, trace);
    R xd = 0;
    const SolveNode<R> none{};
    for (int i = w; i < A.n_nodes; i += A.n_warps)
        update_node<R, MS, true, false>(A, G, none, i, dt, dtn_inv, istim_amp, rec_now, trace, xd);
    if (w == 0) A.bad[G.inst] = 0;
}

// Per timestep:
//   S1  every warp: leaf -> root elimination of its subtrees (they hang off
//       the top tree, so no two warps touch the same node; contributions of
//       subtree roots go to the top parents' FP64 accumulators)
//   S2  warp 0: elimination and back-substitution of the small top tree,
//       V update of the top nodes
//   S3  every warp: fused back-substitution + V update + channels + next-step
//       assembly for its subtrees, then channels + assembly of its share of
//       the top nodes
template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps) k_sim_advance(SimArgs<R> A, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    const Group<R> G = group_of(A);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    stage_solve_topology(A, smem);
    const SolveNode<R>* sn = (const SolveNode<R>*)smem;
    const int s_lo = A.seg_off[w], s_hi = A.seg_off[w + 1];
    const int c_lo = A.tch_off[w], c_hi = A.tch_off[w + 1];
    int bad = 0;
    for (int t = t0; t < t0 + n_steps; ++t) {
        // S1
        for (int k = s_hi - 1; k >= s_lo; --k) {
            const int2 sg = A.seg[k];
            eliminate_range(G, sn, sg.x, sg.y);
        }
        __syncthreads();
        // S2
        if (w == 0) {
            R carry_d = 0, carry_r = 0;
            for (int k = A.n_top - 1; k >= 0; --k) {
                const int i = A.top[k];
                const R* row = G.scr + (size_t)i * 3 * kLanes;
                eliminate_node(G, sn[i], i, row[0], row[kLanes], row[2 * kLanes], carry_d, carry_r);
            }
            R x_prev = 0;
            for (int k = 0; k < A.n_top; ++k) {
                const int i = A.top[k];
                const SolveNode<R> s = sn[i];
                R* o = G.scr + (size_t)i * 3 * kLanes;
                const R xp = (i == 0) ? (R)0 : (s.pslot < 0 ? x_prev : G.jx[(size_t)s.pslot * kLanes]);
                const R x = o[0] - o[kLanes] * xp;
                if (s.jslot >= 0) G.jx[(size_t)s.jslot * kLanes] = x;
                x_prev = x;
                R* vo = G.vbuf + (size_t)i * 2 * kLanes;
                R V = vo[0], vc = vo[kLanes];
                kahan_add(V, vc, x);
                vo[0] = V;
                vo[kLanes] = vc;
                if (i == 0 && !(fabs(V) < (R)1e6)) bad = 1;  // NaN / Inf / blow-up
            }
        }
        __syncthreads();
        // S3
        R dt, dtn_inv, istim_amp;
        bool rec_now;
        float* trace;
        step_inputs(A, G, t, false, dt, dtn_inv, istim_amp, rec_now, trace);
        for (int k = s_lo; k < s_hi; ++k) {
            const int2 sg = A.seg[k];
            R x_prev = 0;
            for (int i = sg.x; i < sg.y; ++i) {
                if (i + 1 < sg.y) prefetch_node(A, G, i + 1, lane);
                update_node<R, MS, false, true>(A, G, sn[i], i, dt, dtn_inv, istim_amp, rec_now, trace, x_prev);
            }
        }
        R xd = 0;
        for (int k = c_lo; k < c_hi; ++k) {
            const int i = A.tch[k];
            update_node<R, MS, false, false>(A, G, sn[i], i, dt, dtn_inv, istim_amp, rec_now, trace, xd);
        }
        __syncthreads();
    }
    if (w == 0 && bad) A.bad[G.inst] = 1;
}

// Parameter table: ptab[g][row][lane] = params[set][row_param[row]][row_sec[row]]
// for instance g*32+lane = set*n_stim + stim (padding lanes repeat the last instance).
__global__ void k_gather_params(const float* __restrict__ params, const int* __restrict__ row_param,
                                const int* __restrict__ row_sec, int ptab_rows, int n_params,
                                int n_sections, int n_stim, int n_inst, int n_groups,
                                float* __restrict__ ptab) {
    const size_t total = (size_t)n_groups * ptab_rows * kLanes;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(idx % kLanes);
        const size_t rem = idx / kLanes;
        const int row = (int)(rem % ptab_rows);
        const int g = (int)(rem / ptab_rows);
        int inst = g * kLanes + lane;
        if (inst >= n_inst) inst = n_inst - 1;
        const int set = inst / n_stim;
        ptab[idx] = params[((size_t)set * n_params + row_param[row]) * n_sections + row_sec[row]];
    }
}

// out[inst][rec][sample] <- trace[sample][rec][inst], tiled through shared memory.
__global__ void k_trace_transpose(const float* __restrict__ trace, int n_samples, int n_rec,
                                  int n_inst_pad, int n_inst, float* __restrict__ out) {
    __shared__ float tile[32][33];
    const int rec = blockIdx.z;
    const int i0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int s = s0 + k, i = i0 + threadIdx.x;
        if (s < n_samples && i < n_inst_pad)
            tile[k][threadIdx.x] = trace[((size_t)s * n_rec + rec) * n_inst_pad + i];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, s = s0 + threadIdx.x;
        if (i < n_inst && s < n_samples)
            out[((size_t)i * n_rec + rec) * n_samples + s] = tile[threadIdx.x][k];
    }
}

}  // namespace ngpu
