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
// Excess form.  A row is not stored with its diagonal d_i but with its
// excess x_i = d_i + (sum of the row's off-diagonal couplings): at assembly
// the grounded part g_i + cm_i/dt, later plus what eliminated children leak
// to ground.  The diagonal is rebuilt as x_i - a_i (- the spine's coupling to
// a lower separator) when the row is eliminated, and a child passes
// -b_c x_c / d_c to its parent's excess.  Every update is then a sum of
// nonnegative terms (the couplings a, b are negative), so FP32 keeps its
// relative precision even where couplings differ by twenty orders of
// magnitude, as between the near zero-area compartments of NEURON exports and
// ordinary ones; the textbook update d_p - b_c a_c / d_c cancels there.
//
// Storage per group of 32 instances (rows of 32 elements, one per lane):
//   vbuf   [N][2]  V and its Kahan compensation
//   slab   channel state rows, per node in mechanism order
//   ptab   parameter rows per distinct (section, mechanism set) pair
//   scr    [N][3]  (x, rhs, e) after assembly, e = b_i (V_p - V_i) the
//                  parent-row axial term; (r, c, -) after elimination with
//                  dV_i = r_i - c_i dV_parent (spines: (r, c, w), below)
//   jacc   [J][2]  FP64 (excess, rhs) accumulators of junction parents
//   jx     [J]     dV of junction parents for their far children
#pragma once
#include "channels_mainen.cuh"
#include "channels_ttpc.cuh"
#include "ngpu_math.cuh"

namespace ngpu {

constexpr int kLanes = 32;
constexpr int kMaxWarps = 8;   // 256 threads; with 3 CTAs per SM the 85-register cap keeps a whole batch resident
#ifndef NGPU_ADV_MIN_BLOCKS
#define NGPU_ADV_MIN_BLOCKS 3
#endif

// Per-node record, identical for every instance; staged in shared memory
// once per launch (32 bytes in FP32).
template <typename R>
struct NodeRec {
    R a;        // row i, column parent(i)
    R b;        // row parent(i), column i
    R cm;       // cm_i / 1000  (uF/cm2 -> mA/cm2/mV per 1/ms)
    int32_t srow;    // first channel-state row in slab
    int16_t parent;  // -1 for the root
    int16_t jslot;   // junction slot of this node, or -1
    int16_t pslot;   // the parent's junction slot if this node is a far child / subtree root
    int16_t rec;     // recording column or -1
    uint16_t mask;   // mechanism bits
    uint16_t prow;   // first parameter row
    uint16_t srows;  // number of state rows
    uint16_t prows;  // number of parameter rows
};

// A work item of the split (see make_partition on the host): a plain
// subtree [r, r + size) hanging off separator u, or a segment: spine r..l-1
// just above lower separator l plus the spine's light subtrees [lo, hi).
struct DevComp {
    int r, u, l, lk;   // root, upper separator, lower separator (-1 plain), l's skeleton index
    int lo, hi;        // light node range (plain: the whole subtree)
};
// A separator: node, skeleton parent (index) and, for a lower separator, the
// segment item that links it to its skeleton parent (-1: direct tree edge).
struct DevSep {
    int node, par, seg, pad;
};

template <typename R>
struct SimArgs {
    const NodeRec<R>* nodes;  // [N], staged into shared memory by every CTA
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
    const DevComp* comps;  // work items, by decreasing cost
    int n_comps;
    const DevSep* seps;    // skeleton, ascending node index
    int n_seps;
    R* sepv;               // [n_seps][4] rows per group: A, B, excess, rhs terms of segment links
};

template <typename R, int MS, bool INIT>
__device__ __forceinline__ void channels(uint32_t mk, R v, R dt, R* st, const float* pr, R& I, R& G) {
    if constexpr (MS == 0) ttpc_node<R, INIT>(mk, v, dt, st, pr, I, G);
    else mainen_node<R, INIT>(mk, v, dt, st, pr, I, G);
}

// The per-step channel update as one out-of-line function: the kernel calls
// it from three places (spine nodes, light subtrees, separators), and one
// shared copy keeps the instruction cache warm where warps at different
// nodes run different mechanisms.  (I, G) come back in registers.
template <typename R>
struct CurrentG {
    R I, G;
};
template <typename R, int MS>
__device__ __noinline__ CurrentG<R> channels_step(uint32_t mk, R v, R dt, R* st, const float* pr) {
    CurrentG<R> o;
    channels<R, MS, false>(mk, v, dt, st, pr, o.I, o.G);
    return o;
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
    R* sepv;
    int inst;
};

template <typename R>
__device__ __forceinline__ Group<R> group_of(const SimArgs<R>& A, int g) {
    const int lane = threadIdx.x & 31;
    const size_t N = (size_t)A.n_nodes;
    Group<R> p;
    p.vbuf = A.vbuf + (size_t)g * N * 2 * kLanes + lane;
    p.slab = A.slab + (size_t)g * A.slab_rows * kLanes + lane;
    p.ptab = A.ptab + (size_t)g * A.ptab_rows * kLanes + lane;
    p.scr = A.scr + (size_t)g * N * 3 * kLanes + lane;
    p.jacc = A.jacc + (size_t)g * 2 * A.n_jslots * kLanes + lane;
    p.jx = A.jx + (size_t)g * A.n_jslots * kLanes + lane;
    p.sepv = A.sepv + (size_t)g * 4 * A.n_seps * kLanes + lane;
    p.inst = g * kLanes + lane;
    return p;
}

// Shared memory: the node records.
template <typename R>
struct SmemPlan {
    static size_t bytes(int n_nodes) { return sizeof(NodeRec<R>) * (size_t)n_nodes; }
};

// Bulk prefetch of a run of rows into L2 (one instruction per contiguous block).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename R>
__device__ __forceinline__ void prefetch_node(const Group<R>& G, const NodeRec<R>& n, int i) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        prefetch_l2(G.scr - lane + (size_t)i * 3 * kLanes, 3 * kLanes * sizeof(R));
        prefetch_l2(G.vbuf - lane + (size_t)i * 2 * kLanes, 2 * kLanes * sizeof(R));
        if (n.srows) prefetch_l2(G.slab - lane + (size_t)n.srow * kLanes, n.srows * kLanes * sizeof(R));
        if (n.prows) prefetch_l2(G.ptab - lane + (size_t)n.prow * kLanes, n.prows * kLanes * sizeof(float));
    }
}

// Elimination of node i given its (x, rhs, e); updates the chain carry or the
// parent's FP64 junction accumulator, writes (r, c).
template <typename R>
__device__ __forceinline__ void eliminate_node(const Group<R>& G, const NodeRec<R>& s, int i, R x0, R r0,
                                               R e0, R& carry_x, R& carry_r) {
    using M = Math<R>;
    R x, r;
    if (s.jslot >= 0) {
        double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
        x = (R)((double)x0 + (double)carry_x + ja[0]);
        r = (R)((double)r0 + (double)carry_r + ja[kLanes]);
        ja[0] = 0.0;
        ja[kLanes] = 0.0;
    } else {
        x = x0 + carry_x;
        r = r0 + carry_r;
    }
    R* out = G.scr + (size_t)i * 3 * kLanes;
    if (i == 0) {  // root: no coupling left, d_0 = x_0
        out[0] = M::dv(r, x);
        out[kLanes] = 0;
        carry_x = carry_r = 0;
        return;
    }
    const R inv = M::rc(x - s.a);
    const R rr = r * inv, cc = s.a * inv;
    out[0] = rr;
    out[kLanes] = cc;
    const R cx = -s.b * (x * inv), cr = e0 - s.b * rr;  // e0: parent-row axial term
    if (s.pslot < 0) {
        carry_x = cx;
        carry_r = cr;
    } else {
        double* ja = G.jacc + (size_t)(2 * s.pslot) * kLanes;
        atomicAdd(ja, (double)cx);
        atomicAdd(ja + kLanes, (double)cr);
        carry_x = 0;
        carry_r = 0;
    }
}

// Leaf -> root elimination over the nodes idx(hi-1) .. idx(lo) of a list
// (a node range or the top-tree list), with rows read two nodes ahead.
template <typename R, typename Idx>
__device__ __forceinline__ void eliminate_list(const Group<R>& G, const NodeRec<R>* nr, int lo, int hi, Idx idx) {
    if (hi <= lo) return;
    R carry_x = 0, carry_r = 0;
    auto load = [&](int k, R& x, R& r, R& e) {
        if (k >= lo) {
            const R* row = G.scr + (size_t)idx(k) * 3 * kLanes;
            x = row[0];
            r = row[kLanes];
            e = row[2 * kLanes];
        }
    };
    R x0 = 0, r0 = 0, e0 = 0, x1 = 0, r1 = 0, e1 = 0;
    load(hi - 1, x0, r0, e0);
    load(hi - 2, x1, r1, e1);
    for (int k = hi - 1; k >= lo; --k) {
        R x2 = 0, r2 = 0, e2 = 0;
        load(k - 2, x2, r2, e2);
        const int i = idx(k);
        eliminate_node(G, nr[i], i, x0, r0, e0, carry_x, carry_r);
        x0 = x1; r0 = r1; e0 = e1;
        x1 = x2; r1 = r2; e1 = e2;
    }
}

// One node of the fused root -> leaf pass: back-substitution and V update
// (BACKSUB), channel update at the new V, next-step assembly.  Every store
// is issued after the channel code so that its loads (one round trip for all
// of the node's rows) are not held back behind them.
template <typename R, int MS, bool INIT, bool BACKSUB>
__device__ __forceinline__ void update_node(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>& n,
                                            int i, R dt, R dtn_inv, R istim_amp, bool rec_now,
                                            float* trace, R& x_prev, R& v_prev, const R* x_given) {
    R* vo = G.vbuf + (size_t)i * 2 * kLanes;
    R* o = G.scr + (size_t)i * 3 * kLanes;
    R V, vc = 0, x = 0;
    if (INIT) {
        V = (R)A.v_init;
    } else if (BACKSUB) {
        V = vo[0];
        vc = vo[kLanes];
        if (x_given) {
            x = *x_given;
        } else {
            const R r = o[0], c = o[kLanes];
            const R xp = (i == 0) ? (R)0 : (n.pslot < 0 ? x_prev : G.jx[(size_t)n.pslot * kLanes]);
            x = r - c * xp;
        }
        x_prev = x;
        kahan_add(V, vc, x);
    } else {
        V = vo[0];
    }
    // parent's new V: the previous node's for a chain child of this pass
    const R vp = INIT || i == 0 ? V
                 : (BACKSUB && n.pslot < 0) ? v_prev : G.vbuf[(size_t)n.parent * 2 * kLanes];
    v_prev = V;
    R I, Gm;
    if constexpr (INIT) {
        channels<R, MS, true>(n.mask, V, dt, G.slab + (size_t)n.srow * kLanes, G.ptab + (size_t)n.prow * kLanes,
                              I, Gm);
    } else {
        const CurrentG<R> ig = channels_step<R, MS>(n.mask, V, dt, G.slab + (size_t)n.srow * kLanes,
                                                   G.ptab + (size_t)n.prow * kLanes);
        I = ig.I;
        Gm = ig.G;
    }
    if (INIT || BACKSUB) {
        vo[0] = V;
        vo[kLanes] = vc;
    }
    if (BACKSUB && n.jslot >= 0) G.jx[(size_t)n.jslot * kLanes] = x;
    const R istim = (i == A.stim_node) ? istim_amp : (R)0;
    const R dvp = vp - V;
    o[0] = Gm + n.cm * dtn_inv;  // the row's excess: its grounded conductance
    o[kLanes] = istim - I - n.a * dvp;
    o[2 * kLanes] = n.b * dvp;
    if (rec_now && n.rec >= 0) trace[(size_t)n.rec * A.n_inst_pad] = (float)V;
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
__device__ __forceinline__ const NodeRec<R>* stage_nodes(const SimArgs<R>& A, char* smem) {
    NodeRec<R>* nr = (NodeRec<R>*)smem;
    for (int i = threadIdx.x; i < A.n_nodes; i += blockDim.x) nr[i] = A.nodes[i];
    __syncthreads();
    return nr;
}

// Initial state of group g: channels at steady state for v_init, the first
// step's rows, sample 0.  Nodes are independent here, so any number of warps
// shares them.
template <typename R, int MS>
__device__ __forceinline__ void init_body(const SimArgs<R>& A, int g) {
    const Group<R> G = group_of(A, g);
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (w == 0)
        for (int j = 0; j < 2 * A.n_jslots; ++j) G.jacc[(size_t)j * kLanes] = 0.0;
    R dt, dtn_inv, istim_amp;
    bool rec_now;
    float* trace;
    step_inputs(A, G, 0, true, dt, dtn_inv, istim_amp, rec_now, trace);
    R xd = 0, vd = 0;
    for (int i = w; i < A.n_nodes; i += nw)
        update_node<R, MS, true, false>(A, G, A.nodes[i], i, dt, dtn_inv, istim_amp, rec_now, trace, xd, vd,
                                        nullptr);
    if (w == 0) A.bad[G.inst] = 0;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps) k_sim_init(SimArgs<R> A) {
    init_body<R, MS>(A, blockIdx.x);
}

// Segment item, S1: leaf -> root elimination of the spine r..l-1 after its
// light subtrees.  Each spine row also couples to the lower separator's dV
// (w: b_l of row l-1, then the fill-in carried up the spine), so its diagonal
// is x - a + w and the row solves as dV_i = r_i - c_i dV_parent + w_i dV_l
// (stored as (r, c, w) for S3).  The same sweep accumulates what separator
// l needs for the skeleton, dV_{l-1} = gamma + alpha dV_u + beta dV_l
// expanded down the spine: alpha (row l's coupling to u), gamma (its
// right-hand side) and delta = 1 - alpha - beta, the fraction of dV_{l-1}
// that leaks to ground along the spine, which becomes l's excess.  delta is
// summed from the rows' leak fractions x_i / d_i, never as 1 - alpha - beta.
template <typename R>
__device__ __forceinline__ void eliminate_segment(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr,
                                                  const DevComp& c) {
    using M = Math<R>;
    const int r = c.r, l = c.l, b = l - 1;
    const NodeRec<R> nl = nr[l];
    const R e_l = G.scr[(size_t)l * 3 * kLanes + 2 * kLanes];
    R carry_x = 0, carry_r = 0, carry_w = 0;
    R P = 1, gam = 0, del = 0;  // P: product of -c over the rows below
    R* sv = G.sepv + (size_t)c.lk * 4 * kLanes;
    for (int i = b; i >= r; --i) {
        const NodeRec<R> s = nr[i];
        R* row = G.scr + (size_t)i * 3 * kLanes;
        R x, rh;
        const R e_i = row[2 * kLanes];
        if (s.jslot >= 0) {
            double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
            x = (R)((double)row[0] + (double)carry_x + ja[0]);
            rh = (R)((double)row[kLanes] + (double)carry_r + ja[kLanes]);
            ja[0] = 0.0;
            ja[kLanes] = 0.0;
        } else {
            x = row[0] + carry_x;
            rh = row[kLanes] + carry_r;
        }
        R w = carry_w;
        if (i == b) {
            w = -nl.b;
            rh += e_l;
        }
        const R inv = M::rc(x - s.a + w);
        const R rr = rh * inv, cc = s.a * inv, om = w * inv, lam = x * inv;
        row[0] = rr;
        row[kLanes] = cc;
        row[2 * kLanes] = om;
        gam += rr * P;
        del += lam * P;
        P *= -cc;
        if (i > r) {
            carry_x = -s.b * lam;
            carry_r = e_i - s.b * rr;
            carry_w = -s.b * om;
        } else {
            double* ja = G.jacc + (size_t)(2 * s.pslot) * kLanes;  // the upper separator
            atomicAdd(ja, (double)(-s.b * lam));
            atomicAdd(ja + kLanes, (double)(e_i - s.b * rr));
            sv[kLanes] = s.b * om;  // B: row u's coupling to dV_l
        }
    }
    sv[0] = nl.a * P;              // A: row l's coupling to dV_u (alpha = P)
    sv[2 * kLanes] = -nl.a * del;  // added to l's excess
    sv[3 * kLanes] = -nl.a * gam;  // added to rhs_l
}

// Warp-level work queue: lane 0 takes the next item, the warp shares it.
__device__ __forceinline__ int next_item(int* ctr) {
    int k = 0;
    if ((threadIdx.x & 31) == 0) k = atomicAdd(ctr, 1);
    return __shfl_sync(0xffffffffu, k, 0);
}

// Per timestep (three barriers):
//   S1  all warps take items from a queue, largest first: leaf -> root
//       elimination of plain subtrees and of segments (above); each item's
//       contribution to its upper separator goes to that separator's FP64
//       accumulator
//   S2  warp 0 solves the skeleton (the separators, a few dozen nodes) with
//       the reduced couplings of the segments, and updates their V
//   S3  all warps take items again: back-substitution + V update + channel
//       update + next-step assembly of every node of the item (a segment
//       also does its lower separator's channels, which need the spine's new
//       V); separators linked directly to the skeleton are items too
// n_steps timesteps of group g; the items are shared by however many warps
// the CTA has (the split was sized for A.n_warps).
template <typename R, int MS>
__device__ __forceinline__ void advance_body(const SimArgs<R>& A, int g, int t0, int n_steps, char* smem,
                                             int* ctr) {
    const Group<R> G = group_of(A, g);
    const int w = threadIdx.x >> 5;
    const NodeRec<R>* nr = stage_nodes(A, smem);
    if (threadIdx.x == 0) { ctr[0] = 0; ctr[1] = 0; }
    __syncthreads();
    int bad = 0;
    const int n_items3 = A.n_comps + A.n_seps;
    for (int t = t0; t < t0 + n_steps; ++t) {
        // S1
        if (threadIdx.x == 0) ctr[1] = 0;
        for (int k = next_item(&ctr[0]); k < A.n_comps; k = next_item(&ctr[0])) {
            const DevComp c = A.comps[k];
            eliminate_list(G, nr, c.lo, c.hi, [](int q) { return q; });
            if (c.l >= 0) eliminate_segment(A, G, nr, c);
        }
        __syncthreads();
        // S2: skeleton
        if (w == 0) {
            using M = Math<R>;
            for (int k = A.n_seps - 1; k >= 0; --k) {
                const DevSep sp = A.seps[k];
                const NodeRec<R> s = nr[sp.node];
                R* row = G.scr + (size_t)sp.node * 3 * kLanes;
                double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
                R x = (R)((double)row[0] + ja[0]);
                R rh = (R)((double)row[kLanes] + ja[kLanes]);
                ja[0] = 0.0;
                ja[kLanes] = 0.0;
                R Acp = s.a, Bcp = s.b, e_up = row[2 * kLanes];
                if (sp.seg >= 0) {
                    const R* sv = G.sepv + (size_t)k * 4 * kLanes;
                    Acp = sv[0];
                    Bcp = sv[kLanes];
                    x += sv[2 * kLanes];
                    rh += sv[3 * kLanes];
                    e_up = 0;  // the segment already folded this node's axial term in
                }
                if (k == 0) {
                    row[0] = M::dv(rh, x);
                    break;
                }
                const R inv = M::rc(x - Acp);
                const R rr = rh * inv, cc = Acp * inv;
                row[0] = rr;
                row[kLanes] = cc;
                double* jp = G.jacc + (size_t)(2 * nr[A.seps[sp.par].node].jslot) * kLanes;
                jp[0] += (double)(-Bcp * (x * inv));
                jp[kLanes] += (double)(e_up - Bcp * rr);
            }
            for (int k = 0; k < A.n_seps; ++k) {
                const DevSep sp = A.seps[k];
                const NodeRec<R> s = nr[sp.node];
                const R* row = G.scr + (size_t)sp.node * 3 * kLanes;
                R x;
                if (k == 0) x = row[0];
                else x = row[0] - row[kLanes] * G.jx[(size_t)nr[A.seps[sp.par].node].jslot * kLanes];
                G.jx[(size_t)s.jslot * kLanes] = x;
                R* vo = G.vbuf + (size_t)sp.node * 2 * kLanes;
                R V = vo[0], vc = vo[kLanes];
                kahan_add(V, vc, x);
                vo[0] = V;
                vo[kLanes] = vc;
                if (k == 0 && !(fabs(V) < (R)1e6)) bad = 1;  // NaN / Inf / blow-up
            }
        }
        __syncthreads();
        // S3
        if (threadIdx.x == 0) ctr[0] = 0;
        R dt, dtn_inv, istim_amp;
        bool rec_now;
        float* trace;
        step_inputs(A, G, t, false, dt, dtn_inv, istim_amp, rec_now, trace);
        for (int k = next_item(&ctr[1]); k < n_items3; k = next_item(&ctr[1])) {
            if (k < A.n_comps) {
                const DevComp c = A.comps[k];
                R x_prev = 0, v_prev = 0;
                if (c.l >= 0) {  // spine: dV_i = r_i - c_i dV_parent + w_i dV_l, from separator u down
                    R xp = G.jx[(size_t)nr[c.u].jslot * kLanes];
                    const R xl = G.jx[(size_t)nr[c.l].jslot * kLanes];
                    v_prev = G.vbuf[(size_t)c.u * 2 * kLanes];
                    for (int i = c.r; i < c.l; ++i) {
                        if (i + 2 < c.l) prefetch_node(G, nr[i + 2], i + 2);
                        const R* row = G.scr + (size_t)i * 3 * kLanes;
                        const R xi = row[0] - row[kLanes] * xp + row[2 * kLanes] * xl;
                        xp = xi;
                        update_node<R, MS, false, true>(A, G, nr[i], i, dt, dtn_inv, istim_amp, rec_now, trace,
                                                        x_prev, v_prev, &xi);
                    }
                }
                x_prev = 0;
                for (int i = c.lo; i < c.hi; ++i) {
                    if (i + 2 < c.hi) prefetch_node(G, nr[i + 2], i + 2);
                    update_node<R, MS, false, true>(A, G, nr[i], i, dt, dtn_inv, istim_amp, rec_now, trace, x_prev,
                                                    v_prev, nullptr);
                }
                if (c.l >= 0) {
                    R xd = 0, vd = 0;
                    update_node<R, MS, false, false>(A, G, nr[c.l], c.l, dt, dtn_inv, istim_amp, rec_now, trace,
                                                     xd, vd, nullptr);
                }
            } else {
                const DevSep sp = A.seps[k - A.n_comps];
                if (sp.seg < 0) {
                    R xd = 0, vd = 0;
                    update_node<R, MS, false, false>(A, G, nr[sp.node], sp.node, dt, dtn_inv, istim_amp, rec_now,
                                                     trace, xd, vd, nullptr);
                }
            }
        }
        __syncthreads();
    }
    if (w == 0 && bad) A.bad[G.inst] = 1;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps, NGPU_ADV_MIN_BLOCKS) k_sim_advance(SimArgs<R> A, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    __shared__ int ctr[2];
    advance_body<R, MS>(A, blockIdx.x, t0, n_steps, smem, ctr);
}

// Several simulations (morphologies of different sizes, one mechanism set)
// in one launch: CTAs [cta0[k], cta0[k+1]) run the groups of simulation k.
// The arguments live in the kernel's parameter space (__grid_constant__), so
// a CTA reads its simulation's fields through the constant cache.
constexpr int kMaxBatch = 16;
template <typename R>
struct BatchArgs {
    SimArgs<R> sim[kMaxBatch];
    int cta0[kMaxBatch + 1];
    int n;
};

__device__ __forceinline__ int batch_member(const int* cta0, int n) {
    int k = 0;
    while (k + 1 < n && (int)blockIdx.x >= cta0[k + 1]) ++k;
    return k;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps) k_batch_init(const __grid_constant__ BatchArgs<R> B) {
    const int k = batch_member(B.cta0, B.n);
    init_body<R, MS>(B.sim[k], blockIdx.x - B.cta0[k]);
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps, NGPU_ADV_MIN_BLOCKS)
    k_batch_advance(const __grid_constant__ BatchArgs<R> B, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    __shared__ int ctr[2];
    const int k = batch_member(B.cta0, B.n);
    advance_body<R, MS>(B.sim[k], blockIdx.x - B.cta0[k], t0, n_steps, smem, ctr);
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

// One recording site of the trace into a caller's [instance][site][sample]
// array: out[(inst * out_sites + out_site) * n_samples + s] <-
// trace[(s * n_rec + col) * n_inst_pad + inst].  Used by the allocation-free
// entry point, which writes straight into the caller's buffer.
__global__ void k_trace_transpose_site(const float* __restrict__ trace, int n_samples, int n_rec, int col,
                                       int n_inst_pad, int n_inst, int out_sites, int out_site,
                                       float* __restrict__ out) {
    __shared__ float tile[32][33];
    const int i0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int s = s0 + k, i = i0 + threadIdx.x;
        if (s < n_samples && i < n_inst_pad) tile[k][threadIdx.x] = trace[((size_t)s * n_rec + col) * n_inst_pad + i];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, s = s0 + threadIdx.x;
        if (i < n_inst && s < n_samples) out[((size_t)i * out_sites + out_site) * n_samples + s] = tile[threadIdx.x][k];
    }
}

}  // namespace ngpu
