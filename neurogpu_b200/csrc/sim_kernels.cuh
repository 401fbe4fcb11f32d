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
// The tree is split once on the host into a skeleton of separator nodes
// (containing the root) and work items hanging off it, sized by channel
// cost for the CTA's W warps: plain subtrees, and segments (a heavy-path
// spine between two separators plus the spine's light subtrees).  Items are
// contiguous node ranges in Hines (depth-first, heavy-first) order and
// independent given their separators, so all warps work on items at once and
// warp 0 alone solves the skeleton in between (S2 / S3 in advance_body).
// Within an item a warp makes two passes per step: root -> leaf,
// back-substitution and V update; leaf -> root, each node's channel update,
// its row for the next step and the row's elimination, so assembled rows
// never leave registers.  A chain child hands its elimination term to node
// i-1 in registers; any other child (branch junction, or an item root) adds
// it to an FP64 junction accumulator of its parent.
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
//   scr    [N][3]  eliminated rows (r, c, -) with dV_i = r_i - c_i dV_parent
//                  (spines: (r, c, w), below); separators: their assembled
//                  rows (x, rhs, e), e = b_i (V_p - V_i) the parent-row
//                  axial term, for the skeleton solve
//   jacc   [J][2]  FP64 (excess, rhs) accumulators of junction parents
//   jx     [J]     dV of junction parents for their far children
#pragma once
#include "channels_mainen.cuh"
#include "channels_ttpc.cuh"
#include "ngpu_math.cuh"
#include "node_classes.cuh"
#ifdef NGPU_GENERATED_NODE  // a mechanism set generated from NMODL files (runtime compilation only)
#include "ngpu_generated.cuh"
#endif

namespace ngpu {

constexpr int kLanes = 32;
constexpr int kMaxWarps = 8;   // 256 threads; with 3 CTAs per SM the 85-register cap keeps a whole batch resident
#ifndef NGPU_ADV_MIN_BLOCKS
#define NGPU_ADV_MIN_BLOCKS 3
#endif
// L2 prefetch of each node's state and parameter rows two nodes ahead in the
// channel pass.  A compile-time choice: it pays on models whose nodes read
// many rows (every node of the HH-type cells carries 7 mechanisms, ~30 rows)
// and costs where most nodes read few (the TTPC-like cell, ~12), even when a
// runtime flag turns it off; the runtime-specialised kernels set it per model.
#ifndef NGPU_CH_PREFETCH
#define NGPU_CH_PREFETCH 1
#endif
// Without that prefetch, the channel pass starts each node's loads one node
// early (channels_item).  The runtime-specialised kernels for CTAs of more
// than 8 warps at one CTA per SM turn it off: there it measured 4 % slower.
#ifndef NGPU_CH_AHEAD
#define NGPU_CH_AHEAD 1
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
    uint8_t srows;   // number of state rows
    uint8_t prows;   // number of parameter rows
    uint8_t cls;     // mechanism-set class (node_class)
    uint8_t pad_;
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
    int n_inst;            // instances holding a (set, stimulus) pair; the rest pad the last group
    float v_init;
    int* bad;              // [n_inst_pad] non-finite voltage flags
    int n_warps;
    const DevComp* comps;  // work items, by decreasing cost
    int n_comps;
    const DevSep* seps;    // skeleton, ascending node index
    int n_seps;
    R* sepv;               // [n_seps][4] rows per group: A, B, excess, rhs terms of segment links
    int s2_stage;          // skeleton solve from shared memory (SmemPlan)
};

// mk: the node's mechanism bits, a runtime value or a std::integral_constant
// (then every mechanism test folds at compile time).
// MS: 0 TTPC, 1 Mainen, 2 the generated set of this translation unit.
template <typename R, int MS, bool INIT, typename MK>
__device__ __forceinline__ void channels(MK mk, R v, R dt, R* st, const float* pr, R& I, R& G) {
    if constexpr (MS == 0) ttpc_node<R, INIT>(mk, v, dt, st, pr, I, G);
    else if constexpr (MS == 1) mainen_node<R, INIT>(mk, v, dt, st, pr, I, G);
#ifdef NGPU_GENERATED_NODE
    else generated_node<R, INIT>(mk, v, dt, st, pr, I, G);
#endif
}

// Channel update of a node of mechanism-set class cls: class k < sizeof...(Ms)
// runs the code specialised for mask Ms[k] (straight-line code in which the
// compiler interleaves all of the node's gates); other nodes run the generic
// code on their runtime mask.
template <typename R, int MS, bool INIT, uint32_t M0, uint32_t... Ms>
__device__ __forceinline__ void channels_cls(int cls, uint32_t mk, R v, R dt, R* st, const float* pr, R& I, R& G) {
    if (cls == 0) {
        channels<R, MS, INIT>(MaskC<M0>{}, v, dt, st, pr, I, G);
    } else if constexpr (sizeof...(Ms) > 0) {
        channels_cls<R, MS, INIT, Ms...>(cls - 1, mk, v, dt, st, pr, I, G);
    } else {
#if NGPU_CLASSES_COMPLETE
        // every node's mask is one of the classes (the host compiles this only
        // then): no node comes here, and the generic code's registers are not
        // reserved for a path that never runs
        I = (R)0;
        G = (R)0;
#else
        channels<R, MS, INIT>(mk, v, dt, st, pr, I, G);
#endif
    }
}
template <typename R, int MS, bool INIT, uint32_t... Ms>
__device__ __forceinline__ void channels_list(MaskList<Ms...>, int cls, uint32_t mk, R v, R dt, R* st,
                                              const float* pr, R& I, R& G) {
    if constexpr (sizeof...(Ms) > 0) channels_cls<R, MS, INIT, Ms...>(cls, mk, v, dt, st, pr, I, G);
    else channels<R, MS, INIT>(mk, v, dt, st, pr, I, G);
}

// The per-step channel update.  (I, G) come back in registers.
template <typename R>
struct CurrentG {
    R I, G;
};
template <typename R, int MS, typename Classes>
__device__ __forceinline__ CurrentG<R> channels_step(int cls, uint32_t mk, R v, R dt, R* st, const float* pr) {
    CurrentG<R> o;
    channels_list<R, MS, false>(Classes{}, cls, mk, v, dt, st, pr, o.I, o.G);
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

// Pointers of group g at lane `lane` (instance g * 32 + lane).
template <typename R>
__device__ __forceinline__ Group<R> group_lane(const SimArgs<R>& A, int g, int lane) {
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

// Lane = instance: this thread's lane of group g.
template <typename R>
__device__ __forceinline__ Group<R> group_of(const SimArgs<R>& A, int g) {
    return group_lane(A, g, (int)(threadIdx.x & 31));
}

// Shared memory: the node records, then (s2_stage) the skeleton's staging
// rows, [n_seps][32] each: two FP64 accumulators (excess, right-hand side)
// and five R rows (coupling A / later c, coupling B / later r, axial term
// e / later dV, V, Kahan term).
template <typename R>
struct SmemPlan {
    static __host__ __device__ size_t nodes(int n_nodes) {
        return (sizeof(NodeRec<R>) * (size_t)n_nodes + 15) / 16 * 16;
    }
    static __host__ __device__ size_t bytes(int n_nodes, int n_seps = 0, int stage = 0) {
        return nodes(n_nodes) + (stage ? (size_t)n_seps * 32 * (2 * sizeof(double) + 5 * sizeof(R)) : 0);
    }
    // thread-item layout: the node records, then per warp (one instance) the
    // skeleton's staging rows, [n_seps] each of the same seven
    static __host__ __device__ size_t ti_stage(int n_seps) {
        return ((size_t)n_seps * (2 * sizeof(double) + 5 * sizeof(R)) + 15) / 16 * 16;
    }
    static __host__ __device__ size_t ti_bytes(int n_nodes, int n_seps, int warps) {
        return nodes(n_nodes) + (size_t)warps * ti_stage(n_seps);
    }
};

// Bulk prefetch of a run of rows into L2 (one instruction per contiguous block).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L2 prefetch of the rows the back-substitution pass reads for nodes
// [i, i + n): (r, c, w) and (V, Kahan term), two contiguous blocks.
template <typename R>
__device__ __forceinline__ void prefetch_backsub(const Group<R>& G, int i, int n) {
    if ((threadIdx.x & 31) == 0 && n > 0) {  // lane 0's pointers carry no lane offset
        prefetch_l2(G.scr + (size_t)i * 3 * kLanes, (uint32_t)n * 3 * kLanes * sizeof(R));
        prefetch_l2(G.vbuf + (size_t)i * 2 * kLanes, (uint32_t)n * 2 * kLanes * sizeof(R));
    }
}

// L2 prefetch of the rows node n's channel update reads: states and parameters.
template <typename R>
__device__ __forceinline__ void prefetch_channels(const Group<R>& G, const NodeRec<R>& n) {
    if ((threadIdx.x & 31) == 0) {
        if (n.srows) prefetch_l2(G.slab + (size_t)n.srow * kLanes, n.srows * kLanes * sizeof(R));
        if (n.prows) prefetch_l2(G.ptab + (size_t)n.prow * kLanes, n.prows * kLanes * sizeof(float));
    }
}

// L2 prefetch of node n's state and parameter rows, one row per lane (the
// row's 128 bytes are one cache line; lane r's own element lies in row r).
template <typename R>
__device__ __forceinline__ void prefetch_rows_l2(const Group<R>& G, const NodeRec<R>& n) {
    const int r = threadIdx.x & 31;
    if (r < n.srows) asm volatile("prefetch.global.L2 [%0];" ::"l"(G.slab + (size_t)(n.srow + r) * kLanes));
    if (r < n.prows) asm volatile("prefetch.global.L2 [%0];" ::"l"(G.ptab + (size_t)(n.prow + r) * kLanes));
}

// A junction row: its FP64 sum with the chain carry and the accumulator of
// its far children, which is cleared for the next step.  Out of line, so
// that the other rows (most of them) do not issue this path predicated off.
template <typename R>
struct RowSum {
    R x, r;
};
template <typename R>
__device__ __forceinline__ RowSum<R> junction_sum(double* ja, R x0, R cx, R r0, R cr) {
    RowSum<R> o;
    o.x = (R)((double)x0 + (double)cx + ja[0]);
    o.r = (R)((double)r0 + (double)cr + ja[kLanes]);
    ja[0] = 0.0;
    ja[kLanes] = 0.0;
    return o;
}

// Elimination of a non-root node i given its (x, rhs, e); updates the chain
// carry or the parent's FP64 junction accumulator, writes (r, c).
template <typename R>
__device__ __forceinline__ void eliminate_node(const Group<R>& G, const NodeRec<R>& s, int i, R x0, R r0,
                                               R e0, R& carry_x, R& carry_r) {
    using M = Math<R>;
    R x, r;
    if (s.jslot >= 0) {
        const RowSum<R> j = junction_sum(G.jacc + (size_t)(2 * s.jslot) * kLanes, x0, carry_x, r0, carry_r);
        x = j.x;
        r = j.r;
    } else {
        x = x0 + carry_x;
        r = r0 + carry_r;
    }
    R* out = G.scr + (size_t)i * 3 * kLanes;
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

// Leaf -> root elimination of the node range [lo, hi).  row(i, x, rhs, e)
// supplies node i's assembled row: read back from scr (first step after
// init), or assembled on the spot from the node's channel update.
template <typename R, typename Row>
__device__ __forceinline__ void eliminate_range(const Group<R>& G, const NodeRec<R>* nr, int lo, int hi, Row&& row) {
    R carry_x = 0, carry_r = 0;
    for (int i = hi - 1; i >= lo; --i) {
        R x0, r0, e0;
        row(i, x0, r0, e0);
        eliminate_node(G, nr[i], i, x0, r0, e0, carry_x, carry_r);
    }
}

// Channel update of node i at its new voltage V (INIT: steady state at V),
// then the node's row for the next step: its excess x (the grounded
// conductance g + cm/dt), right-hand side, and e = b_i (V_p - V_i), the
// axial term of the parent's row.
template <typename R, int MS, bool INIT, typename Classes = NoClasses>
__device__ __forceinline__ void assemble_node(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>& n, int i,
                                              R V, R vp, R dt, R dtn_inv, R istim_amp, R& x, R& rhs, R& e) {
    R I, Gm;
    if constexpr (INIT) {
        channels<R, MS, true>((uint32_t)n.mask, V, dt, G.slab + (size_t)n.srow * kLanes, G.ptab + (size_t)n.prow * kLanes,
                              I, Gm);
    } else {
        const CurrentG<R> ig = channels_step<R, MS, Classes>(n.cls, n.mask, V, dt, G.slab + (size_t)n.srow * kLanes,
                                                   G.ptab + (size_t)n.prow * kLanes);
        I = ig.I;
        Gm = ig.G;
    }
    const R istim = (i == A.stim_node) ? istim_amp : (R)0;
    const R dvp = vp - V;
    x = Gm + n.cm * dtn_inv;
    rhs = istim - I - n.a * dvp;
    e = n.b * dvp;
}

template <typename R>
__device__ __forceinline__ void store_row(const Group<R>& G, int i, R x, R rhs, R e) {
    R* o = G.scr + (size_t)i * 3 * kLanes;
    o[0] = x;
    o[kLanes] = rhs;
    o[2 * kLanes] = e;
}

template <typename R>
__device__ __forceinline__ void record(const SimArgs<R>& A, const NodeRec<R>& n, R V, bool rec_now, float* trace) {
    if (rec_now && n.rec >= 0) trace[(size_t)n.rec * A.n_inst_pad] = (float)V;
}

// A voltage that is NaN, infinite or beyond 1e6 mV: the instance has blown up.
template <typename R>
__device__ __forceinline__ bool v_bad(R V) {
    return !(fabs(V) < (R)1e6);
}

// Back-substitution result x = dV_i of node i: V update (Kahan), dV for the
// node's far children, recording; bad is set when the new V is not finite.
template <typename R>
__device__ __forceinline__ void backsub_node(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>& n, int i,
                                             R x, bool rec_now, float* trace, int& bad) {
    R* vo = G.vbuf + (size_t)i * 2 * kLanes;
    R V = vo[0], vc = vo[kLanes];
    kahan_add(V, vc, x);
    vo[0] = V;
    vo[kLanes] = vc;
    if (n.jslot >= 0) G.jx[(size_t)n.jslot * kLanes] = x;
    record(A, n, V, rec_now, trace);
    bad |= v_bad(V);
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

// Segment item, leaf -> root elimination of the spine r..l-1 (after its
// light subtrees).  Each spine row also couples to the lower separator's dV
// (w: b_l of row l-1, then the fill-in carried up the spine), so its diagonal
// is x - a + w and the row solves as dV_i = r_i - c_i dV_parent + w_i dV_l
// (stored as (r, c, w) for the back-substitution).  The same sweep
// accumulates what separator l needs for the skeleton, dV_{l-1} = gamma +
// alpha dV_u + beta dV_l expanded down the spine: alpha (row l's coupling to
// u), gamma (its right-hand side) and delta = 1 - alpha - beta, the fraction
// of dV_{l-1} that leaks to ground along the spine, which becomes l's
// excess.  delta is summed from the rows' leak fractions x_i / d_i, never as
// 1 - alpha - beta.
template <typename R>
struct SpineCarry {
    R x, r, w;    // chain carries (excess, right-hand side, coupling to dV_l)
    R P, gam, del;  // P: product of -c over the rows below
    __device__ __forceinline__ void reset() {
        x = r = w = 0;
        P = 1;
        gam = del = 0;
    }
};

// One spine row i (rows are visited from b = l-1 down to r) with its row
// (x0, r0, e_i); e_l: the lower separator's parent-row axial term; sv: the
// segment link's rows (A, B, excess, rhs terms).
template <typename R>
__device__ __forceinline__ void eliminate_spine_row(const Group<R>& G, const NodeRec<R>& s, const NodeRec<R>& nl,
                                                    int i, int b, int r, R x0, R r0, R e_i, R e_l,
                                                    SpineCarry<R>& k, R* sv) {
    using M = Math<R>;
    R x, rh;
    if (s.jslot >= 0) {
        const RowSum<R> j = junction_sum(G.jacc + (size_t)(2 * s.jslot) * kLanes, x0, k.x, r0, k.r);
        x = j.x;
        rh = j.r;
    } else {
        x = x0 + k.x;
        rh = r0 + k.r;
    }
    R w = k.w;
    if (i == b) {
        w = -nl.b;
        rh += e_l;
    }
    const R inv = M::rc(x - s.a + w);
    const R rr = rh * inv, cc = s.a * inv, om = w * inv, lam = x * inv;
    R* out = G.scr + (size_t)i * 3 * kLanes;
    out[0] = rr;
    out[kLanes] = cc;
    out[2 * kLanes] = om;
    k.gam += rr * k.P;
    k.del += lam * k.P;
    k.P *= -cc;
    if (i > r) {
        k.x = -s.b * lam;
        k.r = e_i - s.b * rr;
        k.w = -s.b * om;
    } else {
        double* ja = G.jacc + (size_t)(2 * s.pslot) * kLanes;  // the upper separator
        atomicAdd(ja, (double)(-s.b * lam));
        atomicAdd(ja + kLanes, (double)(e_i - s.b * rr));
        sv[kLanes] = s.b * om;  // B: row u's coupling to dV_l
        sv[0] = nl.a * k.P;              // A: row l's coupling to dV_u (alpha = P)
        sv[2 * kLanes] = -nl.a * k.del;  // added to l's excess
        sv[3 * kLanes] = -nl.a * k.gam;  // added to rhs_l
    }
}

// The spine of segment c, from rows supplied by row(i, x, rhs, e).
template <typename R, typename Row>
__device__ __forceinline__ void eliminate_segment(const Group<R>& G, const NodeRec<R>* nr, const DevComp& c, R e_l,
                                                  Row&& row) {
    const NodeRec<R> nl = nr[c.l];
    SpineCarry<R> k;
    k.reset();
    R* sv = G.sepv + (size_t)c.lk * 4 * kLanes;
    for (int i = c.l - 1; i >= c.r; --i) {
        R x0, r0, e_i;
        row(i, x0, r0, e_i);
        eliminate_spine_row(G, nr[i], nl, i, c.l - 1, c.r, x0, r0, e_i, e_l, k, sv);
    }
}

// Warp-level work queue: lane 0 takes the next item, the warp shares it.
__device__ __forceinline__ int next_item(int* ctr) {
    int k = 0;
    if ((threadIdx.x & 31) == 0) k = atomicAdd(ctr, 1);
    return __shfl_sync(0xffffffffu, k, 0);
}

// Initial state of group g: channels at steady state for v_init, the first
// step's rows (nodes are independent here, so any number of warps shares
// them), sample 0; then every item's elimination for the first step, from
// the rows just stored, so that a launch of k_sim_advance starts on
// eliminated rows.  ctr: a shared-memory work counter.
template <typename R, int MS>
__device__ __forceinline__ void init_body(const SimArgs<R>& A, int g, int* ctr) {
    const Group<R> G = group_of(A, g);
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) *ctr = 0;
    if (w == 0)
        for (int j = 0; j < 2 * A.n_jslots; ++j) G.jacc[(size_t)j * kLanes] = 0.0;
    R dt, dtn_inv, istim_amp;
    bool rec_now;
    float* trace;
    step_inputs(A, G, 0, true, dt, dtn_inv, istim_amp, rec_now, trace);
    const R V = (R)A.v_init;
    for (int i = w; i < A.n_nodes; i += nw) {
        const NodeRec<R> n = A.nodes[i];
        R x, rhs, e;
        assemble_node<R, MS, true>(A, G, n, i, V, V, dt, dtn_inv, istim_amp, x, rhs, e);
        R* vo = G.vbuf + (size_t)i * 2 * kLanes;
        vo[0] = V;
        vo[kLanes] = 0;
        store_row(G, i, x, rhs, e);
        record(A, n, V, rec_now, trace);
    }
    if (w == 0) A.bad[G.inst] = 0;
    __syncthreads();
    auto row = [&](int i, R& x, R& rhs, R& e) {
        const R* o = G.scr + (size_t)i * 3 * kLanes;
        x = o[0];
        rhs = o[kLanes];
        e = o[2 * kLanes];
    };
    for (int k = next_item(ctr); k < A.n_comps; k = next_item(ctr)) {
        const DevComp c = A.comps[k];
        eliminate_range(G, A.nodes, c.lo, c.hi, row);
        if (c.l >= 0) eliminate_segment(G, A.nodes, c, G.scr[(size_t)c.l * 3 * kLanes + 2 * kLanes], row);
    }
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps) k_sim_init(SimArgs<R> A) {
    __shared__ int ctr;
    init_body<R, MS>(A, blockIdx.x, &ctr);
}

// Back-substitution pass of an item, root -> leaf: the spine of a segment
// (dV_i = r_i - c_i dV_parent + w_i dV_l, from separator u down), then the
// light nodes; V update of each node.  Rows are prefetched into L2 in
// blocks of four nodes, four nodes ahead.
// TI: thread-item layout (lanes on different items; no lane-0 prefetch).
// One node's back-substitution operands: its eliminated row (r, c; on a
// spine also w) and its voltage with the Kahan term.
template <typename R>
struct BackRow {
    R r, c, w, V, C;
};
template <typename R, bool SPINE>
__device__ __forceinline__ BackRow<R> load_back_row(const Group<R>& G, int i) {
    BackRow<R> b;
    const R* row = G.scr + (size_t)i * 3 * kLanes;
    const R* vo = G.vbuf + (size_t)i * 2 * kLanes;
    b.r = row[0];
    b.c = row[kLanes];
    b.w = SPINE ? row[2 * kLanes] : (R)0;
    b.V = vo[0];
    b.C = vo[kLanes];
    return b;
}

// The V update of node i from its loaded (V, Kahan term) and dV = x: store,
// dV for the node's far children, recording, non-finite check.
template <typename R>
__device__ __forceinline__ void backsub_store(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>& n, int i,
                                              R x, R V, R vc, bool rec_now, float* trace, int& bad) {
    R* vo = G.vbuf + (size_t)i * 2 * kLanes;
    kahan_add(V, vc, x);
    vo[0] = V;
    vo[kLanes] = vc;
    if (n.jslot >= 0) G.jx[(size_t)n.jslot * kLanes] = x;
    record(A, n, V, rec_now, trace);
    bad |= v_bad(V);
}

// Back-substitution pass of an item, root -> leaf: the spine of a segment
// (dV_i = r_i - c_i dV_parent + w_i dV_l, from separator u down), then the
// light nodes; V update of each node.  Software-pipelined one node deep: the
// next node's operands (row, V, Kahan term, and a far child's parent dV) are
// loaded before this node's update, so a node's memory latency overlaps the
// previous node's arithmetic and stores (no node writes what the next one
// reads: its own V and, for a junction, a dV its later children read).  Rows
// are also prefetched into L2 in blocks of four nodes, four nodes ahead.
// TI: thread-item layout (lanes on different items; no lane-0 prefetch).
template <typename R, bool TI = false>
__device__ __forceinline__ void backsub_item(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr,
                                             const DevComp& c, bool rec_now, float* trace, int& bad) {
    constexpr int kBlk = 4;
    if (c.l >= 0) {
        R xp = G.jx[(size_t)nr[c.u].jslot * kLanes];
        const R xl = G.jx[(size_t)nr[c.l].jslot * kLanes];
        if constexpr (!TI) prefetch_backsub(G, c.r, min(kBlk, c.l - c.r));
        BackRow<R> cur = load_back_row<R, true>(G, c.r);
        for (int i = c.r; i < c.l; ++i) {
            if constexpr (!TI)
                if (((i - c.r) & (kBlk - 1)) == 0) prefetch_backsub(G, i + kBlk, min(kBlk, c.l - i - kBlk));
            const BackRow<R> nxt = i + 1 < c.l ? load_back_row<R, true>(G, i + 1) : cur;
            const R xi = cur.r - cur.c * xp + cur.w * xl;
            xp = xi;
            backsub_store(A, G, nr[i], i, xi, cur.V, cur.C, rec_now, trace, bad);
            cur = nxt;
        }
    }
    if (c.hi <= c.lo) return;
    R x_prev = 0;
    if constexpr (!TI) prefetch_backsub(G, c.lo, min(kBlk, c.hi - c.lo));
    NodeRec<R> n = nr[c.lo];
    BackRow<R> cur = load_back_row<R, false>(G, c.lo);
    R xj = n.pslot < 0 ? (R)0 : G.jx[(size_t)n.pslot * kLanes];
    for (int i = c.lo; i < c.hi; ++i) {
        if constexpr (!TI)
            if (((i - c.lo) & (kBlk - 1)) == 0) prefetch_backsub(G, i + kBlk, min(kBlk, c.hi - i - kBlk));
        // the next node: its parent is this node (a chain child, pslot < 0)
        // or an earlier one, whose dV is already stored
        NodeRec<R> nn = n;
        BackRow<R> nxt = cur;
        R xjn = 0;
        if (i + 1 < c.hi) {
            nn = nr[i + 1];
            nxt = load_back_row<R, false>(G, i + 1);
            if (nn.pslot >= 0) xjn = G.jx[(size_t)nn.pslot * kLanes];
        }
        const R xp = n.pslot < 0 ? x_prev : xj;
        const R x = cur.r - cur.c * xp;
        x_prev = x;
        backsub_store(A, G, n, i, x, cur.V, cur.C, rec_now, trace, bad);
        n = nn;
        cur = nxt;
        xj = xjn;
    }
}

// Channel pass of an item, leaf -> root: each node's channel update at its
// new V and its next-step row, which is eliminated at once (children come
// first in this order), so assembled rows stay in registers.  One loop
// visits, in this order, the light nodes hi-1 .. lo, the separator sep (a
// segment's lower separator, or a separator linked directly to the
// skeleton: its row goes to the skeleton), and, for a segment (lk >= 0),
// the spine sep-1 .. r.  Every channel update of a step goes through this
// one loop, so the channel code is inlined once.
template <typename R, int MS, typename Classes, bool TI = false>
__device__ __forceinline__ void channels_item(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr,
                                              int lo, int hi, int sep, int r, int lk, R dt, R dtn_inv,
                                              R istim_amp) {
    const int n_light = hi - lo;
    const int n_sep = n_light + (sep >= 0 ? 1 : 0);
    const int n = n_sep + (lk >= 0 ? sep - r : 0);
    const int b = sep - 1;
    auto node_at = [&](int p) { return p < n_light ? hi - 1 - p : (p < n_sep ? sep : b - (p - n_sep)); };
    NodeRec<R> nl;
    R* sv = nullptr;
    if (lk >= 0) {
        nl = nr[sep];
        sv = G.sepv + (size_t)lk * 4 * kLanes;
    }
    SpineCarry<R> k;
    k.reset();
    R e_l = 0;
    constexpr bool pf = NGPU_CH_PREFETCH != 0 && !TI;
    // Without the bulk prefetch (models whose nodes read few rows), a node's
    // loads are started one node early instead: its voltages (its own and
    // its parent's; the pass writes no voltage) into registers, its state and
    // parameter rows into L2 (one prefetch per row, lane r taking row r).
    // Either alone measured slower on B200 (the node still waits for the
    // other); both together, 2.7 % faster on the TTPC-like cell.  Models with
    // the bulk prefetch keep the register budget for their channel code.
    constexpr bool ahead = NGPU_CH_AHEAD != 0 && !pf && !TI;
    if (pf && n > 0) prefetch_channels(G, nr[node_at(0)]);
    if (pf && n > 1) prefetch_channels(G, nr[node_at(1)]);
    int vi = -1;  // node whose V was read last as a parent voltage (!ahead)
    R vv = 0;
    int i_nx = 0;  // the next node and its voltages (ahead)
    R v_nx = 0, vp_nx = 0;
    if (ahead && n > 0) {
        i_nx = node_at(0);
        v_nx = G.vbuf[(size_t)i_nx * 2 * kLanes];
        vp_nx = i_nx == 0 ? v_nx : G.vbuf[(size_t)nr[i_nx].parent * 2 * kLanes];
    }
    for (int p = 0; p < n; ++p) {
        const int i = ahead ? i_nx : node_at(p);
        const NodeRec<R> nd = nr[i];
        if (pf && p + 2 < n) prefetch_channels(G, nr[node_at(p + 2)]);
        R V, vp;
        if constexpr (ahead) {
            V = v_nx;
            vp = vp_nx;
            if (p + 1 < n) {
                i_nx = node_at(p + 1);
                const NodeRec<R>& nn = nr[i_nx];
                v_nx = i_nx == nd.parent ? vp : G.vbuf[(size_t)i_nx * 2 * kLanes];
                vp_nx = i_nx == 0 ? v_nx : G.vbuf[(size_t)nn.parent * 2 * kLanes];
                prefetch_rows_l2(G, nn);
            }
        } else {
            if (vi == i) V = vv;
            else V = G.vbuf[(size_t)i * 2 * kLanes];
            vp = i == 0 ? V : G.vbuf[(size_t)nd.parent * 2 * kLanes];
            vi = nd.parent;
            vv = vp;
        }
        R x, rhs, e;
        assemble_node<R, MS, false, Classes>(A, G, nd, i, V, vp, dt, dtn_inv, istim_amp, x, rhs, e);
        if (p < n_light) {
            eliminate_node(G, nd, i, x, rhs, e, k.x, k.r);
        } else if (p < n_sep) {
            store_row(G, i, x, rhs, e);
            e_l = e;
            k.reset();
        } else {
            eliminate_spine_row(G, nd, nl, i, b, r, x, rhs, e, e_l, k, sv);
        }
    }
}

// S2 through shared memory.  Every warp stages a share of the separators
// at once (their accumulated rows, couplings and voltages: one memory round
// trip for all of them), then warp 0 runs the skeleton's elimination and
// back-substitution on the staged rows, where each separator's dependence
// on its children goes through shared memory instead of a global
// read-modify-write, and writes back dV and V.
template <typename R>
__device__ __forceinline__ void skeleton_staged(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr,
                                                char* smem, bool rec_now, float* trace, int& bad) {
    using M = Math<R>;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int S = A.n_seps;
    double* acx = (double*)(smem + SmemPlan<R>::nodes(A.n_nodes));
    double* acr = acx + (size_t)S * kLanes;
    R* sA = (R*)(acr + (size_t)S * kLanes);
    R* sB = sA + (size_t)S * kLanes;
    R* sE = sB + (size_t)S * kLanes;
    R* sV = sE + (size_t)S * kLanes;
    R* sC = sV + (size_t)S * kLanes;
    for (int k = w; k < S; k += nw) {
        const DevSep sp = A.seps[k];
        const NodeRec<R> s = nr[sp.node];
        const R* row = G.scr + (size_t)sp.node * 3 * kLanes;
        double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
        const R* vo = G.vbuf + (size_t)sp.node * 2 * kLanes;
        double x = (double)row[0] + ja[0], rh = (double)row[kLanes] + ja[kLanes];
        R a = s.a, b = s.b, e = row[2 * kLanes];
        if (sp.seg >= 0) {
            const R* sv = G.sepv + (size_t)k * 4 * kLanes;
            a = sv[0];
            b = sv[kLanes];
            x += (double)sv[2 * kLanes];
            rh += (double)sv[3 * kLanes];
            e = 0;  // the segment already folded this node's axial term in
        }
        ja[0] = 0.0;
        ja[kLanes] = 0.0;
        const size_t o = (size_t)k * kLanes + lane;
        acx[o] = x;
        acr[o] = rh;
        sA[o] = a;
        sB[o] = b;
        sE[o] = e;
        sV[o] = vo[0];
        sC[o] = vo[kLanes];
    }
    __syncthreads();
    if (w != 0) return;
    for (int k = S - 1; k >= 0; --k) {
        const size_t o = (size_t)k * kLanes + lane;
        const R x = (R)acx[o], rh = (R)acr[o];
        if (k == 0) {
            sB[o] = M::dv(rh, x);
            break;
        }
        const R Acp = sA[o], Bcp = sB[o], e_up = sE[o];
        const R inv = M::rc(x - Acp);
        const R rr = rh * inv, cc = Acp * inv;
        sA[o] = cc;
        sB[o] = rr;
        const size_t op = (size_t)A.seps[k].par * kLanes + lane;
        acx[op] += (double)(-Bcp * (x * inv));
        acr[op] += (double)(e_up - Bcp * rr);
    }
    for (int k = 0; k < S; ++k) {
        const DevSep sp = A.seps[k];
        const NodeRec<R> s = nr[sp.node];
        const size_t o = (size_t)k * kLanes + lane;
        const R x = k == 0 ? sB[o] : sB[o] - sA[o] * sE[(size_t)sp.par * kLanes + lane];
        sE[o] = x;
        G.jx[(size_t)s.jslot * kLanes] = x;
        R* vo = G.vbuf + (size_t)sp.node * 2 * kLanes;
        R V = sV[o], vc = sC[o];
        kahan_add(V, vc, x);
        vo[0] = V;
        vo[kLanes] = vc;
        record(A, s, V, rec_now, trace);
        bad |= v_bad(V);
    }
}

// Work item k of a step: an item's back-substitution pass, then its channel
// pass; k >= n_comps: a separator linked directly to the skeleton (its
// channel update and its row for the skeleton solve).
template <typename R, int MS, typename Classes, bool TI>
__device__ __forceinline__ void run_item(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr, int k,
                                         R dt, R dtn_inv, R istim_amp, bool rec_now, float* trace, int& bad) {
    int lo = 0, hi = 0, sep = -1, r = 0, lk = -1;
    if (k < A.n_comps) {
        const DevComp c = A.comps[k];
        backsub_item<R, TI>(A, G, nr, c, rec_now, trace, bad);
        lo = c.lo;
        hi = c.hi;
        sep = c.l;
        r = c.r;
        lk = c.lk;
    } else {
        const DevSep sp = A.seps[k - A.n_comps];
        if (sp.seg < 0) sep = sp.node;  // separators ending a segment are their segment's
    }
    channels_item<R, MS, Classes, TI>(A, G, nr, lo, hi, sep, r, lk, dt, dtn_inv, istim_amp);
}

// Per timestep (two barriers, three with a staged skeleton):
//   S2  warp 0 solves the skeleton (the separators, a few dozen nodes) with
//       the reduced couplings of the segments, and updates (and records)
//       their V; staged (skeleton_staged), all warps first load its rows
//   S3  all warps take items from a queue, largest first: an item's
//       back-substitution pass, then its channel pass (channel update,
//       next-step assembly and elimination node by node, above); each
//       item's contribution to its upper separator goes to that
//       separator's FP64 accumulator.  Separators linked directly to the
//       skeleton are items too (channel update and row for S2).
// Between launches the rows are eliminated (k_sim_init eliminates the first
// step's rows), so a run split into several launches performs the same
// operations as one launch.  n_steps timesteps of group g; the items are
// shared by however many warps the CTA has (the split was sized for
// A.n_warps).
template <typename R, int MS, typename Classes>
__device__ __forceinline__ void advance_body(const SimArgs<R>& A, int g, int t0, int n_steps, char* smem,
                                             int* ctr) {
    const Group<R> G = group_of(A, g);
    const int w = threadIdx.x >> 5;
    const NodeRec<R>* nr = stage_nodes(A, smem);
    if (threadIdx.x == 0) { ctr[0] = 0; ctr[1] = 0; }
    __syncthreads();
    int bad = 0;
    const int n_items = A.n_comps + A.n_seps;
    for (int t = t0; t < t0 + n_steps; ++t) {
        // this step's queue is ctr[t & 1]; the other counter was last used
        // by the previous step's queue, which the barrier ended
        int* const q = &ctr[t & 1];
        if (threadIdx.x == 0) ctr[(t + 1) & 1] = 0;
        R dt, dtn_inv, istim_amp;
        bool rec_now;
        float* trace;
        step_inputs(A, G, t, false, dt, dtn_inv, istim_amp, rec_now, trace);
        // S2: skeleton
        if (A.s2_stage) {
            skeleton_staged<R>(A, G, nr, smem, rec_now, trace, bad);
        } else if (w == 0) {
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
                record(A, s, V, rec_now, trace);
                bad |= v_bad(V);
            }
        }
        __syncthreads();
        // S3: items
        for (int k = next_item(q); k < n_items; k = next_item(q))
            run_item<R, MS, Classes, false>(A, G, nr, k, dt, dtn_inv, istim_amp, rec_now, trace, bad);
        __syncthreads();
    }
    // any warp that saw a non-finite voltage of this group's instance (lane)
    if (bad) A.bad[G.inst] = 1;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps, NGPU_ADV_MIN_BLOCKS) k_sim_advance(SimArgs<R> A, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    __shared__ int ctr[2];
    advance_body<R, MS, NoClasses>(A, blockIdx.x, t0, n_steps, smem, ctr);
}

// ---------------------------------------------------------------------------
// Thread-item layout, for batches too small to fill the GPU 32 instances per
// CTA: one warp per instance, a CTA holds blockDim.x / 32 instances.
//
// The instance's tree is split for the warp's 32 lanes (make_partition with
// 32 units): every lane takes work items from the warp's queue in
// shared memory, largest first, and runs on each the same two passes as the
// layout above; lane 0 solves the skeleton from shared memory between
// __syncwarp()s, the other lanes load and write back its rows.  Storage and
// its [group][row][32 lanes] layout are those of the lane-instance layout
// (one simulation's buffers, traces and features serve both): a lane touches
// its instance's element of each row, four bytes, which the L1 and L2 serve
// well at the batch sizes this layout is for.  The channel code is the same
// inlined call site; lanes on nodes of different mechanism classes take
// turns through it.

// S2 of one instance (warp): staged rows, lane 0's serial elimination and
// back-substitution over the separators, all lanes' write-back.
template <typename R>
__device__ __forceinline__ void skeleton_ti(const SimArgs<R>& A, const Group<R>& G, const NodeRec<R>* nr,
                                            char* st, bool rec_now, float* trace, int& bad) {
    using M = Math<R>;
    const int lane = threadIdx.x & 31;
    const int S = A.n_seps;
    double* acx = (double*)st;
    double* acr = acx + S;
    R* sA = (R*)(acr + S);
    R* sB = sA + S;
    R* sE = sB + S;
    R* sV = sE + S;
    R* sC = sV + S;
    for (int k = lane; k < S; k += kLanes) {
        const DevSep sp = A.seps[k];
        const NodeRec<R> s = nr[sp.node];
        const R* row = G.scr + (size_t)sp.node * 3 * kLanes;
        double* ja = G.jacc + (size_t)(2 * s.jslot) * kLanes;
        const R* vo = G.vbuf + (size_t)sp.node * 2 * kLanes;
        double x = (double)row[0] + ja[0], rh = (double)row[kLanes] + ja[kLanes];
        R a = s.a, b = s.b, e = row[2 * kLanes];
        if (sp.seg >= 0) {
            const R* sv = G.sepv + (size_t)k * 4 * kLanes;
            a = sv[0];
            b = sv[kLanes];
            x += (double)sv[2 * kLanes];
            rh += (double)sv[3 * kLanes];
            e = 0;  // the segment already folded this node's axial term in
        }
        ja[0] = 0.0;
        ja[kLanes] = 0.0;
        acx[k] = x;
        acr[k] = rh;
        sA[k] = a;
        sB[k] = b;
        sE[k] = e;
        sV[k] = vo[0];
        sC[k] = vo[kLanes];
    }
    __syncwarp();
    if (lane == 0) {
        for (int k = S - 1; k >= 0; --k) {
            const R x = (R)acx[k], rh = (R)acr[k];
            if (k == 0) {
                sB[0] = M::dv(rh, x);
                break;
            }
            const R Acp = sA[k], Bcp = sB[k], e_up = sE[k];
            const R inv = M::rc(x - Acp);
            const R rr = rh * inv, cc = Acp * inv;
            sA[k] = cc;
            sB[k] = rr;
            const int p = A.seps[k].par;
            acx[p] += (double)(-Bcp * (x * inv));
            acr[p] += (double)(e_up - Bcp * rr);
        }
        for (int k = 0; k < S; ++k) sE[k] = k == 0 ? sB[0] : sB[k] - sA[k] * sE[A.seps[k].par];
    }
    __syncwarp();
    for (int k = lane; k < S; k += kLanes) {
        const DevSep sp = A.seps[k];
        const NodeRec<R> s = nr[sp.node];
        const R x = sE[k];
        G.jx[(size_t)s.jslot * kLanes] = x;
        R* vo = G.vbuf + (size_t)sp.node * 2 * kLanes;
        R V = sV[k], vc = sC[k];
        kahan_add(V, vc, x);
        vo[0] = V;
        vo[kLanes] = vc;
        record(A, s, V, rec_now, trace);
        bad |= v_bad(V);
    }
    __syncwarp();
}

// n_steps timesteps of instance blockIdx.x * (blockDim.x / 32) + warp.
// q: [warps][2] shared-memory queue counters.
template <typename R, int MS, typename Classes>
__device__ __forceinline__ void advance_body_ti(const SimArgs<R>& A, int t0, int n_steps, char* smem, int* q) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const NodeRec<R>* nr = stage_nodes(A, smem);  // the CTA's only block-wide barrier
    const int inst = blockIdx.x * nw + w;
    if (inst >= A.n_inst) return;
    const Group<R> G = group_lane(A, inst / kLanes, inst % kLanes);
    char* st = smem + SmemPlan<R>::nodes(A.n_nodes) + (size_t)w * SmemPlan<R>::ti_stage(A.n_seps);
    int* const qw = q + 2 * w;
    if (lane == 0) {
        qw[0] = 0;
        qw[1] = 0;
    }
    __syncwarp();
    int bad = 0;
    const int n_items = A.n_comps + A.n_seps;
    for (int t = t0; t < t0 + n_steps; ++t) {
        // this step's queue is qw[t & 1]; the other was last used by the
        // previous step's queue, which the warp barrier ended
        int* const qs = &qw[t & 1];
        if (lane == 0) qw[(t + 1) & 1] = 0;
        R dt, dtn_inv, istim_amp;
        bool rec_now;
        float* trace;
        step_inputs(A, G, t, false, dt, dtn_inv, istim_amp, rec_now, trace);
        skeleton_ti<R>(A, G, nr, st, rec_now, trace, bad);
        for (int k = atomicAdd(qs, 1); k < n_items; k = atomicAdd(qs, 1))
            run_item<R, MS, Classes, true>(A, G, nr, k, dt, dtn_inv, istim_amp, rec_now, trace, bad);
        __syncwarp();
    }
    if (bad) A.bad[G.inst] = 1;
}

// The thread-item layout runs small batches (a few warps per SM at most):
// registers are plentiful, so the kernel is compiled for 2 CTAs per SM.
#ifndef NGPU_TI_MIN_BLOCKS
#define NGPU_TI_MIN_BLOCKS 2
#endif
template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps, NGPU_TI_MIN_BLOCKS)
    k_sim_advance_ti(SimArgs<R> A, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    __shared__ int q[2 * kMaxWarps];
    advance_body_ti<R, MS, NoClasses>(A, t0, n_steps, smem, q);
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
    __shared__ int ctr;
    const int k = batch_member(B.cta0, B.n);
    init_body<R, MS>(B.sim[k], blockIdx.x - B.cta0[k], &ctr);
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes * kMaxWarps, NGPU_ADV_MIN_BLOCKS)
    k_batch_advance(const __grid_constant__ BatchArgs<R> B, int t0, int n_steps) {
    extern __shared__ __align__(128) char smem[];
    __shared__ int ctr[2];
    const int k = batch_member(B.cta0, B.n);
    advance_body<R, MS, NoClasses>(B.sim[k], blockIdx.x - B.cta0[k], t0, n_steps, smem, ctr);
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

// Per parameter-table row: the smallest and largest bit pattern over every
// instance (equal: one value, the same bits, in every parameter set).
__global__ void __launch_bounds__(256) k_ptab_range(const float* __restrict__ ptab, int ptab_rows, int n_groups,
                                                    uint2* __restrict__ out) {
    __shared__ unsigned lo_s[8], hi_s[8];
    const int row = blockIdx.x;
    unsigned lo = 0xFFFFFFFFu, hi = 0u;
    for (int t = threadIdx.x; t < n_groups * kLanes; t += blockDim.x) {
        const unsigned b = __float_as_uint(ptab[((size_t)(t >> 5) * ptab_rows + row) * kLanes + (t & 31)]);
        lo = min(lo, b);
        hi = max(hi, b);
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0) {
        lo_s[threadIdx.x >> 5] = lo;
        hi_s[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = min(lo, lo_s[w]);
            hi = max(hi, hi_s[w]);
        }
        out[row] = make_uint2(lo, hi);
    }
}

// Per parameter-table row: a hash of its values at every instance (the sum
// of a 64-bit mix of each (instance, bit pattern) pair: position-aware and
// independent of the summation order).  Equal rows hash alike; rows that
// hash alike are compared exactly (k_ptab_blocks_equal) before they share.
__device__ __forceinline__ uint64_t ptab_mix(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    return x ^ (x >> 33);
}

__global__ void __launch_bounds__(256) k_ptab_hash(const float* __restrict__ ptab, int ptab_rows, int n_groups,
                                                   unsigned long long* __restrict__ out) {
    __shared__ unsigned long long part[8];
    const int row = blockIdx.x;
    unsigned long long h = 0;
    for (int t = threadIdx.x; t < n_groups * kLanes; t += blockDim.x) {
        const unsigned b = __float_as_uint(ptab[((size_t)(t >> 5) * ptab_rows + row) * kLanes + (t & 31)]);
        h += ptab_mix(((uint64_t)t << 32) | b);
    }
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) h += part[w];
        out[row] = h;
    }
}

// pairs[k] = (first row of block a, first row of block b, rows): same[k] = 1
// when the two blocks hold the same bits at every instance, else 0
__global__ void __launch_bounds__(256) k_ptab_blocks_equal(const float* __restrict__ ptab, int ptab_rows,
                                                           int n_groups, const int3* __restrict__ pairs,
                                                           int* __restrict__ same) {
    const int3 pr = pairs[blockIdx.x];
    int diff = 0;
    for (int r = 0; r < pr.z && !diff; ++r)
        for (int t = threadIdx.x; t < n_groups * kLanes; t += blockDim.x) {
            const size_t g = (size_t)(t >> 5) * ptab_rows;
            const unsigned x = __float_as_uint(ptab[(g + pr.x + r) * kLanes + (t & 31)]);
            const unsigned y = __float_as_uint(ptab[(g + pr.y + r) * kLanes + (t & 31)]);
            diff |= x != y;
        }
    diff = __syncthreads_or(diff);
    if (threadIdx.x == 0) same[blockIdx.x] = !diff;
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
