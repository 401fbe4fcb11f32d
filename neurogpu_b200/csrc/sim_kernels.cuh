// Fused multi-compartment simulation kernels (thread-per-instance layout).
//
// One warp advances 32 instances (parameter set x stimulus) through every
// timestep.  All lanes of a warp always work on the same node, so the
// per-node mechanism branches are warp-uniform and every state / parameter /
// scratch access is one coalesced 128-byte row (structure of arrays with the
// instance index innermost).  Per timestep the warp makes two sweeps over the
// tree in Hines order (parent < child), which is the reference's per-step
// algorithm (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/CudaStuff.cu:227-330):
//
//   sweep A, leaf -> root (nodes N-1 .. 0):  Gaussian elimination of the
//     tree matrix (the reference's BeforeLU, CudaStuff.cu:31-69).  A chain
//     child passes its elimination term to node i-1 in registers; a child
//     whose parent is not i-1 (a branch junction) adds it to an FP64
//     junction accumulator of the parent.
//   sweep B, root -> leaf (nodes 0 .. N-1):  back-substitution (BkSub,
//     CudaStuff.cu:72-104), V += dV with Kahan compensation, cnexp channel
//     state update at the new V (nrn_state, CudaStuff.cu:324-326), then the
//     channel currents at the new V (nrn_current of the NEXT step,
//     CudaStuff.cu:262-267) and the assembly of the next step's diagonal and
//     right-hand side (CudaStuff.cu:268-291).
//
// Storage per group of 32 instances (rows of 32 elements, one per lane):
//   slab   rows per node: V, Kahan term, then the node's channel states
//   ptab   parameter rows per distinct (section, mechanism set) pair
//   scr    2 rows per node: (d, rhs) after sweep B, (dV/rhs', coupling) after A
//   jacc   FP64 (d, rhs) accumulators of junction parents
//   jx     (dV, V) of junction parents for their far children in sweep B
#pragma once
#include "channels_mainen.cuh"
#include "channels_ttpc.cuh"
#include "ngpu_math.cuh"

namespace ngpu {

constexpr int kLanes = 32;

struct NodeInfo {
    int32_t parent;  // -1 for the root
    uint32_t mask;   // mechanism bits
    int32_t srow;    // slab row of V (Kahan term at +1, states from +2)
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
struct SimArgs {
    const NodeInfo* info;
    const NodeCoef<R>* coef;
    int n_nodes;
    R* slab;
    int slab_rows;
    const float* ptab;
    int ptab_rows;
    R* scr;
    double* jacc;
    R* jx;
    int n_jslots;
    const float* amps;   // [n_stim][nt]
    const float* dts;    // [nt]
    int nt;
    int stim_node;
    float stim_scale;    // 100 / area (nA/um2 -> mA/cm2)
    const int* inst_stim;  // [n_inst_pad]
    float* trace;        // [n_samples][n_rec][n_inst_pad]
    int n_rec;
    int rec_every;
    int n_inst_pad;
    float v_init;
    int* bad;            // [n_inst_pad] non-finite voltage flags
};

template <typename R, int MS, bool INIT>
__device__ __forceinline__ void channels(uint32_t mk, R v, R dt, R* st, const float* pr, R& I,
                                         R& G) {
    if constexpr (MS == 0) ttpc_node<R, INIT>(mk, v, dt, st, pr, I, G);
    else mainen_node<R, INIT>(mk, v, dt, st, pr, I, G);
}

// v + x with the running compensation c (Kahan); explicit round-to-nearest
// intrinsics keep the compiler from re-associating the correction away.
__device__ __forceinline__ void kahan_add(float& v, float& c, float x) {
    float y = __fsub_rn(x, c);
    float t = __fadd_rn(v, y);
    c = __fsub_rn(__fsub_rn(t, v), y);
    v = t;
}
__device__ __forceinline__ void kahan_add(double& v, double& c, double x) { v += x; (void)c; }

// Sweep A: leaf -> root elimination for the current step.
template <typename R>
__device__ __forceinline__ void sweep_eliminate(const SimArgs<R>& A, R* __restrict__ scr,
                                                double* __restrict__ jacc) {
    using M = Math<R>;
    const int N = A.n_nodes;
    R carry_d = 0, carry_r = 0;
    for (int i = N - 1; i >= 0; --i) {
        const NodeInfo ni = A.info[i];
        const NodeCoef<R> c = A.coef[i];
        R* s = scr + (size_t)(2 * i) * kLanes;
        R d, r;
        if (ni.jslot >= 0) {
            double* ja = jacc + (size_t)(2 * ni.jslot) * kLanes;
            d = (R)((double)s[0] + (double)carry_d + ja[0]);
            r = (R)((double)s[kLanes] + (double)carry_r + ja[kLanes]);
            ja[0] = 0.0;
            ja[kLanes] = 0.0;
        } else {
            d = s[0] + carry_d;
            r = s[kLanes] + carry_r;
        }
        if (i == 0) {  // root: dV_0 = rhs_0 / d_0
            s[0] = M::dv(r, d);
            s[kLanes] = 0;
            break;
        }
        const R inv = M::rc(d);
        const R rr = r * inv, cc = c.a * inv;  // dV_i = rr - cc * dV_parent
        s[0] = rr;
        s[kLanes] = cc;
        const R cd = -c.b * cc, cr = -c.b * rr;
        if (ni.pslot < 0) {
            carry_d = cd;
            carry_r = cr;
        } else {
            double* ja = jacc + (size_t)(2 * ni.pslot) * kLanes;
            ja[0] += (double)cd;
            ja[kLanes] += (double)cr;
            carry_d = 0;
            carry_r = 0;
        }
    }
}

// Sweep B: root -> leaf.  INIT: V := v_init, steady-state channels, and the
// matrix of step 0.  Otherwise: apply step t's solution, update channels
// over dt_t, assemble step t+1.
template <typename R, int MS, bool INIT>
__device__ __forceinline__ void sweep_update(const SimArgs<R>& A, int t, int inst, R* __restrict__ slab,
                                             const float* __restrict__ ptab, R* __restrict__ scr,
                                             double* __restrict__ jacc, R* __restrict__ jx,
                                             int& bad) {
    const int N = A.n_nodes;
    const int tn = INIT ? 0 : t + 1;
    const int tnc = tn < A.nt ? tn : A.nt - 1;
    const R dt = INIT ? (R)0 : (R)A.dts[t];
    const R dtn_inv = (R)1 / (R)A.dts[tnc];
    const int stim = A.inst_stim[inst];
    const R istim_amp = (R)A.stim_scale * (R)A.amps[(size_t)stim * A.nt + tnc];
    const bool rec_now = tn < A.nt && (tn % A.rec_every) == 0;
    float* trace = A.trace + (size_t)(tn / A.rec_every) * A.n_rec * A.n_inst_pad + inst;
    R x_prev = 0, v_prev = 0, d_pend = 0, r_pend = 0;
    for (int i = 0; i < N; ++i) {
        const NodeInfo ni = A.info[i];
        const NodeCoef<R> c = A.coef[i];
        R* sv = slab + (size_t)ni.srow * kLanes;
        R* s = scr + (size_t)(2 * i) * kLanes;
        R V, x = 0;
        if (INIT) {
            V = (R)A.v_init;
            sv[0] = V;
            sv[kLanes] = 0;
        } else {
            const R rr = s[0], cc = s[kLanes];
            const R xp = (i == 0) ? (R)0 : (ni.pslot < 0 ? x_prev : jx[(size_t)(2 * ni.pslot) * kLanes]);
            x = rr - cc * xp;
            V = sv[0];
            R vc = sv[kLanes];
            kahan_add(V, vc, x);
            sv[0] = V;
            sv[kLanes] = vc;
        }
        const R vp = (i == 0) ? V : (ni.pslot < 0 ? v_prev : jx[(size_t)(2 * ni.pslot + 1) * kLanes]);
        if (ni.jslot >= 0) {
            jx[(size_t)(2 * ni.jslot) * kLanes] = x;
            jx[(size_t)(2 * ni.jslot + 1) * kLanes] = V;
        }
        R I, G;
        channels<R, MS, INIT>(ni.mask, V, dt, sv + 2 * kLanes, ptab + (size_t)ni.prow * kLanes, I, G);
        const R istim = (i == A.stim_node) ? istim_amp : (R)0;
        const R d = G + c.cm * dtn_inv + c.dconst;
        const R dvp = vp - V;
        const R rhs = istim - I - c.a * dvp;
        if (i > 0) {
            if (ni.pslot < 0) r_pend += c.b * dvp;
            else jacc[(size_t)(2 * ni.pslot + 1) * kLanes] += (double)(c.b * dvp);
            R* sp = s - 2 * kLanes;
            sp[0] = d_pend;
            sp[kLanes] = r_pend;
        }
        d_pend = d;
        r_pend = rhs;
        if (rec_now && ni.rec >= 0) trace[(size_t)ni.rec * A.n_inst_pad] = (float)V;
        if (i == 0 && !(fabs(V) < (R)1e6)) bad = 1;  // catches NaN / Inf / blow-up
        x_prev = x;
        v_prev = V;
    }
    R* sl = scr + (size_t)(2 * (N - 1)) * kLanes;
    sl[0] = d_pend;
    sl[kLanes] = r_pend;
}

template <typename R>
struct GroupPtrs {
    R* slab;
    const float* ptab;
    R* scr;
    double* jacc;
    R* jx;
    int inst;
};

template <typename R>
__device__ __forceinline__ GroupPtrs<R> group_ptrs(const SimArgs<R>& A) {
    const int g = blockIdx.x, lane = threadIdx.x;
    GroupPtrs<R> p;
    p.slab = A.slab + (size_t)g * A.slab_rows * kLanes + lane;
    p.ptab = A.ptab + (size_t)g * A.ptab_rows * kLanes + lane;
    p.scr = A.scr + (size_t)g * 2 * A.n_nodes * kLanes + lane;
    p.jacc = A.jacc + (size_t)g * 2 * A.n_jslots * kLanes + lane;
    p.jx = A.jx + (size_t)g * 2 * A.n_jslots * kLanes + lane;
    p.inst = g * kLanes + lane;
    return p;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes) k_sim_init(SimArgs<R> A) {
    GroupPtrs<R> p = group_ptrs(A);
    for (int j = 0; j < 2 * A.n_jslots; ++j) p.jacc[(size_t)j * kLanes] = 0.0;
    int bad = 0;
    sweep_update<R, MS, true>(A, 0, p.inst, p.slab, p.ptab, p.scr, p.jacc, p.jx, bad);
    A.bad[p.inst] = bad;
}

template <typename R, int MS>
__global__ void __launch_bounds__(kLanes) k_sim_advance(SimArgs<R> A, int t0, int n_steps) {
    GroupPtrs<R> p = group_ptrs(A);
    int bad = 0;
    for (int t = t0; t < t0 + n_steps; ++t) {
        sweep_eliminate(A, p.scr, p.jacc);
        sweep_update<R, MS, false>(A, t, p.inst, p.slab, p.ptab, p.scr, p.jacc, p.jx, bad);
    }
    if (bad) A.bad[p.inst] = 1;
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
