/*
 * CPU oracle for the NeuroGPU multi-compartment simulation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is loaded by
 * tests/, by __graft_entry__.smoke() and by the cpu_baseline / reference arm
 * of bench.py.  The product (neurogpu_b200) never links or calls it.
 *
 * It restates, in plain C, the per-timestep algorithm of the reference's
 * fused simulation kernel (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/
 * CudaStuff.cu:142-335, runSimulation) and its Hines solve (BeforeLU
 * :31-69, BkSub :72-104), together with the channel equations of the two
 * generated channel libraries the reference ships:
 *   - TTPC set (13 mechanisms): GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/
 *     AllModels.cu:66-516
 *   - Mainen set (9 mechanisms): Figures/FigureS4_mainen/CParsed/
 *     AllModels.cu:92-383
 *
 * The file is compiled twice: with ONG_REAL=double (the FP64 ground truth,
 * symbols suffixed _f64) and ONG_REAL=float (symbols suffixed _f32).
 */
#ifndef NGPU_ORACLE_H
#define NGPU_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ONG_MECHSET_TTPC = 0, ONG_MECHSET_MAINEN = 1 };

/* Tree in Hines order: parent[i] < i for i > 0, parent[0] = -1.
 * Row i of the node matrix reads  d_i x_i + a_i x_parent(i) + sum_c b_c x_c.
 * a = the reference's "f" (Fmatrix column A), b = its "e" (column B). */
typedef struct {
    int n_nodes;
    const int *parent;
    const double *a;
    const double *b;
    const double *cm;            /* uF/cm2 */
    const int *section;          /* node -> section (the reference's SegToComp) */
    int n_sections;
    int mechset;                 /* ONG_MECHSET_* */
    const unsigned char *mech_mask; /* [n_mech][n_nodes], the reference's boolModel */
} ong_model;

/* Flags. */
#define ONG_FLAG_FD_CONDUCTANCE 1  /* g from (I(v+0.001)-I(v))/0.001 as the reference (default on) */

/*
 * Simulate n_sets parameter sets x n_stim stimuli for nt steps.
 *   params  [n_sets][n_params][n_sections]  float, reference AllParams layout
 *   amps    [n_stim][nt] nA; dts [nt] ms (the reference's times.csv)
 *   out     [n_sets][n_stim][n_rec][nt]: V at rec node BEFORE step t's update
 * Returns 0 on success, negative on invalid input.
 */
int ong_run_f64(const ong_model *m, int n_sets, const float *params, int n_stim,
                int nt, const float *amps, const float *dts, int stim_node,
                double stim_area, int n_rec, const int *rec_nodes, double v_init,
                int flags, double *out, int n_threads);
int ong_run_f32(const ong_model *m, int n_sets, const float *params, int n_stim,
                int nt, const float *amps, const float *dts, int stim_node,
                double stim_area, int n_rec, const int *rec_nodes, double v_init,
                int flags, double *out, int n_threads);

/* Number of parameters / states / mechanisms of a mechanism set. */
int ong_n_params(int mechset);
int ong_n_states(int mechset);
int ong_n_mechs(int mechset);

/*
 * Gate-level entry points (single node), used to pin the channel equations
 * against the reference's own AllModels.cu compiled for the host.
 *   state: [n_states] per-node state vector (reference state_macro index),
 *          plus cai at index n_states, eca at n_states+1, ica at n_states+2.
 *   p:     [n_params] the node's parameter vector.
 */
void ong_node_init_f64(int mechset, const unsigned char *mask, double v,
                       const double *p, double *state);
void ong_node_deriv_f64(int mechset, const unsigned char *mask, double dt,
                        double v, const double *p, double *state);
/* Returns the summed current; *g gets the summed conductance, state[ica] updated. */
double ong_node_current_f64(int mechset, const unsigned char *mask, double v,
                            const double *p, double *state, double *g);

#ifdef __cplusplus
}
#endif
#endif
