/*
 * libngpu -- C ABI of the B200 NeuroGPU simulation core.
 *
 * Plain pointers and sizes only.  Every call returns 0 on success or a
 * negative NGPU_E* code; ngpu_last_error() gives a thread-local message.
 * Nothing here exits, aborts or traps.  Host pointers are caller-owned;
 * device buffers are owned by the model / sim handles.
 *
 * Reference interfaces replaced (paths in the reference project; U/ =
 * GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/):
 *   - the files-and-process boundary: Python writes Data/AllParams.csv
 *     (NeuroGPU_Base/scripts/template/extractModel_mappings.py:326-330) and
 *     spawns ../bin/neuroGPU <stim> (Figures/Figure4_DEAP/
 *     neurogpu_multistim_evaluator_par.py:175); U/kernel.cu:8-33 main;
 *   - topology upload U/CudaStuff.cu:372-437 (initFrameWork, topology into
 *     __constant__), read from BasicConstSegP.csv by U/MainC.cu:335-551;
 *   - launch and copies U/CudaStuff.cu:443-516 (callKernel) and
 *     U/CudaStuff.cu:518-587 (stEfork2Main: timing, VHotP<dev>.dat output).
 */
#ifndef NGPU_H
#define NGPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NGPU_ABI_VERSION 1

enum {
    NGPU_OK = 0,
    NGPU_E_INVALID = -1,   /* bad argument / malformed model */
    NGPU_E_CUDA = -2,      /* a CUDA runtime call failed */
    NGPU_E_NOMEM = -3,     /* host or device allocation failed */
    NGPU_E_STATE = -4,     /* call out of order (e.g. advance before init) */
    NGPU_E_NUMERIC = -5    /* non-finite voltage detected in a run */
};

/* Mechanism sets compiled into the library (the reference generates one
 * channel library per model: U/AllModels.cu for the TTPC cell,
 * Figures/FigureS4_mainen/CParsed/AllModels.cu for the Mainen cell). */
enum { NGPU_MECHSET_TTPC = 0, NGPU_MECHSET_MAINEN = 1, NGPU_MECHSET_GENERATED = 2 /* first defined set */ };
enum { NGPU_FP32 = 0, NGPU_FP64 = 1 };
/* How instances map onto the GPU (ngpu_sim_create_layout). */
enum { NGPU_LAYOUT_LANE_INSTANCE = 0, NGPU_LAYOUT_WARP_INSTANCE = 1 };

typedef struct ngpu_model ngpu_model;
typedef struct ngpu_sim ngpu_sim;
typedef struct ngpu_batch ngpu_batch;

const char *ngpu_last_error(void);
int ngpu_abi_version(void);
/* Device selection for the calling thread (the reference binary takes its
 * GPU from argv[1], U/kernel.cu:24-31). */
int ngpu_device_count(int32_t *n);
int ngpu_set_device(int32_t device);
/* Mechanism set description: number of mechanisms / parameters. */
int ngpu_mechset_info(int32_t mechset, int32_t *n_mech, int32_t *n_params);

/*
 * A mechanism set defined by its channel source, generated from NMODL files
 * by neurogpu_b200.nmodl (the counterpart of the reference's per-model
 * AllModels.cu, which P/extractModel.py writes from NEURON's translation of
 * the .mod files and the simulator is rebuilt with).  source defines
 *   template <typename R, bool INIT, typename MK> NGPU_HD void
 *   ngpu::generated_node(MK mk, R v, R dt, R* st, const float* pr, R& I, R& G)
 * over the mechanisms in mask-bit order; state_rows[k], n_mech_params[k] and
 * the concatenated mech_param_index give each mechanism's state rows and the
 * parameters (indices into the n_params of an AllParams row block) it reads;
 * cost[k] weighs it for the split over warps.  *mechset receives the new id
 * (NGPU_MECHSET_GENERATED + k), usable with ngpu_model_create.  Models of a
 * defined set run only through runtime compilation (FP32 and FP64; not
 * ngpu_run_static): their first initialisation compiles the kernels.
 */
int ngpu_mechset_define(const char *name, const char *source, int32_t n_mech, const int32_t *state_rows,
                        const int32_t *n_mech_params, const int32_t *mech_param_index, int32_t n_params,
                        const int32_t *cost, int32_t *mechset);

/*
 * Morphology + channel placement, shared by every instance.
 * Replaces ReadParallelNeuronData + initFrameWork (U/MainC.cu:335-551,
 * U/CudaStuff.cu:372-437).
 *   parent[n]   parent node, -1 for the root; parent[i] < i (Hines order).
 *               The reference's parent of node i is N - Ks[N-i] (U/CudaStuff.cu:195).
 *   a[n], b[n]  axial coupling: row i holds a[i] in column parent(i); row
 *               parent(i) holds b[i] in column i (the reference's f and e,
 *               read reversed from BasicConstSegP.csv lines 3-4).
 *   cm[n]       uF/cm2;  section[n]: node -> parameter section (SegToComp)
 *   mech_mask   [n_mech][n] 0/1, the reference's boolModel (line 9)
 * Nodes joined by an edge whose absolute conductance exceeds 1e7 times the
 * median edge's (near zero-area compartments of NEURON exports) are merged
 * into one internal node; callers keep addressing every node in their own
 * numbering (a merged node's voltage is its group's).  The environment
 * variable NGPU_CONTRACT=0 disables the merge (diagnostics).
 */
int ngpu_model_create(int32_t n_nodes, const int32_t *parent, const double *a, const double *b,
                      const double *cm, const int32_t *section, int32_t n_sections,
                      int32_t mechset, const uint8_t *mech_mask, ngpu_model **out);
int ngpu_model_destroy(ngpu_model *m);
/* Derived layout numbers (for tests and the bench's byte accounting). */
int ngpu_model_layout(const ngpu_model *m, int32_t *state_rows, int32_t *param_rows,
                      int32_t *n_jslots, int64_t *state_vars, int64_t *param_reads);

/* Node bookkeeping after stiff-edge merging: internal node count, the
 * caller's node count, node_internal[n_caller] (caller node -> internal
 * node) and density_scale[n_caller] (caller node's area over its internal
 * node's area; a stimulus current density on a merged node is scaled by it).
 * No counterpart in the reference, which keeps every node.  Any pointer may
 * be NULL. */
int ngpu_model_nodes(const ngpu_model *m, int32_t *n_internal, int32_t *n_caller, int32_t *node_internal,
                     double *density_scale);
/* The merged model in internal order: parent[n_internal], a, b, cm (the
 * coefficients the kernels use).  For tests and tools; any pointer may be
 * NULL. */
int ngpu_model_arrays(const ngpu_model *m, int32_t *parent, double *a, double *b, double *cm);

/* Introspection of the tree split used by a CTA of n_warps warps, per node in
 * the caller's numbering: sep_flag (1 = separator, solved by warp 0 in the
 * skeleton), item (work item holding the node, -1 for separators), junction
 * slot and parent junction slot.  Any pointer may be NULL. */
int ngpu_model_partition(const ngpu_model *m, int32_t n_warps, int32_t *sep_flag, int32_t *item,
                         int32_t *jslot, int32_t *pslot, int32_t *n_jslots);
/* The same split in the library's internal node order (heavy-first depth
 * first): perm[n_internal] maps internal -> caller's node (a merged node's
 * representative); comps[6*k] = (root, upper
 * separator, lower separator or -1, its separator index, light range lo, hi);
 * seps[3*k] = (node, skeleton parent index, linking item or -1); jslot/pslot
 * per internal node.  For tests and tools. */
int ngpu_model_split_info(const ngpu_model *m, int32_t n_warps, int32_t *perm, int32_t *n_comps,
                          int32_t *comps, int32_t max_comps, int32_t *n_seps, int32_t *seps,
                          int32_t max_seps, int32_t *jslot, int32_t *pslot);

/*
 * One complete run from host buffers (the drop-in for one neuroGPU process).
 * Replaces callKernel + stEfork2Main (U/CudaStuff.cu:443-587).
 *   params [n_sets][n_params][n_sections] float (AllParams.csv rows, U/Util.cu:210-234)
 *   amps   [n_stim][nt] nA (Stim_raw.csv); dts [nt] ms (times.csv)
 *   stim_node, stim_area_um2: Stim_meta.csv loc (0-based) and area
 *   rec_nodes[n_rec]: recorded nodes (Sim.csv RecSites)
 *   out    [n_sets][n_stim][n_rec][nt] float: V before step t's update
 *          (U/CudaStuff.cu:234-248, VHotP layout U/CudaStuff.cu:237)
 *   precision: NGPU_FP32 (production) or NGPU_FP64 (GPU oracle run)
 */
/* ngpu_run keeps its simulation's device buffers with the model and reuses
 * them when the next call has the same n_sets, n_stim and precision (a call
 * with another shape replaces them; ngpu_model_destroy releases them), so
 * repeated calls allocate and release no device memory.  With them it keeps a
 * pinned host staging buffer, sized for the larger of the parameter table and
 * the trace, through which both host copies run (the host side split over
 * threads).  Concurrent calls on one model are safe: a call that finds the
 * buffers in use runs on its own. */
int ngpu_run(ngpu_model *m, int32_t n_sets, const float *params, int32_t n_stim, int32_t nt,
             const float *amps, const float *dts, int32_t stim_node, float stim_area_um2,
             int32_t n_rec, const int32_t *rec_nodes, float v_init, int32_t precision,
             float *out);

/* ---- resident simulation: state stays in HBM across calls ---- */
/* n_sets x n_stim instances; instance k*n_stim + s runs set k on stimulus s. */
int ngpu_sim_create(ngpu_model *m, int32_t n_sets, int32_t n_stim, int32_t precision,
                    ngpu_sim **out);
int ngpu_sim_destroy(ngpu_sim *s);
/* params as in ngpu_run; on_device != 0: a device pointer.  Synchronous: it
 * gathers the parameter table, then reads back which parameters hold one
 * value (compiled into the specialised kernel, ngpu_sim_param_folds) and
 * which sections repeat another's values (they share rows,
 * ngpu_sim_param_rows); after ngpu_sim_init, values that change either
 * re-select the kernel or re-upload the node records before the next launch. */
int ngpu_sim_set_params(ngpu_sim *s, const float *params, int32_t on_device);
int ngpu_sim_set_stimulus(ngpu_sim *s, int32_t nt, const float *amps, const float *dts,
                          int32_t stim_node, float stim_area_um2, int32_t on_device);
/* rec_every: record every k-th step (1 = every step, as the reference). */
int ngpu_sim_set_recording(ngpu_sim *s, int32_t n_rec, const int32_t *rec_nodes,
                           int32_t rec_every);
/* V := v_init, channel states := steady state (U/CudaStuff.cu:186-221). */
int ngpu_sim_init(ngpu_sim *s, float v_init, void *cuda_stream);
/* Steps [t0, t0 + n_steps) of the stimulus, enqueued on cuda_stream. */
int ngpu_sim_advance(ngpu_sim *s, int32_t t0, int32_t n_steps, void *cuda_stream);

/* As ngpu_sim_create with the CTA's warp count chosen by the caller (1..8;
 * 0 = the library's choice from the morphology size).  The warp count sets
 * how the tree is split over the CTA's warps; an autotuner picks it per
 * morphology by timing. */
int ngpu_sim_create_ex(ngpu_model *m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t n_warps,
                       ngpu_sim **out);
/* As ngpu_sim_create_ex, also choosing how many work items per warp the tree
 * is split into (1..8; 0 = the library's choice: 2 where the channel pass
 * prefetches rows, 3 where it does not).  More items balance the warps'
 * dynamic queue better at the price of more skeleton nodes; the best count
 * depends on the morphology, so the autotuner times it.  No counterpart in
 * the reference (one thread per compartment group, no split). */
int ngpu_sim_create_shaped(ngpu_model *m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t n_warps,
                           int32_t items_per_warp, ngpu_sim **out);
/*
 * As ngpu_sim_create with the layout chosen by the caller.
 *   NGPU_LAYOUT_LANE_INSTANCE  one lane per instance, 32 instances per CTA,
 *       cta_warps warps sharing the tree (1..16; above 8 only through the
 *       runtime-compiled kernel, bounded for 3 CTAs per SM), items work
 *       items per warp (1..8); 0 = the library's choice.  With up to 8 warps
 *       this is ngpu_sim_create_shaped.
 *       A B200 fills from about 148 x 32 x 2 instances on.
 *   NGPU_LAYOUT_WARP_INSTANCE  one warp per instance (its lanes share the
 *       instance's tree, split into `items` work items, 1..512; 0 = 32),
 *       cta_warps instances per CTA (1..8; 0 = enough CTAs for every SM):
 *       for batches too small to fill the GPU 32 instances per CTA.
 * Both compute the same step (U/CudaStuff.cu:227-330) on the same buffers;
 * traces, features and checks read the same.  The reference's kernel is
 * one CTA per parameter set, 32 threads x NILP compartments each
 * (U/CudaStuff.cu:164-167); neurogpu_b200.autotune times both layouts.
 * Batches (ngpu_batch_create) hold lane-instance simulations.
 */
int ngpu_sim_create_layout(ngpu_model *m, int32_t n_sets, int32_t n_stim, int32_t precision, int32_t layout,
                           int32_t cta_warps, int32_t items, ngpu_sim **out);
/* The simulation's layout, CTA warps and items (as ngpu_sim_create_layout's
 * arguments, with the library's choices filled in); any pointer may be NULL. */
int ngpu_sim_layout(const ngpu_sim *s, int32_t *layout, int32_t *cta_warps, int32_t *items);

/*
 * Several simulations in one launch (morphologies of different sizes, one
 * mechanism set and precision): CTAs are dealt to the members in order, each
 * runs its member's groups exactly as a separate launch would (bitwise the
 * same results).  Members keep their own parameters, stimuli, recordings and
 * traces (ngpu_sim_get_trace).  Up to 16 members.  The reference runs one
 * morphology per process (U/CudaStuff.cu:518-587); no counterpart.
 *   ngpu_batch_init       ngpu_sim_init of every member, one launch
 *   ngpu_batch_advance    ngpu_sim_advance of every member, one launch
 *   ngpu_batch_run_graph  init + ceil(nt/chunk) advance launches captured once
 *                         as a CUDA graph on `cuda_stream` (non-default) and
 *                         replayed; the capture is reused while the members'
 *                         buffers, nt, chunk and stream are unchanged.
 */
int ngpu_batch_create(ngpu_sim *const *sims, int32_t n, ngpu_batch **out);
int ngpu_batch_destroy(ngpu_batch *b);
int ngpu_batch_init(ngpu_batch *b, float v_init, void *cuda_stream);
int ngpu_batch_advance(ngpu_batch *b, int32_t t0, int32_t n_steps, void *cuda_stream);
int ngpu_batch_run_graph(ngpu_batch *b, float v_init, int32_t nt, int32_t chunk, void *cuda_stream);
/* Number of recorded samples per (instance, site): ceil(nt / rec_every). */
int ngpu_sim_n_samples(const ngpu_sim *s);
/* out [n_sets][n_stim][n_rec][n_samples]; on_device != 0: device pointer. */
int ngpu_sim_get_trace(ngpu_sim *s, float *out, int32_t on_device, void *cuda_stream);
/* Count of instances whose voltage became non-finite (read after sync). */
int ngpu_sim_check(ngpu_sim *s, int32_t *n_bad, void *cuda_stream);
/* Device pointer of the trace buffer, layout [n_samples][n_rec][n_inst_padded]. */
int ngpu_sim_trace_device(ngpu_sim *s, const float **trace, int32_t *n_inst_padded);

/*
 * 20 spike / ISI / amplitude / AHP / voltage features per trace on the GPU,
 * the vector of neurogpu_b200.features.FEATURES (spikes: upward crossings
 * of `threshold` inside [stim_on, stim_off) ms; every feature defined
 * without spikes).  Replaces the reference's per-trace extraction on a CPU
 * pool (P/efel_ext.py:23-96 with eFEL, GUI/score_functions.py).
 *   ngpu_trace_features  traces at v_dev[t * stride_trace + s * stride_sample]
 *                        (device memory), out_dev [n_traces][20]
 *   ngpu_sim_features    from a simulation's own trace buffer, recording site
 *                        `site`, without copying it: out_dev [n_sets][n_stim][20];
 *                        dt is the sample spacing (step dt x rec_every)
 */
int ngpu_trace_features(const float *v_dev, int64_t stride_trace, int64_t stride_sample, int32_t n_traces,
                        int32_t n_samples, double dt, double stim_on, double stim_off, float threshold,
                        float *out_dev, void *cuda_stream);
int ngpu_sim_features(ngpu_sim *s, int32_t site, double dt, double stim_on, double stim_off, float threshold,
                      float *out_dev, void *cuda_stream);

/*
 * Parameter-exploration score per trace: the number of peaks that
 * scipy.signal.find_peaks(dvdt, height=height, distance=distance) finds in
 * dvdt = diff(v) / dt (dt: the sample spacing, ms), computed on the GPU.
 * Replaces the host scoring of the reference's exploration run
 * (GUI/plot_param_explor.py:77-107: find_peaks(dvdt, 15, distance=5) on each
 * of the 10,000 traces of GUI/run_neuroGPU.py's grid, read back from
 * VHotP0.dat).  Equal-height peaks closer than `distance` keep the later one.
 *   ngpu_trace_dvdt_peaks  traces at v_dev[t * stride_trace + s * stride_sample]
 *                          (device memory); out_dev [n_traces] int32
 *   ngpu_sim_dvdt_peaks    a simulation's own trace buffer, recording site
 *                          `site`: out_dev [n_sets][n_stim]
 *   scratch_dev: device memory of at least ngpu_dvdt_peaks_scratch_bytes
 *   bytes (the candidate peaks of every trace), owned by the caller.
 *   The kernel runs on cuda_stream: the simulation's launches must be on
 *   the same stream or finished.  Errors: dt <= 0, distance < 1, a NaN
 *   height, too small a scratch.
 */
int64_t ngpu_dvdt_peaks_scratch_bytes(int32_t n_traces, int32_t n_samples);
int ngpu_trace_dvdt_peaks(const float *v_dev, int64_t stride_trace, int64_t stride_sample, int32_t n_traces,
                          int32_t n_samples, double dt, double height, int32_t distance, void *scratch_dev,
                          int64_t scratch_bytes, int32_t *out_dev, void *cuda_stream);
int ngpu_sim_dvdt_peaks(ngpu_sim *s, int32_t site, double dt, double height, int32_t distance, void *scratch_dev,
                        int64_t scratch_bytes, int32_t *out_dev, void *cuda_stream);

/*
 * Runtime specialisation of the advance kernel.  At initialisation a
 * simulation (or, at creation, a batch), FP32 or FP64, gets a kernel compiled
 * with NVRTC for its model's mechanism masks (up to 16): nodes with those masks
 * run channel code in which the mask is a compile-time constant.  The
 * reference regenerates and recompiles its simulator per model ahead of time
 * (AllModels.cu / AllModels.cuh); no API counterpart.  Without NVRTC, after a
 * failed compile, or with NGPU_JIT=0 in the environment, the ahead-of-time
 * kernel runs (same results up to rounding order within a node).
 *   ngpu_sim_classes  masks compiled for the kernel that runs s (0: the
 *                     ahead-of-time kernel); valid after ngpu_sim_init
 *   ngpu_jit_build    compile only (no device needed) for compute
 *                     capability cc_major.cc_minor: the cubin's size
 *   ngpu_jit_log      the last compile failure or reason for falling back
 */
int ngpu_sim_classes(const ngpu_sim *s, int32_t *n_classes);
/* Parameters the simulation's runtime-specialised kernel compiles in as
 * constants (after init): those with one value in every parameter set and
 * every section that uses them, found by set_params; 0 where folding does
 * not apply (NGPU_JIT=0 or NGPU_PARAM_FOLD=0).  For a
 * member of a batch: those its batch's kernel compiles in, the parameters
 * every member holds at the same value.
 * The reference compiles its model's GLOBAL parameters into its generated
 * channel code in the same way (AllModels.cu). */
int ngpu_sim_param_folds(const ngpu_sim *s, int32_t *n_folds);
/* Parameter rows per group of 32 instances that the kernels read, and the
 * rows the table holds: set_params lets the nodes of a section whose
 * parameter values (every row, every instance) repeat another section's of
 * the same mechanism combination read that section's rows, so only distinct
 * rows are touched (NGPU_PARAM_DEDUP=0 keeps every section's own).  No
 * counterpart in the reference, which stores parameters per compartment. */
int ngpu_sim_param_rows(const ngpu_sim *s, int32_t *rows_read, int32_t *rows_total);
int ngpu_jit_build(int32_t mechset, int32_t precision, const uint32_t *masks, int32_t n_masks,
                   int32_t cc_major, int32_t cc_minor, int64_t *cubin_bytes);
const char *ngpu_jit_log(void);

/*
 * Allocation-free variant of ngpu_run.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory -- a host program that
 * owns a fixed device-memory arena and budget and hands the library only
 * slices of it, or a loop with latency limits that cannot take the device-wide
 * synchronisation and unbounded time of cudaMalloc / cudaFree.  The run's
 * internal buffers (node records, channel states, parameter table, solver
 * scratch, trace) live in one file-scope __device__ array of 16 MiB inside
 * the library, which every GPU that loads the library holds until exit.
 * Nothing is allocated: no cudaMalloc, cudaFree or other allocating call.
 *
 *   params_dev, amps_dev, dts_dev, out_dev: the caller's DEVICE memory, in the
 *     layouts of ngpu_run; rec_nodes: host array.  FP32 only.
 *   Limits: at most 512 nodes, 256 instances (sets x stimuli), 16 recording
 *     sites, and the run must fit the 16 MiB array (nodes x instances x
 *     states plus the nt-sample trace); larger runs are rejected with
 *     NGPU_E_INVALID and a message giving the bytes needed.
 *   Each call copies its small host tables (node records, work items,
 *     recording columns) to the array with cudaMemcpyAsync on cuda_stream and
 *     synchronises cuda_stream before it enqueues the simulation, so all
 *     earlier work on that stream has finished when the call returns; the
 *     simulation itself runs on after the call returns.  Non-finite voltages
 *     are not reported.
 *   Every call looks up the array's device address (cudaGetSymbolAddress)
 *     with the caller's device current, which allocates nothing; the first
 *     call on a device also loads the library's kernels onto it, so make that
 *     first call before any stream capture.  All calls share the array and
 *     find the previous call's contents in it (each call resets what it
 *     relies on), so calls that overlap on the GPU race: serialise them.
 */
int ngpu_run_static(ngpu_model *m, int32_t n_sets, const float *params_dev, int32_t n_stim,
                    int32_t nt, const float *amps_dev, const float *dts_dev, int32_t stim_node,
                    float stim_area_um2, int32_t n_rec, const int32_t *rec_nodes, float v_init,
                    float *out_dev, void *cuda_stream);

/* Kernel launches issued by this thread since the last call (for accounting). */
int64_t ngpu_launch_count(int32_t reset);

/*
 * BF16 tensor-core GEMM (tcgen05) of the surrogate network, device pointers:
 *   D[M][N] = A[M][K] . B[N][K]^T, A and B bf16 row-major (K contiguous),
 *   K a multiple of 64, lda/ldb multiples of 8, 16-byte aligned; fp32
 *   accumulation.  epilogue: 0 out_f32 = D; 1 z = D + bias: out_f32 = z,
 *   out_bf16 = gelu(z) (tanh form) and its transpose out_bf16_t[n][m];
 *   2 out_f32 = D + bias; 3 dz = D * gelu'(zin): out_bf16 = dz and
 *   out_bf16_t = dz^T; 4 out_f32 = D with K split over CTAs (for K much
 *   larger than M and N, as in the network's weight gradients: the output
 *   is zeroed on the stream, the slices add their partial sums with
 *   atomics, so the summation order varies from run to run within fp32
 *   rounding).  bn: the N tile (32, 64, 128, 256).  GELU's tanh is the
 *   hardware approximation (relative error ~5e-4, below the bf16 outputs'
 *   rounding).  More than two tiles per SM run on the persistent kernel
 *   (one CTA per SM, results bit for bit those of one CTA per tile).  A
 *   wait that exceeds its bound sets a device flag read (and cleared) by
 *   ngpu_gemm_error.  No counterpart in the reference.
 */
int ngpu_gemm_bf16_tn(const void *A, const void *B, int32_t M, int32_t N, int32_t K, int32_t lda, int32_t ldb,
                      int32_t epilogue, int32_t bn, float *out_f32, void *out_bf16, void *out_bf16_t, int32_t ldo,
                      int32_t ldt, const float *bias, const float *zin, void *cuda_stream);
int ngpu_gemm_error(int32_t *flag);

/*
 * Genetic-algorithm steps on the device (all pointers device memory, all
 * objectives minimised), so that a generation needs no host round trip.
 * They replace the host-side DEAP operators between simulator calls
 * (GUI/DEAP_helper.py:126-182 varOr; bluepyopt's selector set up at
 * Figures/Figure4_DEAP/optimize_parameters_genetic_alg.py:49).
 *
 *   ngpu_ga_offspring       n_kids children of the population pop[mu][n_genes]:
 *                           binary tournaments on (rank asc, crowd desc), with
 *                           probability cx_prob bounded SBX (eta_c, per-gene
 *                           probability 1/2) of the two winners, then bounded
 *                           polynomial mutation (eta_m, per-gene probability
 *                           p_mut), genes in [low, up].  Random draws are
 *                           SplitMix64 of (seed, generation, child, draw): the
 *                           same arguments give the same children.
 *   ngpu_ga_select_truncation  the mu smallest scores (ties: lower index
 *                           first; NaN last) -> out_idx[mu], in score order.
 *   ngpu_ga_select_nsga2    NSGA-II survivors of obj[n][m]: front ranks by
 *                           non-dominated sorting (rank[n]), crowding distance
 *                           within fronts (crowd[n]; +inf at a front's ends),
 *                           out_idx[mu] in (rank asc, crowd desc, index asc)
 *                           order; n_fronts[0] = number of fronts.  NaN counts
 *                           as +inf.  n <= 32768, m <= 192.
 * Scratch memory is taken from and returned to the device's default
 * stream-ordered pool (cudaMallocAsync); the first call raises that pool's
 * release threshold so that freed scratch stays in the pool for the next
 * call (for the life of the process).
 */
int ngpu_ga_offspring(const double *pop_dev, const int32_t *rank_dev, const double *crowd_dev, int32_t mu,
                      int32_t n_genes, int32_t n_kids, double low, double up, double eta_c, double eta_m, double cx_prob,
                      double p_mut, uint64_t seed, uint64_t generation, double *kids_dev, void *cuda_stream);
int ngpu_ga_select_truncation(const double *score_dev, int32_t n, int32_t mu, int32_t *out_idx_dev,
                              void *cuda_stream);
int ngpu_ga_select_nsga2(const double *obj_dev, int32_t n, int32_t m, int32_t mu, int32_t *out_idx_dev,
                         int32_t *rank_dev, double *crowd_dev, int32_t *n_fronts_dev, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif
