/*
 * mwdg2.h -- C ABI of the B200-native adaptive MWDG2/HWFV1 shallow-water time step.
 *
 * Drop-in boundary for the reference (al0vya/gpu-mwdg2). The reference has no library
 * interface: its boundary is the process entry
 *     gpu-mwdg2 [-epsilon e] [-solver hwfv1|mwdg2] [-dirroot d] case.par
 * (source/MAIN.cu:3-24, source/input/read_command_line_params.cpp:3-47) and the
 * in-process call
 *     void run_simulation(int argc, char** argv)      (source/run_simulation.cuh:60-63).
 * This header replaces the second with status-returning entry points; the
 * `gpu-mwdg2` executable built from this library replaces the first.
 *
 * Conventions: every call returns mwdg2_status; no call exits the process; memory is
 * owned by the library; one mwdg2_sim per host thread (calls on the same handle must
 * not overlap). Arrays are plain host pointers. Leaf arrays are in the reference's
 * leaf order (Z-order of the non-uniform grid, source/mra/traverse_tree_of_sig_details.cu)
 * and hierarchy indices follow get_lvl_idx (source/utilities/get_lvl_idx.cuh:6-24).
 */
#ifndef MWDG2_H
#define MWDG2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum mwdg2_status
{
    MWDG2_OK          = 0,
    MWDG2_ERR_IO      = 1,  /* an input file is missing or unreadable */
    MWDG2_ERR_PARSE   = 2,  /* an input is malformed or unsupported */
    MWDG2_ERR_CUDA    = 3,  /* a CUDA call failed or no device is available */
    MWDG2_ERR_NUMERIC = 4,  /* NaN or negative depth detected in the state */
    MWDG2_ERR_TIMEOUT = 5,  /* a bounded device wait gave up */
    MWDG2_ERR_ARG     = 6,  /* invalid argument (null handle, short buffer, ...) */
    MWDG2_ERR_STATE   = 7,  /* call not valid in the current state (e.g. run finished) */
    MWDG2_DONE        = 8   /* mwdg2_step: simulated time already reached; nothing done */
} mwdg2_status;

typedef struct mwdg2_sim mwdg2_sim;

typedef struct mwdg2_opts
{
    int         precision;        /* 32 or 64 (arithmetic type of the state); 0 = 64 */
    int         device;           /* CUDA device ordinal; -1 = current */
    double      epsilon;          /* < 0: take from the .par (CLI -epsilon) */
    int         solver;           /* 0: from the .par; 1: HWFV1; 2: MWDG2 (CLI -solver) */
    const char* dirroot;          /* NULL: from the .par (CLI -dirroot) */
    int         write_outputs;    /* 1: write res.stage / res.cumu as the reference does */
    int         verbose;          /* 1: print the reference's progress lines */
} mwdg2_opts;

/* Fill opts with defaults (precision 64, device -1, epsilon -1, solver 0, dirroot NULL,
 * write_outputs 1, verbose 0). */
void mwdg2_default_opts(mwdg2_opts* opts);

/* Text of the last error on this thread (never NULL). */
const char* mwdg2_last_error(void);

/* Read the case and set up device state (replaces the initialisation part of
 * run_simulation, source/run_simulation.cu:9-222). Relative file names in the .par are
 * opened relative to the working directory, as the reference does. max_ref_lvl must lie in
 * 6..14 (MWDG2_ERR_PARSE otherwise: below 6 the reference itself indexes past its arrays,
 * above 14 the hierarchy's slot count leaves 32-bit range and one GPU's memory). */
mwdg2_status mwdg2_create(const char* par_path, const mwdg2_opts* opts, mwdg2_sim** out);

/* Advance one adaptive time step (one iteration of run_simulation.cu:226-774).
 * dt_out: the CFL step computed at the end of this step (the next step's dt);
 * n_leaves_out: number of leaves (active cells) updated in this step.
 * Returns MWDG2_DONE without work once the simulated time has reached sim_time. */
mwdg2_status mwdg2_step(mwdg2_sim* sim, double* dt_out, int64_t* n_leaves_out);

/* Advance up to max_steps steps (<= 0: until sim_time), writing outputs at massint as
 * the reference does. steps_done_out and leaf_updates_out may be NULL. */
mwdg2_status mwdg2_run(mwdg2_sim* sim, int64_t max_steps, int64_t* steps_done_out,
                       int64_t* leaf_updates_out);

/* Whole-process replacement of run_simulation(argc, argv): parse the reference's
 * command line, create, run to sim_time with outputs, destroy. */
mwdg2_status mwdg2_run_simulation(int argc, char** argv);

/* Scalars: [0] current time, [1] dt, [2] timestep counter (next step number),
 * [3] n_leaves, [4] max_ref_lvl, [5] xsz, [6] ysz, [7] dx, [8] epsilon, [9] solver,
 * [10] precision, [11] sim_time, [12] n_details (get_lvl_idx(L)),
 * [13] n_hierarchy (get_lvl_idx(L+1)). n must be >= 14. */
mwdg2_status mwdg2_info(mwdg2_sim* sim, double* out, int n);

/* Leaf list of the current grid: hierarchy index and level of each leaf, and its four
 * neighbours (north, east, south, west) as hierarchy index (-1 at the domain border)
 * and level, laid out [4][n]. Any pointer may be NULL. cap: capacity in leaves. */
mwdg2_status mwdg2_get_leaves(mwdg2_sim* sim, int32_t* act_idcs, int32_t* levels,
                              int32_t* nb_ids, int32_t* nb_levels, int64_t cap);

/* Leaf state after the last step, 12 rows of n values laid out [12][n]:
 * h0 qx0 qy0 z0 h1x qx1x qy1x z1x h1y qx1y qy1y z1y (HWFV1: the slope rows are 0). */
mwdg2_status mwdg2_get_state(mwdg2_sim* sim, double* out, int64_t cap);

/* Significance flags of all parents (n_details bytes, 1 = significant). */
mwdg2_status mwdg2_get_sig(mwdg2_sim* sim, uint8_t* out, int64_t cap);

/* One hierarchy array: field 0 eta, 1 qx, 2 qy, 3 z; mode 0, 1 (1x), 2 (1y);
 * n_hierarchy values. After an MWDG2 step the leaves' entries hold the new state and the
 * significant parents the scale coefficients encoded at the start of that step. After an
 * HWFV1 step the leaves' entries of eta, qx and qy hold the new state (the step wrote them
 * into the second of two alternating buffers); the other entries are not current. */
mwdg2_status mwdg2_get_hierarchy(mwdg2_sim* sim, int field, int mode, double* out, int64_t cap);

/* Depth h = eta - z of the leaf containing each stage point, in .stage file order
 * (the value written to res.stage, source/output/write_stage_point_data.cu:155-186). */
mwdg2_status mwdg2_read_stage(mwdg2_sim* sim, double* out, int n);

/* Device timing of the last step's kernels, in milliseconds, by phase:
 * [0] step open: maxima (first step only; later steps take them, and the re-inserted state,
 * from the previous step's last solver kernel) + point sources, [1] encode + threshold +
 * regularisation,
 * [2] decode bands + extra significance of the upper levels, [3] leaf topology (tile
 * counts, scan, leaf list and neighbours) beside the value decode of the upper levels,
 * [4] MWDG2 stage 1 (or the HWFV1 update), [5] scale re-encode of the stage-1 result +
 * stage-2 maximum depth, [6] MWDG2 stage 2, [7] whole step including the scalar read-back.
 * Timing mode 2 (phases; opts.verbose >= 2 at create) fills all; mode 1 (step) fills [7];
 * otherwise zeros. n <= 8. */
mwdg2_status mwdg2_last_step_timing(mwdg2_sim* sim, double* out, int n);

/* Timing of the following steps: 0 none; 1 step (two CUDA events around each step's device
 * work, outside its captured graph: no effect on the step); 2 phases (events between the
 * step's phases, captured into the step's graph, which costs ~10 us per phase boundary).
 * No counterpart in the reference (its timing is host wall time around the loop). */
mwdg2_status mwdg2_set_timing(mwdg2_sim* sim, int mode);

/* Counters of the last step used for the algorithmic-bytes roofline:
 * [0] parents encoded (E), [1] parents re-encoded scale-only (E2), [2] parents decoded (D),
 * [3] leaves (N_a), [4] detail slots (T = get_lvl_idx(L) - 3), [5] kernels launched in the
 * step, [6] / [7] MWDG2 leaves not dry in RK stage 1 / stage 2 (0 for HWFV1), [8] bytes the
 * step copied host->device (dt, boundary and point-source values), [9] bytes it copied
 * device->host (its scalars and the stage-point values), [10] dry leaves that the RK stages
 * left as they stood (keep-values decode or learned proposal; MWDG2). n <= 11. */
mwdg2_status mwdg2_last_step_counters(mwdg2_sim* sim, int64_t* out, int n);

/* Water volume of the current state, sum over leaves of h0 x leaf area (m^3), reduced on
 * the device in FP64 whatever the state's precision. No counterpart in the reference (its
 * c-prop outputs print states, not volumes). */
mwdg2_status mwdg2_volume(mwdg2_sim* sim, double* out);

/* Decode of the following steps. 0 (the default): every significant parent's children are
 * decoded from its scale coefficients and details, as the reference does
 * (mra/decoding.cu:3-67); trees, neighbours and states follow the reference build bit for
 * bit. 1 (keep values; no counterpart in the reference): the children of a parent that the
 * step's encode visited keep the values the encode read (the decode returns them only up to
 * rounding), and only the parents refined this step are decoded; their extra significance
 * comes from the encode's detail norms. The same method without the decode's round trip:
 * in FP32 the depth eta - z of a dry leaf no longer takes the round trip's rounding of eta
 * every step, and the step skips most of its decode. Since nothing then rewrites a leaf
 * that persists, an MWDG2 leaf that was dry in both RK stages of the last step and is dry
 * again keeps its state as it stands (the dry-leaf writers skip it; the leaves holding point
 * sources excepted), on steps whose two stages take the wet list, and the scale re-encode
 * between the stages keeps a parent whose four children all stand unchanged. Results are
 * those of the same decode without these skips. Graphs captured earlier are dropped. */
mwdg2_status mwdg2_set_decode_mode(mwdg2_sim* sim, int mode);

void mwdg2_destroy(mwdg2_sim* sim);

/* ---------------------------------------------------------------- batched ensembles
 * Several independent simulations advanced together, for ensembles of scenarios (different
 * DEMs, inflows, Manning n, epsilon). The reference runs one case per process; the
 * `mwdg2_batch_create(n, pars, ...)` / `mwdg2_batch_step` pair is this library's way to run
 * many. Each member keeps its own device state and CUDA stream. A batch step advances the
 * clock of every unfinished member, enqueues one time step of each from a few host threads
 * without waiting, then waits for all of them, so the members' kernels overlap on the GPU
 * and small members fill SMs that one alone would leave idle. Members may differ in size,
 * solver and end time; all take the options given at creation. Relative file names inside
 * each member's .par, and its dirroot, resolve against that .par's folder (a single
 * simulation resolves them against the working directory, as the reference does);
 * mwdg2_batch_create changes the working directory while it reads each member, so call it
 * while no other thread depends on the working directory. Members write their output files
 * like mwdg2_run. */
typedef struct mwdg2_batch mwdg2_batch;

mwdg2_status mwdg2_batch_create(int n, const char* const* par_paths, const mwdg2_opts* opts, mwdg2_batch** out);

/* One time step of every member that has not reached its sim_time. dts and leaves (n
 * entries each, either may be NULL) receive each member's next dt and leaf count (0 and 0
 * for members already done); *active (may be NULL) the number of members stepped.
 * Returns MWDG2_DONE when every member is done; on an error, the first failing member's
 * status, with mwdg2_last_error naming the member. */
mwdg2_status mwdg2_batch_step(mwdg2_batch* b, double* dts, int64_t* leaves, int32_t* active);

/* Batch steps until every member is done (max_batch_steps <= 0: no limit): batch steps
 * taken, member steps taken and leaf updates summed over members. */
mwdg2_status mwdg2_batch_run(mwdg2_batch* b, int64_t max_batch_steps, int64_t* batch_steps, int64_t* member_steps,
                             int64_t* updates);

/* Members of the batch that are MWDG2, past their first step and of the same max_ref_lvl
 * (at most `level`) and precision step together with one launch per kernel for the whole
 * size class; the others step as their own CUDA graphs on their own streams. Default 0 (no
 * classes): own graphs on own streams measured faster at every member size tried. Takes
 * effect at the next step. */
mwdg2_status mwdg2_batch_group_max_level(mwdg2_batch* b, int level);

/* Member i as a simulation handle for the getters above (mwdg2_info, mwdg2_get_state, ...).
 * The batch owns it: do not pass it to mwdg2_destroy or step it on its own. */
mwdg2_status mwdg2_batch_member(mwdg2_batch* b, int i, mwdg2_sim** out);

void mwdg2_batch_destroy(mwdg2_batch* b);

/* Leaf topology from significance flags, allocating no device memory. No counterpart in
 * the reference: it is for callers that cannot call cudaMalloc -- code running under a
 * memory manager that owns all device memory (a framework that reserves the device heap
 * up front) and real-time loops that must not enter the CUDA allocator, which may
 * synchronise the device and take driver locks. It computes what mwdg2_step computes
 * after remeshing: the leaves of the tree given by d_sig in Z order, their levels and
 * their four neighbours (north, east, south, west; -1 at the border), exactly as
 * mwdg2_get_leaves reports them.
 *
 *   d_sig        device, get_lvl_idx(max_ref_lvl) bytes, 1 = significant (as returned
 *                by mwdg2_get_sig); every significant node's parent must be significant;
 *                4-byte aligned (cudaMalloc pointers are), else MWDG2_ERR_ARG
 *   max_ref_lvl  5..13: the kernels' scratch is a file-scope device array of 65536 tile
 *                counts (about 256 KiB per device, held until the process exits); larger
 *                levels are rejected with MWDG2_ERR_ARG
 *   xsz, ysz     DEM size in cells (1..2^max_ref_lvl)
 *   d_act        device int32[cap]; d_levels device uint8[cap]
 *   d_nb_ids     device int32[4*cap]; d_nb_levels device uint8[4*cap] ([4][cap] layout)
 *   cap          at least 4^max_ref_lvl (every finest cell a leaf)
 *   n_leaves_out host; number of leaves written
 *   stream       cudaStream_t to run on (NULL: the default stream)
 * The call blocks until the outputs are complete: it waits for `stream` and copies the leaf
 * count into host memory. Each call looks up the scratch array's device address on the
 * current device (cudaGetSymbolAddress), so a device reset between calls is harmless. Every
 * call on a device shares the one scratch array, so calls whose work overlaps on the GPU
 * (different host threads or streams) race: serialise them. */
mwdg2_status mwdg2_leaf_topology_static(const uint8_t* d_sig, int max_ref_lvl, int xsz, int ysz,
                                        int32_t* d_act, uint8_t* d_levels, int32_t* d_nb_ids,
                                        uint8_t* d_nb_levels, int64_t cap, int64_t* n_leaves_out,
                                        void* stream);


/* ---------------------------------------------------------------- learned refinement proposal
 * No counterpart in the reference (which encodes every previously significant parent and
 * decodes every significant one each step, source/mra/encode_flow.cu:14-92,
 * source/mra/decoding.cu:3-67). A small MLP (128 -> 64 -> 64 -> 64 -> 4, ReLU, BF16 weights and
 * activations, FP32 accumulation on the tensor cores) proposes, per node of a coarse level C
 * (max(max_ref_lvl - 3, 9)), which of its four child subtrees the step's encode and decode
 * visit. Parameters are one FP32 block of MWDG2_MLP_PARAMS values:
 *   W1[64][128] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[4][64] b4[4]
 * Features are rows of up to 128 values (MWDG2_MLP_FEATURES used, the rest zero); labels are
 * one byte per row, bit j = child j active. */
#define MWDG2_MLP_PARAMS 16836
#define MWDG2_MLP_FEATURES 113

/* Logits [n][4] (may be NULL) and proposal bytes [n][4] (1 where the logit exceeds
 * `threshold`; may be NULL) of n feature rows of `nfeat` floats (host arrays). */
mwdg2_status mwdg2_mlp_forward(const float* params, const float* feats, int nfeat, int64_t n, float threshold,
                               float* logits, uint8_t* proposal);

/* Gradient [MWDG2_MLP_PARAMS] of the weighted logistic loss
 * sum over rows and outputs of w (softplus(z) - y z) / n, w = pos_weight where y = 1 else 1,
 * and that loss (may be NULL), for n rows (host arrays). */
mwdg2_status mwdg2_mlp_grad(const float* params, const float* feats, int nfeat, const uint8_t* labels, int64_t n,
                            float pos_weight, float* grad, float* loss);

/* Trainer: FP32 parameters and Adam moments (beta 0.9 / 0.999) on the device. */
typedef struct mwdg2_trainer mwdg2_trainer;
mwdg2_status mwdg2_trainer_create(const float* init_params, float lr, int device, mwdg2_trainer** out);
/* One Adam step on n host rows. */
mwdg2_status mwdg2_trainer_step(mwdg2_trainer* t, const float* feats, int nfeat, const uint8_t* labels, int64_t n,
                                float pos_weight, float* loss_out);
/* One Adam step on the features and labels a simulation recorded on the device for its last
 * step (mwdg2_proposal_record); every node of the coarse level is one row. */
mwdg2_status mwdg2_trainer_observe(mwdg2_trainer* t, mwdg2_sim* sim, float pos_weight, float* loss_out);
mwdg2_status mwdg2_trainer_params(mwdg2_trainer* t, float* out);
void mwdg2_trainer_destroy(mwdg2_trainer* t);

/* Record, from the next step on, the proposal's features at each step's start and the
 * activity of each child subtree over the step (one of its leaves updated by the RK stages,
 * or its significance flags at the step's end different from the last step's), for
 * mwdg2_trainer_observe. MWDG2 only; results are unchanged. on = 0 stops recording. */
mwdg2_status mwdg2_proposal_record(mwdg2_sim* sim, int on);

/* Let the MLP with `params` (MWDG2_MLP_PARAMS floats, copied) choose, from the next step on,
 * the child subtrees of the coarse level that the encode, decode and scale re-encode visit
 * (logit > threshold); subtrees left out keep their flags and values, and so do their
 * leaves that stay dry through the step (wet leaves are updated everywhere). The first step
 * after this call and every judge_every-th step after it (0: never) run in full as the
 * judge. The subtrees that needed a step
 * are those whose leaves it updated or whose flags gained significance; when the proposal
 * left out more than the fraction miss_bound of them (counted as at least 0.1 % of all
 * subtrees), the next judge_every steps run in full. params = NULL switches the proposal
 * off. MWDG2 only (MWDG2_ERR_STATE). */
mwdg2_status mwdg2_proposal_enable(mwdg2_sim* sim, const float* params, int judge_every, float threshold,
                                   float miss_bound);

/* The features ([n][128] floats, the BF16 values the MLP reads; may be NULL) and labels ([n]
 * bytes; may be NULL) the last recorded step left for its n coarse cells (cap: rows the
 * arrays hold; n is written in any case). */
mwdg2_status mwdg2_proposal_samples(mwdg2_sim* sim, float* feats, uint8_t* labels, int64_t cap, int64_t* n);

/* The last step's proposal: one byte per child subtree of the coarse level (4^(C+1), Z order
 * of level C + 1), 1 = visited. *n receives the count; out may be NULL. */
mwdg2_status mwdg2_proposal_mask(mwdg2_sim* sim, uint8_t* out, int64_t cap, int64_t* n);

/* [0] active subtrees in the last step (leaves updated or significance flags changed), [1]
 * subtrees the proposal left out that needed the step (leaves updated or flags gaining
 * significance), [2] subtrees proposed, [3] 1 if the last step applied the proposal, [4]
 * subtrees in all, [5] steps that applied it, [6] judge steps, [7] missed fraction ([1] /
 * [11]) at the last judge step, [8] fallbacks, [9] full steps left in the current fallback,
 * [10] dry leaves of left-out subtrees that the last step left as they stood, [11] subtrees
 * that needed the step. n <= 12. */
mwdg2_status mwdg2_proposal_stats(mwdg2_sim* sim, double* out, int n);

#ifdef __cplusplus
}
#endif

#endif /* MWDG2_H */
