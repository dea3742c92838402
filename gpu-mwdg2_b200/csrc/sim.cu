// Simulation object and C ABI (include/mwdg2.h).
//
// Host loop per step (mirrors source/run_simulation.cu:226-774 step by step):
//   time update -> maxima + re-insertion -> point sources -> [encode+threshold+regularise
//   -> decode+extra significance -> leaf topology] -> MWDG2 stage 1 -> re-insert ->
//   scale re-encode -> stage 2 (or HWFV1 update) -> one small read-back (dt, leaves).
// MWDG2 folds both re-insertions into the RK stages: stage 1 writes U* straight into a
// second (stage) hierarchy, stage 2 writes U^{n+1} into the hierarchy and reduces the
// maxima the next step starts from, so after the first step the step begins with the
// point sources.
// All per-step state stays on the device; the only host<->device traffic per step is the
// point-source values (when there are sources) and the scalar read-back.
#include "../../include/mwdg2.h"
#include "case_io.hpp"
#include "init.cuh"
#include "outputs.cuh"
#include "proposal_sim.cuh"
#include "solver.cuh"
#include "batch.cuh"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_last_error = "";

mwdg2_status set_err(mwdg2_status st, const std::string& msg)
{
    g_last_error = msg;
    return st;
}

#define CU(call)                                                                                          \
    do                                                                                                    \
    {                                                                                                     \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return set_err(MWDG2_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)

struct SimBase
{
    virtual ~SimBase() = default;
    virtual mwdg2_status init(const char* par, const mwdg2_opts& o) = 0;
    virtual mwdg2_status step(double* dt, int64_t* n) = 0;
    // A step in three parts, so that many simulations can have steps in flight at once:
    // begin_step advances the clock (MWDG2_DONE once sim_time is reached), enqueue_step puts
    // the step's kernels and its scalar read-back on the simulation's stream and returns,
    // finish_step waits for them and takes the new dt and leaf count.
    virtual mwdg2_status begin_step() = 0;
    virtual mwdg2_status enqueue_step() = 0;
    virtual mwdg2_status finish_step(double* dt, int64_t* n) = 0;
    virtual bool first_step() const = 0;
    virtual mwdg2_status prepare_outputs() = 0;
    virtual mwdg2_status after_step(bool first, double dt, int64_t n, double step_seconds) = 0;
    // Make a relative output folder relative to `dir` instead of the working directory.
    virtual void anchor_outputs(const std::string& dir) = 0;
    virtual mwdg2_status run(int64_t max_steps, int64_t* steps, int64_t* updates) = 0;
    virtual mwdg2_status info(double* out, int n) = 0;
    virtual mwdg2_status leaves(int32_t* a, int32_t* l, int32_t* ids, int32_t* lv, int64_t cap) = 0;
    virtual mwdg2_status state(double* out, int64_t cap) = 0;
    virtual mwdg2_status sig(uint8_t* out, int64_t cap) = 0;
    virtual mwdg2_status hierarchy(int f, int m, double* out, int64_t cap) = 0;
    virtual mwdg2_status stage(double* out, int n) = 0;
    virtual mwdg2_status timing(double* out, int n) = 0;
    virtual mwdg2_status set_timing(int mode) = 0;
    virtual mwdg2_status counters(int64_t* out, int n) = 0;
    virtual mwdg2_status volume(double* out) = 0;
    virtual mwdg2_status decode_mode(int mode) = 0;
    // learned refinement proposal
    virtual mwdg2_status proposal_record(bool on) = 0;
    virtual mwdg2_status proposal_enable(const float* params, int judge_every, float threshold, float miss_bound) = 0;
    virtual mwdg2_status proposal_stats(double* out, int n) = 0;
    virtual mwdg2_status proposal_samples(const void** feats, const uint8_t** labels, int64_t* n, int* device) = 0;
    virtual mwdg2_status proposal_samples_host(float* feats, uint8_t* labels, int64_t cap, int64_t* n) = 0;
    virtual mwdg2_status proposal_mask(uint8_t* out, int64_t cap, int64_t* n) = 0;
    // batched ensembles: members with the same key (>= 0) step together in one launch per
    // kernel (Group); -1: this simulation steps on its own
    virtual int group_key() const = 0;
};

template <typename T> class Sim final : public SimBase
{
public:
    ~Sim() override { release(); }

    mwdg2_status init(const char* par, const mwdg2_opts& o) override;
    mwdg2_status step(double* dt_out, int64_t* n_out) override;
    mwdg2_status begin_step() override;
    mwdg2_status enqueue_step() override;
    mwdg2_status finish_step(double* dt_out, int64_t* n_out) override;
    bool first_step() const override { return first_; }
    int group_key() const override
    {
        const bool ok = mw_ && !first_ && !finished_ && cs_.epsilon > T(0) && !prop_on() && !keep_ && timing_mode_ == 0 &&
                        m_args_ && (cs_.srcs.empty() || m_src_) && cs_.stage_codes.size() <= 64;
        return ok ? (L_ | (sizeof(T) == 8 ? 1 << 8 : 0)) : -1;
    }
    template <typename U> friend class Group;
    mwdg2_status prepare_outputs() override;
    mwdg2_status after_step(bool first, double dt, int64_t n, double step_seconds) override;
    void anchor_outputs(const std::string& dir) override
    {
        if (!cs_.dirroot.empty() && cs_.dirroot[0] != '/') cs_.dirroot = dir + "/" + cs_.dirroot;
    }
    mwdg2_status run(int64_t max_steps, int64_t* steps, int64_t* updates) override;
    mwdg2_status info(double* out, int n) override;
    mwdg2_status leaves(int32_t* a, int32_t* l, int32_t* ids, int32_t* lv, int64_t cap) override;
    mwdg2_status state(double* out, int64_t cap) override;
    mwdg2_status sig(uint8_t* out, int64_t cap) override;
    mwdg2_status hierarchy(int f, int m, double* out, int64_t cap) override;
    mwdg2_status stage(double* out, int n) override;
    mwdg2_status timing(double* out, int n) override;
    mwdg2_status set_timing(int mode) override;
    mwdg2_status counters(int64_t* out, int n) override;
    mwdg2_status volume(double* out) override;
    mwdg2_status decode_mode(int mode) override;
    mwdg2_status proposal_record(bool on) override;
    mwdg2_status proposal_enable(const float* params, int judge_every, float threshold, float miss_bound) override;
    mwdg2_status proposal_stats(double* out, int n) override;
    mwdg2_status proposal_samples(const void** feats, const uint8_t** labels, int64_t* n, int* device) override;
    mwdg2_status proposal_samples_host(float* feats, uint8_t* labels, int64_t cap, int64_t* n) override;
    mwdg2_status proposal_mask(uint8_t* out, int64_t cap, int64_t* n) override
    {
        if (!prop_learned_) return set_err(MWDG2_ERR_STATE, "no proposal is enabled");
        if (n) *n = prop_nC_ * 4;
        if (!out) return MWDG2_OK;
        if (cap < prop_nC_ * 4) return set_err(MWDG2_ERR_ARG, "capacity below the number of subtrees");
        CU(cudaSetDevice(device_));
        CU(cudaStreamSynchronize(st_));
        CU(cudaMemcpy(out, d_prop_, (size_t)prop_nC_ * 4, cudaMemcpyDeviceToHost));
        return MWDG2_OK;
    }

private:
    mwio::Case<T> cs_;
    mwdg2_opts opts_{};
    bool mw_ = true;
    int L_ = 0, M_ = 0, n_det_ = 0, n_all_ = 0, D_ = 0, ntiles_ = 0;
    int64_t F_ = 0;
    T dt_ = T(0.001), time_ = T(0);
    bool first_ = true, finished_ = false;
    int timestep_ = 1;
    int n_leaves_ = 0;
    int solver_blocks_ = 0, red_blocks_ = 0;
    int device_ = 0;
    cudaStream_t st_ = nullptr;
    std::vector<void*> allocs_;
    mw::Hier<T> hr_{};
    mw::Hier<T> hs_{};                  // MWDG2 stage hierarchy (U*), bed and flags shared with hr_;
                                        // HWFV1: the buffer the step's FV1 result goes into
    // HWFV1 alternates hr_ and hs_ (eta, qx, qy) every step; a captured graph holds the
    // pointers of one parity, so the parity is part of the graph's key
    bool flip_ = false;
    mw::Leaves<T> lf_{};
    mw::Scalars<T>* sc_ = nullptr;      // device
    mw::Scalars<T>* sc_host_ = nullptr; // pinned
    int32_t* tile_counts_ = nullptr;
    // bands of up to kBandDepth tree levels at and below level kBandMaxLevel, bottom first
    struct Band { int lo, depth, grid; };
    std::vector<Band> bands_;
    int32_t* wet_list_ = nullptr;       // leaves that are not dry in an RK stage
    mw::StepArgs<T>* d_args_ = nullptr; // this step's dt and boundary values (device)
    mw::StepArgs<T>* h_args_ = nullptr; // pinned; copied to d_args_ by the step's first operation
    // device addresses of the pinned h_args_ / h_src_ (mapped host memory), read directly by
    // k_step_open; null where the mapping is not available (then copies and two kernels)
    const mw::StepArgs<T>* m_args_ = nullptr;
    const mw::Src<T>* m_src_ = nullptr;
    // Per-leaf kernels run persistent grids (grid-stride loops): SMs x resident blocks of each
    // kernel, so a step's launches do not depend on the leaf count and can be replayed.
    int grid_leaf_ = 0, grid_wet_ = 0, grid_dry_ = 0, grid_stage_ = 0;
    uint8_t* dry_ = nullptr;            // dry marks of RK stage 1 (k_stage_wet -> k_stage_dry)
    uint8_t* dry2_ = nullptr;           // and of stage 2
    // learned proposal and keep-values decode: per hierarchy index, the tag of the last step
    // in which the leaf there was dry in both stages (k_stage_wet<2>, on steps whose two
    // stages take the wet list)
    uint32_t* clean_tag_ = nullptr;
    // keep-values decode: the dry-leaf writers' mask (nodes of level C + 1, 1 = not frozen):
    // every subtree may hold frozen leaves but those of the point sources
    uint8_t* d_keep_prop_ = nullptr;
    // keep-values decode: the stage hierarchy's slot tags (mw::Hier::tag)
    uint32_t* hs_tag_ = nullptr;
    cudaStream_t st2_ = nullptr;        // the wet-list kernels, beside the dry-leaf writers
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    // the value decode of the levels above the bands, beside the leaf topology (its own
    // stream and events: sharing the stage kernels' ones ties the two forks together in
    // the captured graph and serialised the RK stage-1 branches)
    cudaStream_t st_dec_ = nullptr;
    cudaEvent_t ev_dec_fork_ = nullptr, ev_dec_join_ = nullptr;
    // A step after the first is captured once per variant (which RK stages take the wet
    // list) and replayed as one CUDA graph; capture failures fall back to direct launches.
    bool use_graphs_ = true, capturing_ = false;
    struct Captured { cudaGraphExec_t exec; int launches; };
    std::map<int, Captured> graphs_;   // keyed by the step's launch choices (variant_key)
    // significant parents per level last step (levels above the bands): a level under one
    // in eight significant takes the sparse kernel (k_level_sparse)
    int64_t sig_prev_[16] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    bool sparse_level(int level) const
    {
        return sig_prev_[level] >= 0 && sig_prev_[level] * 8 < ((int64_t)1 << (2 * level));
    }
    int variant_key() const
    {
        int key = (mw_ && use_list(1) ? 1 : 0) | (mw_ && use_list(2) ? 2 : 0) | (timed_ ? 1 << 24 : 0) |
                  (!mw_ && flip_ ? 1 << 23 : 0) | (prop_rec_ ? 1 << 22 : 0) | (prop_learned_ ? 1 << 21 : 0) |
                  (prop_apply_ ? 1 << 20 : 0);
        for (int level = mw::kBandMaxLevel + 1; level < L_; ++level)
            if (sparse_level(level)) key |= 4 << (level - mw::kBandMaxLevel - 1);
        return key;
    }
    int64_t wet_prev_[2] = {-1, -1};    // previous step's wet-leaf count per RK stage
    mw::Src<T>* d_src_ = nullptr;
    mw::Src<T>* h_src_ = nullptr;       // pinned
    int32_t* d_stage_codes_ = nullptr;
    T* d_stage_out_ = nullptr;
    T* h_stage_ = nullptr;              // pinned: stage-point values sampled at the end of each step
    size_t scal_bytes_ = 0;             // scalars + stage-point values (device block sc_, host sc_host_)
    bool stage_fresh_ = false;          // h_stage_ holds the current state's values
    double* d_state_scratch_ = nullptr;
    T* d_dt_leaf_ = nullptr;            // per-leaf CFL step of the last stage (VTK output only)
    T* d_raster_ = nullptr;             // raster rows (saveint raster maps)
    mw::Params<T> P_{};
    // timing
    // timing_mode_ 2 (phases): events between the step's phases, captured into the step's
    // graph as event nodes (each breaks the launch pipelining of the graph, ~10 us);
    // 1 (step): two stream events around the step, outside any graph; 0: none
    int timing_mode_ = 0;
    bool timed_ = false;                // timing_mode_ == 2
    // keep-values decode (mwdg2_set_decode_mode 1): only the parents refined this step are
    // decoded; the children of encoded parents keep the values the encode read
    bool keep_ = false;
    cudaEvent_t ev_[9] = {};
    cudaEvent_t ev_step_[2] = {};
    double last_ms_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t last_cnt_[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int launches_ = 0;
    // learned refinement proposal (csrc/proposal_sim.cuh): record features and activity labels
    // (prop_rec_), propose the subtrees the encode and decode visit (prop_learned_); every
    // judge_every_-th step runs in full as the judge, and a step whose active subtrees the
    // proposal missed beyond miss_bound_ makes the next judge_every_ steps run in full
    bool prop_rec_ = false, prop_learned_ = false, prop_apply_ = false, prop_judge_ = false;
    int prop_C_ = 0;
    int64_t prop_nC_ = 0;
    __nv_bfloat16* d_feat_ = nullptr;   // [4^C][128] features of the step's start
    uint8_t* d_lab_ = nullptr;          // [4^C] activity bits of the children in the last step
    uint16_t* d_ring_ = nullptr;        // [4^C / 128] tile summaries of d_lab_ (mw::ring_bits)
    int32_t* d_prop_src_ = nullptr;     // the subtree (node of level C + 1) of each point source
    uint8_t* d_act_ = nullptr;          // [4^(C+1)] activity marks of this step
    uint8_t* d_prop_ = nullptr;         // [4^(C+1)] proposal of this step
    uint8_t* d_sig5_ = nullptr;         // [4^(C+1)] flags of each subtree's two parent levels, last step
    float* d_mlp_ = nullptr;            // MLP parameters
    uint8_t* d_mlp_pack_ = nullptr;     // their shared-memory image (mlp::k_mlp_pack)
    int* d_mlp_err_ = nullptr;
    float prop_thr_ = 0.0f, prop_bound_ = 0.0f;
    int prop_judge_every_ = 0, prop_since_judge_ = 0, prop_fallback_left_ = 0;
    int64_t prop_learned_steps_ = 0, prop_judge_steps_ = 0, prop_fallbacks_ = 0;
    double prop_last_[6] = {0, 0, 0, 0, 0, 0};   // active, missed, proposed, applied, frozen leaves, needed
    double prop_judge_rate_ = 0.0;            // missed / active at the last judge step
    mwdg2_status prop_alloc();
    mwdg2_status freeze_alloc();        // same-position marks, clean tags (proposal, keep values)
    mw::PropMask keep_mask() const { return mw::PropMask{d_keep_prop_, prop_C_ + 1}; }
    // outputs
    std::chrono::steady_clock::time_point t_start_;
    double time_mra_ = 0, time_solver_ = 0;

    template <typename P> mwdg2_status dalloc(P*& p, size_t count)
    {
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, count * sizeof(P) + 64);
        if (e != cudaSuccess) return set_err(MWDG2_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs_.push_back(v);
        p = static_cast<P*>(v);
        return MWDG2_OK;
    }
    void release();
    mwdg2_status launch_step();    // enqueue only (graph replay or direct launches)
    mwdg2_status launch_step_device();
    void prepare_args();           // this step's dt, boundary and point-source values (host)
    mwdg2_status enqueue_device(); // the step's device work, on st_
    mwdg2_status collect_step();   // wait, timing, counters
    // One MWDG2 RK stage. When fewer than half of the leaves were wet in this stage last
    // step, a light pass finishes the dry leaves and lists the others for the full kernel;
    // otherwise one sweep over all leaves.
    bool use_list(int stage) const
    {
        const int64_t w = wet_prev_[stage - 1];
        return w >= 0 && 2 * w < n_leaves_;
    }
    // With the wet list: the wet test, then the dry leaves' writer on st_ beside the wet-list
    // kernel on st2_ (disjoint leaves; the writer is bandwidth-bound, the wet-list kernel
    // latency-bound), joined before the stage ends.
    template <int STAGE> void stage(const mw::Hier<T>& hin, const mw::Hier<T>& hout, bool fric)
    {
        if (use_list(STAGE))
        {
            uint8_t* marks = STAGE == 1 ? dry_ : dry2_;
            // learned proposal: stage 2 tags the leaves that stayed dry in both stages, and
            // leaves left out by the proposal are frozen, when both stages take the list;
            // keep-values decode: the decode leaves every persistent leaf as it stands, so
            // the dry leaves of every subtree but the point sources' may be frozen
            const bool lists = use_list(1) && use_list(2);
            const mw::PropMask pm = !lists ? mw::PropMask{} : keep_ && d_keep_prop_ ? keep_mask() : prop_mask();
            mw::k_stage_wet<T, STAGE><<<grid_wet_, 256, 0, st_>>>(lf_, hin, sc_, P_, d_args_, marks, wet_list_, dry_,
                                                                  STAGE == 2 && lists ? clean_tag_ : nullptr);
            cudaEventRecord(ev_fork_, st_);
            cudaStreamWaitEvent(st2_, ev_fork_, 0);
            mw::k_mwdg2_stage<T, STAGE, true><<<grid_stage_, mw::kSolverThreads, 0, st2_>>>(lf_, hin, hout, sc_, P_,
                                                                                           d_args_, fric, wet_list_);
            mw::k_stage_dry<T, STAGE><<<grid_dry_, 256, 0, st_>>>(lf_, hin, hout, sc_, P_, fric, marks, dry_, pm,
                                                                  STAGE == 1 ? clean_tag_ : nullptr);
            cudaEventRecord(ev_join_, st2_);
            cudaStreamWaitEvent(st_, ev_join_, 0);
            launches_ += 3;
        }
        else
        {
            mw::k_mwdg2_stage<T, STAGE, false><<<grid_stage_, mw::kSolverThreads, 0, st_>>>(lf_, hin, hout, sc_, P_,
                                                                                           d_args_, fric, nullptr);
            launches_ += 1;
        }
    }
    // Bottom-up walk of the tree: one launch per level above kBandMaxLevel, then the bands.
    // FULL: encode + threshold + regularise; else scale-only re-encode.
    // a sparse level right below a dense one (both above the bands) is walked inside the
    // dense level's kernel (FOLD): each parent's thread takes its own children there
    bool folded_below(int level) const
    {
        return level - 1 > mw::kBandMaxLevel && level <= L_ - 1 && sparse_level(level) && !sparse_level(level - 1);
    }
    // The proposal's mask of this step's encode / decode (prop_on_: the proposal records or
    // applies; the masked kernels are used on the levels at and below its level C + 1).
    bool prop_on() const { return prop_rec_ || prop_learned_; }
    mw::PropMask prop_mask() const { return mw::PropMask{prop_apply_ ? d_prop_ : nullptr, prop_C_ + 1}; }
    template <bool FULL> void encode_tree(const mw::Hier<T>& h, T eps)
    {
        // the scale re-encode between the RK stages also visits the subtrees whose leaves
        // stage 1 updated (stage 2 reads their parents as neighbours)
        mw::PropMask pm = prop_mask();
        if (!FULL && pm.prop) pm.act = d_act_;
        for (int level = L_ - 1; level > mw::kBandMaxLevel; --level)
        {
            if (folded_below(level)) continue;
            const bool fold = folded_below(level + 1);
            const bool pmk = prop_on() && level + (fold ? 1 : 0) >= pm.level;
            if (sparse_level(level))
            {
                const int nb = grid_for(((int64_t)1 << (2 * level)) / 8, 256, 1 << 30);
                if (pmk) mw::k_level_sparse<T, true, FULL ? 0 : 1, true><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps, pm);
                else if (mw_) mw::k_level_sparse<T, true, FULL ? 0 : 1><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
                else mw::k_level_sparse<T, false, FULL ? 0 : 1><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
            }
            else
            {
                const int nb = grid_for((int64_t)1 << (2 * level), 256, 1 << 30);
                if (pmk && fold) mw::k_encode_level<T, true, FULL, true, true><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps, pm);
                else if (pmk) mw::k_encode_level<T, true, FULL, false, true><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps, pm);
                else if (mw_ && fold) mw::k_encode_level<T, true, FULL, true><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
                else if (mw_) mw::k_encode_level<T, true, FULL><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
                else if (fold) mw::k_encode_level<T, false, FULL, true><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
                else mw::k_encode_level<T, false, FULL><<<nb, 256, 0, st_>>>(h, sc_, L_, level, eps);
            }
            ++launches_;
        }
        for (const Band& b : bands_)
        {
            if (mw_) mw::k_encode_band<T, true, FULL><<<b.grid, 256, 0, st_>>>(h, sc_, L_, b.lo, b.depth, eps, pm);
            else mw::k_encode_band<T, false, FULL><<<b.grid, 256, 0, st_>>>(h, sc_, L_, b.lo, b.depth, eps);
            ++launches_;
        }
    }
    mwdg2_status write_outputs(bool first);
    mwdg2_status write_cumulative(bool first);
    mwdg2_status write_saveint(bool first);
    mwdg2_status write_rasters(bool first);
    mwdg2_status write_vtk();
    mwdg2_status write_c_prop(bool first);
    mwdg2_status sample_stage(std::vector<T>& vals);
    mw::Bnd<T> bnd_now() const;
    int grid_for(int64_t n, int threads, int cap) const
    {
        int64_t b = (n + threads - 1) / threads;
        if (b > cap) b = cap;
        return (int)(b < 1 ? 1 : b);
    }
};

template <typename T> void Sim<T>::release()
{
    if (device_ >= 0) cudaSetDevice(device_);
    for (auto& e : ev_) if (e) { cudaEventDestroy(e); e = nullptr; }
    for (auto& e : ev_step_) if (e) { cudaEventDestroy(e); e = nullptr; }
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second.exec);
    graphs_.clear();
    if (h_args_) { cudaFreeHost(h_args_); h_args_ = nullptr; }
    for (void* p : allocs_) cudaFree(p);
    allocs_.clear();
    if (sc_host_) { cudaFreeHost(sc_host_); sc_host_ = nullptr; }
    if (h_src_) { cudaFreeHost(h_src_); h_src_ = nullptr; }
    h_stage_ = nullptr;   // part of the sc_host_ block
    if (ev_fork_) { cudaEventDestroy(ev_fork_); ev_fork_ = nullptr; }
    if (ev_join_) { cudaEventDestroy(ev_join_); ev_join_ = nullptr; }
    if (st2_) { cudaStreamDestroy(st2_); st2_ = nullptr; }
    if (ev_dec_fork_) { cudaEventDestroy(ev_dec_fork_); ev_dec_fork_ = nullptr; }
    if (ev_dec_join_) { cudaEventDestroy(ev_dec_join_); ev_dec_join_ = nullptr; }
    if (st_dec_) { cudaStreamDestroy(st_dec_); st_dec_ = nullptr; }
    if (st_) { cudaStreamDestroy(st_); st_ = nullptr; }
}

template <typename T> mw::Bnd<T> Sim<T>::bnd_now() const
{
    mw::Bnd<T> b{};
    for (int d = 0; d < 4; ++d)
    {
        b.start[d] = cs_.bnd[d].start;
        b.end[d] = cs_.bnd[d].end;
        b.type[d] = cs_.bnd[d].type;
        b.inlet[d] = cs_.bnd[d].inlet;
    }
    b.west_special = cs_.west_special;
    b.time = time_;
    return b;
}

template <typename T> mwdg2_status Sim<T>::init(const char* par, const mwdg2_opts& o)
{
    opts_ = o;
    if (!cs_.read(par, o.epsilon, o.solver))
        return set_err(cs_.error_kind == 1 ? MWDG2_ERR_IO : MWDG2_ERR_PARSE, cs_.error);
    if (o.dirroot) cs_.dirroot = o.dirroot;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err(MWDG2_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
    if (o.device >= 0) CU(cudaSetDevice(o.device));
    CU(cudaGetDevice(&device_));
    CU(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    mw_ = (cs_.solver == 2);
    L_ = cs_.L;
    M_ = 1 << L_;
    F_ = (int64_t)M_ * M_;
    n_det_ = mw::lvl_idx(L_);
    n_all_ = mw::lvl_idx(L_ + 1);
    D_ = std::min(mw::kTileDepth, L_);
    ntiles_ = 1 << (2 * (L_ - D_));
    for (int hi = std::min(L_ - 1, mw::kBandMaxLevel); hi >= 0; hi -= mw::kBandDepth)
    {
        const int lo = std::max(0, hi - mw::kBandDepth + 1);
        bands_.push_back(Band{lo, hi - lo + 1, 1 << (2 * lo)});
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
    solver_blocks_ = sms * 8;
    red_blocks_ = sms * 4;

    // hierarchy, stage hierarchy, flags
    const int modes = mw_ ? 3 : 1;
    for (int f = 0; f < 4; ++f)
        for (int m = 0; m < 3; ++m)
        {
            hr_.s[f][m] = hs_.s[f][m] = nullptr;
            if (m < modes) { mwdg2_status s = dalloc(hr_.s[f][m], n_all_); if (s) return s; }
            if ((mw_ || m == 0) && f < 3) { mwdg2_status s = dalloc(hs_.s[f][m], n_all_); if (s) return s; }
        }
    if (mwdg2_status s = dalloc(hr_.flags, n_det_)) return s;
    for (int m = 0; m < 3; ++m) hs_.s[3][m] = hr_.s[3][m];
    hs_.flags = hr_.flags;
    // HWFV1: the second buffer starts at zero (only slots that a step writes are ever read)
    if (!mw_)
        for (int f = 0; f < 3; ++f) CU(cudaMemset(hs_.s[f][0], 0, sizeof(T) * (size_t)n_all_));
    // leaves (capacity: every finest cell)
    if (mwdg2_status s = dalloc(lf_.act, F_)) return s;
    if (mwdg2_status s = dalloc(lf_.lvl, F_)) return s;
    // neighbour ids only: a neighbour's level is level_of(id) (the leaf's own across a border)
    for (int d = 0; d < 4; ++d)
    {
        if (mwdg2_status s = dalloc(lf_.nb[d], F_)) return s;
        lf_.nbl[d] = nullptr;
    }
    for (int k = 0; k < 9; ++k)
    {
        lf_.un[k] = nullptr;
        if (mw_ || k % 3 == 0) { if (mwdg2_status s = dalloc(lf_.un[k], F_)) return s; }
    }
    // the step's scalars and the stage-point values sampled at its end share one block, so
    // a single copy brings both back
    const int nst = (int)cs_.stage_codes.size();
    const size_t stage_off = (sizeof(mw::Scalars<T>) + 15) / 16 * 16;
    scal_bytes_ = stage_off + sizeof(T) * 4 * nst;
    {
        char* block = nullptr;
        if (mwdg2_status s = dalloc(block, scal_bytes_)) return s;
        CU(cudaMemset(block, 0, scal_bytes_));
        sc_ = reinterpret_cast<mw::Scalars<T>*>(block);
        if (nst > 0) d_stage_out_ = reinterpret_cast<T*>(block + stage_off);
        char* hblock = nullptr;
        CU(cudaMallocHost(&hblock, scal_bytes_));
        sc_host_ = reinterpret_cast<mw::Scalars<T>*>(hblock);
        if (nst > 0) h_stage_ = reinterpret_cast<T*>(hblock + stage_off);
    }
    if (mwdg2_status s = dalloc(tile_counts_, ntiles_)) return s;
    if (mw_)
    {
        if (mwdg2_status s = dalloc(wet_list_, F_)) return s;
        if (mwdg2_status s = dalloc(dry_, F_)) return s;
        if (mwdg2_status s = dalloc(dry2_, F_)) return s;
        CU(cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking));
        CU(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
    }
    CU(cudaStreamCreateWithFlags(&st_dec_, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&ev_dec_fork_, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ev_dec_join_, cudaEventDisableTiming));
    if (mwdg2_status s = dalloc(d_args_, 1)) return s;
    CU(cudaMallocHost(&h_args_, sizeof(mw::StepArgs<T>)));
    {
        void* m = nullptr;
        if (cudaHostGetDevicePointer(&m, h_args_, 0) == cudaSuccess) m_args_ = static_cast<const mw::StepArgs<T>*>(m);
        cudaGetLastError();
    }
    {
        // persistent grids: SMs x resident blocks of the kernel
        auto resident = [&](auto kernel, int threads) {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0) != cudaSuccess || b < 1) b = 1;
            return b;
        };
        grid_leaf_ = sms * resident(mw::k_leaf_maxima<T>, 256);
        grid_wet_ = sms * resident(mw::k_stage_wet<T, 1>, 256);
        grid_dry_ = sms * resident(mw::k_stage_dry<T, 1>, 256);
        grid_stage_ = sms * (mw_ ? resident(mw::k_mwdg2_stage<T, 1, false>, mw::kSolverThreads)
                                 : resident(mw::k_hwfv1<T>, mw::kSolverThreads));
    }
    const int nsrc = (int)cs_.srcs.size();
    if (nsrc > 0)
    {
        if (mwdg2_status s = dalloc(d_src_, nsrc)) return s;
        CU(cudaMallocHost(&h_src_, sizeof(mw::Src<T>) * nsrc));
        void* m = nullptr;
        if (cudaHostGetDevicePointer(&m, h_src_, 0) == cudaSuccess) m_src_ = static_cast<const mw::Src<T>*>(m);
        cudaGetLastError();
    }
    if (nst > 0)
    {
        if (mwdg2_status s = dalloc(d_stage_codes_, nst)) return s;
        CU(cudaMemcpyAsync(d_stage_codes_, cs_.stage_codes.data(), sizeof(int32_t) * nst, cudaMemcpyHostToDevice, st_));
    }

    // finest level of the hierarchy and the initial leaf state, projected on the device from
    // the rasters (zorder/copy_finest_coefficients.cu:3-35; init.cuh)
    {
        const int fin = mw::lvl_idx(L_);
        T* d_raster = nullptr;
        CU(cudaMalloc(&d_raster, sizeof(T) * 4 * F_));
        for (int f = 0; f < 4; ++f)
        {
            cudaError_t e = cudaMemcpy(d_raster + (size_t)f * F_, cs_.raster[f].data(), sizeof(T) * F_, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { cudaFree(d_raster); CU(e); }
            std::vector<T>().swap(cs_.raster[f]);
        }
        const int grid = grid_for(F_, 256, 1 << 20);
        if (mw_) mw::k_init_finest<T, true><<<grid, 256, 0, st_>>>(d_raster, M_, cs_.xsz, cs_.ysz, hr_, lf_, fin);
        else mw::k_init_finest<T, false><<<grid, 256, 0, st_>>>(d_raster, M_, cs_.xsz, cs_.ysz, hr_, lf_, fin);
        const int nsrc0 = (int)cs_.srcs.size();
        if (nsrc0 > 0)
        {
            // source values at t = 0.001, as the reference's PointSources constructor reads them
            for (int i = 0; i < nsrc0; ++i) h_src_[i] = mw::Src<T>{cs_.srcs[i].code, cs_.srcs[i].type, cs_.srcs[i].value};
            CU(cudaMemcpyAsync(d_src_, h_src_, sizeof(mw::Src<T>) * nsrc0, cudaMemcpyHostToDevice, st_));
            mw::k_init_point_srcs<T><<<1, 1, 0, st_>>>(lf_, hr_, d_src_, nsrc0, T(0.001), cs_.dx, fin);
        }
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
        cudaFree(d_raster);
        CU(e);
    }
    // flags: all significant (mra/init_sig_details.cu) plus preflags
    {
        std::vector<uint8_t> fl(n_det_);
        for (int i = 0; i < n_det_; ++i) fl[i] = mw::F_SIG | (cs_.preflag[i] ? mw::F_PRE : 0);
        CU(cudaMemcpy(hr_.flags, fl.data(), n_det_, cudaMemcpyHostToDevice));
    }

    P_.L = L_; P_.M = M_; P_.xsz = cs_.xsz; P_.ysz = cs_.ysz; P_.limit = cs_.limitslopes ? 1 : 0;
    P_.dx = cs_.dx; P_.tol_h = cs_.tol_h; P_.tol_q = cs_.tol_q; P_.tol_s = cs_.tol_s; P_.g = cs_.g;
    P_.manning = cs_.manning; P_.CFL = cs_.CFL; P_.initial_tstep = cs_.initial_tstep;
    P_.wall_height = cs_.wall_height; P_.tol_Krivo = cs_.tol_Krivo; P_.eps = cs_.epsilon;
    P_.dt_leaf = nullptr;
    if (o.write_outputs && cs_.vtk)
    {
        if (mwdg2_status s = dalloc(d_dt_leaf_, F_)) return s;
        P_.dt_leaf = d_dt_leaf_;
    }

    n_leaves_ = (int)F_;
    mw::k_init_leaves<T><<<grid_for(F_, 256, 4096), 256, 0, st_>>>(lf_, L_, (int)F_);
    // maxima of the initial state (run_simulation.cu:190) then bed encoding with preflags
    // (mra/preflag_topo.cu:3-43)
    mw::k_step_begin<T><<<1, 1, 0, st_>>>(sc_, false);
    mw::k_leaf_maxima<T><<<red_blocks_, 256, 0, st_>>>(lf_, hr_, sc_, (int)F_);
    for (int level = L_ - 1; level >= 0; --level)
    {
        const int nb = grid_for((int64_t)1 << (2 * level), 256, 1 << 24);
        if (mw_) mw::k_topo_level<T, true><<<nb, 256, 0, st_>>>(hr_, sc_, L_, level, cs_.epsilon);
        else mw::k_topo_level<T, false><<<nb, 256, 0, st_>>>(hr_, sc_, L_, level, cs_.epsilon);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st_));
    {
        int32_t nl = (int32_t)F_;
        CU(cudaMemcpy(&sc_->n_leaves, &nl, sizeof(nl), cudaMemcpyHostToDevice));
        int32_t zero = 0;
        CU(cudaMemcpy(&sc_->status, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    }
    if (mwdg2_status st = set_timing(o.verbose >= 2 ? 2 : 0)) return st;
    t_start_ = std::chrono::steady_clock::now();
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::launch_step()
{
    const mwdg2_status st = launch_step_device();
    // HWFV1: the step wrote its result into hs_, which the next step reads as its hierarchy
    if (st == MWDG2_OK && !mw_)
    {
        for (int f = 0; f < 3; ++f) std::swap(hr_.s[f][0], hs_.s[f][0]);
        flip_ = !flip_;
    }
    return st;
}

// host-side values of this step: point-source values (classes/PointSources.h:453-472)
// and boundary inlets (classes/Boundaries.h:28-39) at the current time, and dt
template <typename T> void Sim<T>::prepare_args()
{
    for (auto& src : cs_.srcs)
        if (src.varying) src.value = src.series.at(time_);
    for (int i = 0; i < (int)cs_.srcs.size(); ++i)
        h_src_[i] = mw::Src<T>{cs_.srcs[i].code, cs_.srcs[i].type, cs_.srcs[i].value};
    for (int d = 0; d < 4; ++d)
        if (cs_.bnd[d].varying) cs_.bnd[d].inlet = cs_.bnd[d].series.at(time_);
    h_args_->dt = dt_;
    h_args_->B = bnd_now();
}

template <typename T> mwdg2_status Sim<T>::launch_step_device()
{
    prepare_args();
    // step timing: stream events right around the step's device work (after any capture)
    auto rec_step = [&](int k) { if (timing_mode_ == 1) cudaEventRecord(ev_step_[k], st_); };
    auto direct = [&]() {
        rec_step(0);
        const mwdg2_status st = enqueue_device();
        rec_step(1);
        return st;
    };
    // the first step has its own kernels (initial maxima, full encode); later steps differ
    // only in which RK stages take the wet list
    if (!use_graphs_ || first_) return direct();
    const int key = variant_key();
    if (!graphs_.count(key))
    {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        bool ok = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        capturing_ = ok;
        const mwdg2_status st = ok ? enqueue_device() : MWDG2_OK;
        capturing_ = false;
        if (ok) ok = cudaStreamEndCapture(st_, &g) == cudaSuccess && st == MWDG2_OK;
        if (ok) ok = cudaGraphInstantiate(&ge, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();   // a refused capture leaves its error here; the direct path follows
        if (!ok)
        {
            if (ge) cudaGraphExecDestroy(ge);
            use_graphs_ = false;
            return direct();
        }
        graphs_[key] = Captured{ge, launches_};
    }
    launches_ = graphs_[key].launches;
    rec_step(0);
    CU(cudaGraphLaunch(graphs_[key].exec, st_));
    rec_step(1);
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::enqueue_device()
{
    const bool mw = mw_;
    const T eps = cs_.epsilon;
    // under stream capture the records must be external to become event nodes of the graph
    auto rec = [&](int k) {
        if (!timed_) return;
        if (capturing_) cudaEventRecordWithFlags(ev_[k], st_, cudaEventRecordExternal);
        else cudaEventRecord(ev_[k], st_);
    };
    launches_ = 0;
    rec(0);
    // after the first step: the previous step's last solver kernel (MWDG2 stage 2, or the
    // FV1 kernel into the other buffer) re-inserted the state into the hierarchy and reduced
    // its maxima, so only the point sources remain here
    const bool carry = !first_;
    const int nsrc = (int)cs_.srcs.size();
    // one kernel where nothing runs between the scalar reset and the point sources (MWDG2
    // after its first step) and the pinned buffers are mapped; else copies and two kernels
    const bool open = carry && m_args_ && (nsrc == 0 || m_src_);
    if (open)
    {
        mw::k_step_open<T><<<1, 128, 0, st_>>>(sc_, carry, m_args_, d_args_, m_src_, nsrc, hr_, cs_.dx, L_);
        ++launches_;
    }
    else
    {
        CU(cudaMemcpyAsync(d_args_, h_args_, sizeof(mw::StepArgs<T>), cudaMemcpyHostToDevice, st_));
        mw::k_step_begin<T><<<1, 1, 0, st_>>>(sc_, carry);
        ++launches_;
        const int nfix = first_ ? (int)F_ : -1;
        if (!carry)
        {
            mw::k_leaf_maxima<T><<<grid_leaf_, 256, 0, st_>>>(lf_, hr_, sc_, nfix);
            ++launches_;
        }
        if (nsrc > 0)
        {
            CU(cudaMemcpyAsync(d_src_, h_src_, sizeof(mw::Src<T>) * nsrc, cudaMemcpyHostToDevice, st_));
            mw::k_point_sources<T><<<(nsrc + 127) / 128, 128, 0, st_>>>(hr_, d_src_, nsrc, d_args_, cs_.dx, L_);
            ++launches_;
        }
    }
    rec(1);
    const bool remesh = (eps > T(0) || first_);
    if (prop_on() && remesh)
    {
        // the MLP's proposal (applied or, on judge and fallback steps, only scored against the
        // step's activity): one fused kernel; with recording on, the features are written out
        // for the trainer first and the MLP reads them
        const int64_t tiles = (prop_nC_ + mlp::kRows - 1) / mlp::kRows;
        const int g = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 2 * (int64_t)(solver_blocks_ / 8)));
        if (prop_rec_)
        {
            const int grid = grid_for(prop_nC_, 128, 148 * 16);
            mw::k_prop_features<T><<<grid, 128, 0, st_>>>(hr_, prop_C_, d_lab_, d_feat_);
            ++launches_;
            if (prop_learned_)
            {
                mlp::k_mlp_forward<<<g, mlp::kRows, mlp::FwdSmem::Total + 1024, st_>>>(d_mlp_, d_feat_, prop_nC_, nullptr,
                                                                                     d_prop_, prop_thr_, d_mlp_err_);
                ++launches_;
            }
        }
        else if (prop_learned_ && prop_nC_ >= mlp::kRows)
        {
            mw::k_mlp_propose<T><<<g, mlp::kRows, mw::ProposeSmem<T>::Total + 1024, st_>>>(d_mlp_pack_, hr_, prop_C_, d_lab_,
                                                                                        d_ring_, d_prop_, prop_thr_,
                                                                                        &sc_->status);
            ++launches_;
        }
        if (prop_learned_)
        {
            mw::k_prop_force<<<grid_for(prop_nC_, 256, 2 * (solver_blocks_ / 8)), 256, 0, st_>>>(
                d_prop_, d_lab_, prop_nC_, d_prop_src_, (int)cs_.srcs.size());
            ++launches_;
        }
    }
    if (remesh) encode_tree<true>(hr_, eps);
    rec(2);
    if (remesh)
    {
        for (size_t k = bands_.size(); k-- > 0;)  // top band first
        {
            const Band& b = bands_[k];
            if (mw) mw::k_decode_band<T, true><<<b.grid, 256, 0, st_>>>(hr_, sc_, L_, b.lo, b.depth, eps, prop_mask(), keep_);
            else mw::k_decode_band<T, false><<<b.grid, 256, 0, st_>>>(hr_, sc_, L_, b.lo, b.depth, eps, mw::PropMask{},
                                                                      keep_);
            ++launches_;
        }
        // the levels above the bands: their flags first (extra significance from F_XS), so
        // the flags are final and the leaf topology below can run beside the value decode
        for (int level = mw::kBandMaxLevel + 1; level <= L_ - 2; ++level)
        {
            mw::k_extra_sig_level<T><<<grid_for((int64_t)1 << (2 * level - 2), 256, 1 << 30), 256, 0, st_>>>(hr_.flags, sc_,
                                                                                                            L_, level, eps);
            ++launches_;
        }
    }
    rec(3);
    if (remesh)
    {
        const bool fork = L_ - 1 > mw::kBandMaxLevel;
        if (fork)
        {
            CU(cudaEventRecord(ev_dec_fork_, st_));
            CU(cudaStreamWaitEvent(st_dec_, ev_dec_fork_, 0));
            // (no folding here: a thread decoding a child after its parent lengthens the
            // kernel's tail, while the sparse level's own kernel overlaps the topology)
            const mw::PropMask pm = prop_mask();
            for (int level = mw::kBandMaxLevel + 1; level < L_; ++level)
            {
                const bool pmk = prop_on() && level >= pm.level;
                // keep-values decode: the parents refined this step are few on every level
                if (keep_ || sparse_level(level))
                {
                    const int nb = grid_for(((int64_t)1 << (2 * level)) / 8, 256, 1 << 30);
                    if (pmk) mw::k_level_sparse<T, true, 2, true><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps, pm, keep_);
                    else if (mw) mw::k_level_sparse<T, true, 2><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps, pm, keep_);
                    else mw::k_level_sparse<T, false, 2><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps, pm, keep_);
                }
                else
                {
                    const int nb = grid_for((int64_t)1 << (2 * level), 256, 1 << 30);
                    if (pmk) mw::k_decode_level<T, true, true><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps, pm);
                    else if (mw) mw::k_decode_level<T, true><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps);
                    else mw::k_decode_level<T, false><<<nb, 256, 0, st_dec_>>>(hr_, sc_, L_, level, eps);
                }
                ++launches_;
            }
        }
        // 96 threads: the count reads 85 flag words of the tile's subtree
        mw::k_tile_count<<<ntiles_, 96, 0, st_>>>(hr_.flags, L_, tile_counts_);
        ++launches_;
        mw::k_tile_scan<T><<<1, 1024, 0, st_>>>(tile_counts_, ntiles_, sc_);
        ++launches_;
        mw::k_tile_emit<T, false><<<ntiles_, mw::kTileThreads, 0, st_>>>(lf_, hr_.flags, tile_counts_, L_, M_, cs_.xsz, cs_.ysz,
                                                                        &sc_->min_leaf, &sc_->n_prev);
        ++launches_;
        if (fork)
        {
            CU(cudaEventRecord(ev_dec_join_, st_dec_));
            CU(cudaStreamWaitEvent(st_, ev_dec_join_, 0));
        }
    }
    rec(4);
    const bool fric = cs_.manning > T(0);
    if (!mw)
    {
        mw::k_hwfv1<T><<<grid_stage_, mw::kSolverThreads, 0, st_>>>(lf_, hr_, hs_, sc_, P_, d_args_, fric);
        ++launches_;
        rec(5);
        rec(6);
        rec(7);
    }
    else
    {
        stage<1>(hr_, hs_, fric);
        rec(5);
        if (eps > T(0)) encode_tree<false>(hs_, eps);
        if (cs_.limitslopes) { mw::k_stage2_maxh<T><<<grid_leaf_, 256, 0, st_>>>(lf_, hs_, sc_, P_, d_args_); ++launches_; }
        rec(6);
        stage<2>(hs_, hr_, false);
        rec(7);
    }
    if (prop_on() && remesh)
    {
        mw::k_prop_labels<<<grid_for(prop_nC_, 256, 2 * (solver_blocks_ / 8)), 256, 0, st_>>>(
            d_act_, prop_learned_ ? d_prop_ : nullptr, hr_.flags, prop_C_, d_sig5_, d_lab_, d_ring_, prop_nC_,
            &sc_->prop_active);
        ++launches_;
    }
    // the stage points of the new state come back with the step's scalars
    const int np = (int)cs_.stage_codes.size();
    if (np > 0)
    {
        mw::k_sample_points<T><<<(32 * np + 127) / 128, 128, 0, st_>>>(lf_, hr_, sc_, L_, d_stage_codes_, np, tile_counts_,
                                                                  ntiles_, d_stage_out_);
        ++launches_;
    }
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(sc_host_, sc_, scal_bytes_, cudaMemcpyDeviceToHost, st_));
    rec(8);
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::collect_step()
{
    const bool mw = mw_;
    CU(cudaStreamSynchronize(st_));
    stage_fresh_ = !cs_.stage_codes.empty();
    if (timed_)
    {
        float ms = 0;
        const int pairs[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}, {0, 8}};
        for (int k = 0; k < 8; ++k)
        {
            cudaEventElapsedTime(&ms, ev_[pairs[k][0]], ev_[pairs[k][1]]);
            last_ms_[k] = ms;
        }
    }
    else if (timing_mode_ == 1)
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_step_[0], ev_step_[1]);
        last_ms_[7] = ms;
    }
    if (mw)
        for (int s = 0; s < 2; ++s) wet_prev_[s] = sc_host_->wet[s];
    if (cs_.epsilon > T(0) || first_)   // a step that remeshed counted its significant parents
        for (int l = mw::kBandMaxLevel + 1; l < L_ && l < 16; ++l) sig_prev_[l] = sc_host_->sig_level[l];
    last_cnt_[0] = (int64_t)sc_host_->enc;
    last_cnt_[1] = (int64_t)sc_host_->enc2;
    last_cnt_[2] = (int64_t)sc_host_->dec;
    last_cnt_[3] = sc_host_->n_leaves;
    last_cnt_[4] = n_det_ - 3;
    last_cnt_[5] = launches_;
    last_cnt_[6] = mw ? sc_host_->wet[0] : 0;
    last_cnt_[7] = mw ? sc_host_->wet[1] : 0;
    last_cnt_[8] = (int64_t)(sizeof(mw::StepArgs<T>) + sizeof(mw::Src<T>) * cs_.srcs.size());
    last_cnt_[9] = (int64_t)scal_bytes_;
    last_cnt_[10] = mw ? (int64_t)sc_host_->prop_frozen : 0;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::begin_step()
{
    if (finished_ || !(time_ < cs_.sim_time))
    {
        finished_ = true;
        return MWDG2_DONE;
    }
    CU(cudaSetDevice(device_));
    // the proposal: a judge step every prop_judge_every_ steps, full steps while a fallback lasts
    prop_judge_ = prop_learned_ && !first_ && prop_judge_every_ > 0 && prop_since_judge_ >= prop_judge_every_;
    prop_apply_ = prop_learned_ && !first_ && !prop_judge_ && prop_fallback_left_ == 0;
    // run_simulation.cu:228-235
    time_ += dt_;
    if ((time_ - cs_.sim_time) > T(0))
    {
        time_ -= dt_;
        dt_ = cs_.sim_time - time_;
        time_ += dt_;
    }
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::enqueue_step()
{
    CU(cudaSetDevice(device_));
    return launch_step();
}

template <typename T> mwdg2_status Sim<T>::step(double* dt_out, int64_t* n_out)
{
    mwdg2_status s = begin_step();
    if (s != MWDG2_OK) return s;
    if ((s = launch_step()) != MWDG2_OK) return s;
    return finish_step(dt_out, n_out);
}

template <typename T> mwdg2_status Sim<T>::finish_step(double* dt_out, int64_t* n_out)
{
    CU(cudaSetDevice(device_));
    if (mwdg2_status s = collect_step()) return s;
    if (sc_host_->status & 1) return set_err(MWDG2_ERR_NUMERIC, "NaN in the leaf state");
    if (prop_on())
    {
        // the fused kernel reports through the step's status; the recording path's MLP
        // through its own flag
        int mlp_err = (sc_host_->status & 2) ? 1 : 0;
        if (prop_learned_ && prop_rec_) CU(cudaMemcpy(&mlp_err, d_mlp_err_, sizeof(int), cudaMemcpyDeviceToHost));
        if (mlp_err || (sc_host_->status & 2))
            return set_err(MWDG2_ERR_TIMEOUT, "proposal MLP: a tensor-core wait ran out");
        const double active = sc_host_->prop_active, missed = sc_host_->prop_missed;
        const double needed = sc_host_->prop_needed;
        prop_last_[0] = active;
        prop_last_[1] = missed;
        prop_last_[2] = sc_host_->prop_proposed;
        prop_last_[4] = sc_host_->prop_frozen;
        prop_last_[5] = needed;
        prop_last_[3] = prop_apply_ ? 1.0 : 0.0;
        if (prop_learned_ && !first_)
        {
            const double rate = needed > 0 ? missed / needed : 0.0;
            // the fallback test counts the misses over at least 0.1 % of all subtrees, so
            // that one or two misses among the few dozen active subtrees of a starting flood
            // do not throw the next judge_every steps back to the full step
            const double floor_rate = missed / std::max(needed, 1e-3 * (double)(prop_nC_ * 4));
            ++prop_since_judge_;
            if (prop_judge_)
            {
                ++prop_judge_steps_;
                prop_judge_rate_ = rate;
                prop_since_judge_ = 0;
            }
            else if (prop_apply_) ++prop_learned_steps_;
            else if (prop_fallback_left_ > 0) --prop_fallback_left_;
            if ((prop_judge_ || prop_apply_) && floor_rate > prop_bound_)
            {
                prop_fallback_left_ = prop_judge_every_ > 0 ? prop_judge_every_ : 1;
                ++prop_fallbacks_;
            }
        }
    }
    n_leaves_ = sc_host_->n_leaves;
    dt_ = sc_host_->dt_min;
    first_ = false;
    timestep_++;
    if (dt_out) *dt_out = (double)dt_;
    if (n_out) *n_out = n_leaves_;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::volume(double* out)
{
    CU(cudaSetDevice(device_));
    double* d = nullptr;
    CU(cudaMalloc(&d, sizeof(double)));
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(double), st_);
    if (e == cudaSuccess)
    {
        mw::k_volume<T><<<grid_leaf_, 256, 0, st_>>>(lf_, sc_, L_, d);
        e = cudaGetLastError();
    }
    double v = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    cudaFree(d);
    CU(e);
    *out = v * (double)cs_.dx * (double)cs_.dx;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::freeze_alloc()
{
    if (!lf_.same)
    {
        if (mwdg2_status s = dalloc(lf_.same, F_)) return s;
        CU(cudaMemset(lf_.same, 0, F_));
    }
    if (!clean_tag_)
    {
        if (mwdg2_status s = dalloc(clean_tag_, n_all_)) return s;
        CU(cudaMemset(clean_tag_, 0, sizeof(uint32_t) * (size_t)n_all_));
    }
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::prop_alloc()
{
    if (!mw_) return set_err(MWDG2_ERR_STATE, "the refinement proposal applies to MWDG2 only");
    if (L_ < 4) return set_err(MWDG2_ERR_STATE, "the refinement proposal needs max_ref_lvl >= 4");
    if (d_feat_) return MWDG2_OK;
    prop_C_ = mw::proposal_level(L_);
    prop_nC_ = (int64_t)1 << (2 * prop_C_);
    if (mwdg2_status s = dalloc(d_feat_, (size_t)prop_nC_ * mlp::kIn)) return s;
    if (mwdg2_status s = dalloc(d_lab_, (size_t)prop_nC_)) return s;
    const size_t nring = (size_t)std::max<int64_t>(1, prop_nC_ / mw::kPropTile);
    if (mwdg2_status s = dalloc(d_ring_, nring)) return s;
    CU(cudaMemset(d_ring_, 0xff, nring * sizeof(uint16_t)));   // every tile runs until labels exist
    {
        std::vector<int32_t> nodes;
        for (const auto& src : cs_.srcs) nodes.push_back(src.code >> (2 * (L_ - (prop_C_ + 1))));
        if (mwdg2_status s = dalloc(d_prop_src_, std::max<size_t>(1, nodes.size()))) return s;
        if (!nodes.empty())
            CU(cudaMemcpy(d_prop_src_, nodes.data(), sizeof(int32_t) * nodes.size(), cudaMemcpyHostToDevice));
    }
    if (mwdg2_status s = freeze_alloc()) return s;
    if (mwdg2_status s = dalloc(d_act_, (size_t)prop_nC_ * 4)) return s;
    if (mwdg2_status s = dalloc(d_prop_, (size_t)prop_nC_ * 4)) return s;
    if (mwdg2_status s = dalloc(d_sig5_, (size_t)prop_nC_ * 4)) return s;
    CU(cudaMemset(d_sig5_, 0, (size_t)prop_nC_ * 4));
    if (mwdg2_status s = dalloc(d_mlp_, mlp::kParams)) return s;
    if (mwdg2_status s = dalloc(d_mlp_pack_, mlp::kPackBytes)) return s;
    if (mwdg2_status s = dalloc(d_mlp_err_, 1)) return s;
    CU(cudaMemset(d_lab_, 0, (size_t)prop_nC_));
    CU(cudaMemset(d_act_, 0, (size_t)prop_nC_ * 4));
    CU(cudaMemset(d_prop_, 1, (size_t)prop_nC_ * 4));
    CU(cudaMemset(d_mlp_err_, 0, sizeof(int)));
    CU(cudaFuncSetAttribute(mlp::k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(mlp::FwdSmem::Total + 1024)));
    CU(cudaFuncSetAttribute(mw::k_mlp_propose<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(mw::ProposeSmem<T>::Total + 1024)));
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::proposal_record(bool on)
{
    CU(cudaSetDevice(device_));
    if (on) { if (mwdg2_status s = prop_alloc()) return s; }
    prop_rec_ = on;
    P_.act = prop_on() ? d_act_ : nullptr;
    P_.act_level = prop_C_ + 1;
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second.exec);   // they hold the old parameters
    graphs_.clear();
    return MWDG2_OK;
}

template <typename T>
mwdg2_status Sim<T>::proposal_enable(const float* params, int judge_every, float threshold, float miss_bound)
{
    CU(cudaSetDevice(device_));
    if (!params)
    {
        prop_learned_ = false;
        return proposal_record(prop_rec_);
    }
    if (mwdg2_status s = prop_alloc()) return s;
    CU(cudaMemcpy(d_mlp_, params, sizeof(float) * mlp::kParams, cudaMemcpyHostToDevice));
    mlp::k_mlp_pack<<<1, mlp::kRows, 0, st_>>>(d_mlp_, d_mlp_pack_);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st_));
    prop_learned_ = true;
    prop_judge_every_ = judge_every;
    prop_thr_ = threshold;
    prop_bound_ = miss_bound;
    prop_since_judge_ = judge_every;   // the first step after enabling is a judge step
    prop_fallback_left_ = 0;
    return proposal_record(prop_rec_);
}

template <typename T> mwdg2_status Sim<T>::proposal_stats(double* out, int n)
{
    const double nodes = (double)(prop_nC_ * 4);
    const double v[12] = {prop_last_[0], prop_last_[1], prop_last_[2], prop_last_[3], nodes, (double)prop_learned_steps_,
                          (double)prop_judge_steps_, prop_judge_rate_, (double)prop_fallbacks_, (double)prop_fallback_left_,
                          prop_last_[4], prop_last_[5]};
    for (int i = 0; i < n && i < 12; ++i) out[i] = v[i];
    return MWDG2_OK;
}

template <typename T>
mwdg2_status Sim<T>::proposal_samples(const void** feats, const uint8_t** labels, int64_t* n, int* device)
{
    if (!prop_on() || first_) return set_err(MWDG2_ERR_STATE, "no step recorded proposal features yet");
    CU(cudaSetDevice(device_));
    CU(cudaStreamSynchronize(st_));
    *feats = d_feat_;
    *labels = d_lab_;
    *n = prop_nC_;
    *device = device_;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::proposal_samples_host(float* feats, uint8_t* labels, int64_t cap, int64_t* n)
{
    const void* df = nullptr;
    const uint8_t* dl = nullptr;
    int64_t m = 0;
    int dev = 0;
    if (mwdg2_status s = proposal_samples(&df, &dl, &m, &dev)) return s;
    if (n) *n = m;
    if (cap < m) return set_err(MWDG2_ERR_ARG, "capacity below the number of coarse cells");
    if (feats)
    {
        std::vector<uint16_t> h((size_t)m * mlp::kIn);
        CU(cudaMemcpy(h.data(), df, h.size() * 2, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < h.size(); ++i)
        {
            const uint32_t u = (uint32_t)h[i] << 16;
            std::memcpy(feats + i, &u, 4);
        }
    }
    if (labels) CU(cudaMemcpy(labels, dl, (size_t)m, cudaMemcpyDeviceToHost));
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::sample_stage(std::vector<T>& vals)
{
    const int np = (int)cs_.stage_codes.size();
    vals.assign(4 * (size_t)np, T(0));
    if (np == 0) return MWDG2_OK;
    if (stage_fresh_)   // sampled by the last step
    {
        std::copy(h_stage_, h_stage_ + 4 * (size_t)np, vals.begin());
        return MWDG2_OK;
    }
    // before the first step: the leaf list is every finest cell and no tile offsets exist
    mw::k_sample_points<T><<<(32 * np + 127) / 128, 128, 0, st_>>>(lf_, hr_, sc_, L_, d_stage_codes_, np, nullptr, 0,
                                                              d_stage_out_);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(vals.data(), d_stage_out_, sizeof(T) * 4 * np, cudaMemcpyDeviceToHost, st_));
    CU(cudaStreamSynchronize(st_));
    return MWDG2_OK;
}

// output/write_stage_point_data.cu:3-193 and output/write_cumulative_data.cpp:3-53
template <typename T> mwdg2_status Sim<T>::write_outputs(bool first)
{
    const char* fmt = "%lf";  // NUM_FRMT: "%lf" and "%f" print alike
    auto inv = [](int code, int& i, int& j) {
        i = mw::compact(code);
        j = mw::compact(code >> 1);
    };
    if (cs_.cumulative)
    {
        if (mwdg2_status s = write_cumulative(first)) return s;
    }
    const int np = (int)cs_.stage_codes.size();
    if (np == 0) return MWDG2_OK;
    std::vector<T> v;
    if (mwdg2_status s = sample_stage(v)) return s;
    const std::string base = cs_.dirroot + "/" + cs_.resroot;
    FILE* fh = fopen((base + ".stage").c_str(), first ? "w" : "a");
    FILE* fx = fopen((base + ".xvelocity").c_str(), first ? "w" : "a");
    FILE* fy = fopen((base + ".yvelocity").c_str(), first ? "w" : "a");
    if (!fh || !fx || !fy)
    {
        if (fh) fclose(fh);
        if (fx) fclose(fx);
        if (fy) fclose(fy);
        return set_err(MWDG2_ERR_IO, "cannot write stage files under " + cs_.dirroot);
    }
    const T dx = cs_.dx;
    auto header = [&](FILE* f, const char* title, const char* what) {
        fprintf(f, "%s\n\n", title);
        fprintf(f, "Stage information (stage,x,y,elev):\n");
        for (int p = 0; p < np; ++p)
        {
            int i, j;
            inv(cs_.stage_codes[p], i, j);
            fprintf(f, "%d %lf %lf %lf\n", p + 1, (double)(i * dx + dx / T(2.0)), (double)(j * dx + dx / T(2.0)),
                    (double)v[4 * p + 3]);
        }
        fprintf(f, "\nOutput, %s:\n", what);
        fprintf(f, "Time; stages 1 to %d\n", np);
    };
    if (first)
    {
        header(fh, "Stage output, depth (m).", "depths");
        if (cs_.voutput_stage)
        {
            header(fx, "Stage output, x velocity (m/s).", "x velocities");
            header(fy, "Stage output, y velocity (m/s).", "y velocities");
        }
    }
    fprintf(fh, "%lf ", (double)time_);
    if (cs_.voutput_stage) { fprintf(fx, "%lf ", (double)time_); fprintf(fy, "%lf ", (double)time_); }
    for (int p = 0; p < np; ++p)
    {
        const bool last = (p + 1 == np);
        const T h = v[4 * p + 0];
        fprintf(fh, last ? "%lf" : "%lf ", (double)h);
        if (cs_.voutput_stage)
        {
            const T vx = (h < cs_.tol_h) ? T(0.0) : v[4 * p + 1] / h;
            const T vy = (h < cs_.tol_h) ? T(0.0) : v[4 * p + 2] / h;
            fprintf(fx, last ? "%lf" : "%lf ", (double)vx);
            fprintf(fy, last ? "%lf" : "%lf ", (double)vy);
        }
    }
    (void)fmt;
    fprintf(fh, "\n");
    if (cs_.voutput_stage) { fprintf(fx, "\n"); fprintf(fy, "\n"); }
    fclose(fh);
    fclose(fx);
    fclose(fy);
    return MWDG2_OK;
}

// output/write_cumulative_data.cpp:3-53 (runtime columns: host wall seconds of this loop)
template <typename T> mwdg2_status Sim<T>::write_cumulative(bool first)
{
    const std::string path = cs_.dirroot + "/" + cs_.resroot + ".cumu";
    FILE* fp = fopen(path.c_str(), first ? "w" : "a");
    if (!fp) return set_err(MWDG2_ERR_IO, "cannot write " + path);
    if (first) fprintf(fp, "simtime,runtime_mra,runtime_solver,runtime_total,dt,reduction\n");
    const T comp = (T(100.0) - T(100.0) * n_leaves_ / T(cs_.xsz * cs_.ysz)) / T(100.0);
    fprintf(fp, "%lf,%lf,%lf,%lf,%lf,%lf\n", (double)time_, time_mra_, time_solver_, time_mra_ + time_solver_,
            (double)dt_, (double)comp);
    fclose(fp);
    return MWDG2_OK;
}

namespace {

// Value format of the reference's text outputs (types/real.h: "%" NUM_FIG NUM_FRMT).
template <typename T> const char* fig_fmt() { return sizeof(T) == 8 ? "%.15lf" : "%.8f"; }

// Formats `rows` text rows with fmt_row(r, out) on the host's threads and writes them in
// order (the large rasters and VTK sections are tens of millions of printf conversions).
template <typename RowFn> bool write_rows(FILE* fp, int64_t rows, RowFn fmt_row)
{
    const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const int64_t batch = (int64_t)nt * 256;
    std::vector<std::string> buf((size_t)std::min<int64_t>(batch, std::max<int64_t>(rows, 1)));
    for (int64_t r0 = 0; r0 < rows; r0 += batch)
    {
        const int64_t nr = std::min(batch, rows - r0);
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int64_t r = t; r < nr; r += nt)
                {
                    buf[r].clear();
                    fmt_row(r0 + r, buf[r]);
                }
            });
        for (auto& x : th) x.join();
        for (int64_t r = 0; r < nr; ++r)
            if (fwrite(buf[r].data(), 1, buf[r].size(), fp) != buf[r].size()) return false;
    }
    return true;
}

void append_fmt(std::string& out, const char* fmt, double v)
{
    char tmp[64];
    const int k = snprintf(tmp, sizeof(tmp), fmt, v);
    out.append(tmp, (size_t)std::max(0, std::min(k, (int)sizeof(tmp) - 1)));
}

} // namespace

// run_simulation.cu:656-703
template <typename T> mwdg2_status Sim<T>::write_saveint(bool first)
{
    if (cs_.vtk) { if (mwdg2_status s = write_vtk()) return s; }
    if (cs_.raster_out) { if (mwdg2_status s = write_rasters(first)) return s; }
    if (cs_.c_prop) { if (mwdg2_status s = write_c_prop(first)) return s; }
    return MWDG2_OK;
}

// output/write_all_raster_maps{,_dg2,_fv1}.cu and output/write_raster_file.cu: ESRI ASCII
// maps <dirroot>/<resroot>-<save index>.{elev,wd,qx,qy,vx,vy} and, at the first step, .dem.
template <typename T> mwdg2_status Sim<T>::write_rasters(bool first)
{
    struct Map { const char* ext; int field; bool on; };
    const Map maps[] = {{"elev", mw::R_ETA, !cs_.elevoff}, {"wd", mw::R_H, !cs_.depthoff},
                        {"qx", mw::R_QX, cs_.qoutput}, {"qy", mw::R_QY, cs_.qoutput},
                        {"vx", mw::R_VX, cs_.voutput}, {"vy", mw::R_VY, cs_.voutput},
                        {"dem", mw::R_Z, first}};
    unsigned fields = 0;
    for (const Map& m : maps) if (m.on) fields |= 1u << m.field;
    if (!fields) return MWDG2_OK;
    const int nx = cs_.xsz, ny = cs_.ysz;
    const size_t N = (size_t)nx * ny;
    if (!d_raster_) { if (mwdg2_status s = dalloc(d_raster_, mw::R_COUNT * N)) return s; }
    const int grid = grid_for((int64_t)N, 256, 1 << 20);
    if (mw_) mw::k_raster<T, true><<<grid, 256, 0, st_>>>(lf_, hr_, sc_, L_, nx, ny, cs_.tol_h, fields, d_raster_);
    else mw::k_raster<T, false><<<grid, 256, 0, st_>>>(lf_, hr_, sc_, L_, nx, ny, cs_.tol_h, fields, d_raster_);
    CU(cudaGetLastError());
    std::vector<T> host(N);
    const char* vf = fig_fmt<T>();
    const std::string vfs = std::string(vf) + " ";
    for (const Map& m : maps)
    {
        if (!m.on) continue;
        CU(cudaMemcpyAsync(host.data(), d_raster_ + (size_t)m.field * N, sizeof(T) * N, cudaMemcpyDeviceToHost, st_));
        CU(cudaStreamSynchronize(st_));
        const std::string path =
            cs_.dirroot + "/" + cs_.resroot + "-" + std::to_string(cs_.saveint_count - 1) + "." + m.ext;
        FILE* fp = fopen(path.c_str(), "w");
        if (!fp) return set_err(MWDG2_ERR_IO, "cannot write raster " + path);
        fprintf(fp, "ncols        %d\n", nx);
        fprintf(fp, "nrows        %d\n", ny);
        fprintf(fp, "xllcorner    %lf\n", (double)cs_.xmin);
        fprintf(fp, "yllcorner    %lf\n", (double)cs_.ymin);
        fprintf(fp, "cellsize     %lf\n", (double)cs_.dx);
        fprintf(fp, "NODATA_value %d\n", -9999);
        const bool ok = write_rows(fp, ny, [&](int64_t r, std::string& out) {
            const T* row = host.data() + (size_t)(ny - 1 - r) * nx;   // top row first
            for (int i = 0; i < nx; ++i) append_fmt(out, vfs.c_str(), (double)row[i]);
            out.push_back('\n');
        });
        fclose(fp);
        if (!ok) return set_err(MWDG2_ERR_IO, "cannot write raster " + path);
    }
    return MWDG2_OK;
}

// output/write_soln_vtk.cu:3-222: one quad per leaf with its CFL step and mode-0 state.
template <typename T> mwdg2_status Sim<T>::write_vtk()
{
    const int n = n_leaves_;
    std::vector<int32_t> act(n);
    std::vector<uint8_t> lvl(n);
    std::vector<double> st(12 * (size_t)n);
    std::vector<T> dtl(n);
    CU(cudaMemcpyAsync(act.data(), lf_.act, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st_));
    CU(cudaMemcpyAsync(lvl.data(), lf_.lvl, n, cudaMemcpyDeviceToHost, st_));
    CU(cudaMemcpyAsync(dtl.data(), d_dt_leaf_, sizeof(T) * n, cudaMemcpyDeviceToHost, st_));
    CU(cudaStreamSynchronize(st_));
    if (mwdg2_status s = state(st.data(), 12LL * n)) return s;
    const std::string path = cs_.dirroot + "/" + cs_.resroot + "-" + std::to_string(cs_.saveint_count - 1) + ".vtk";
    FILE* fp = fopen(path.c_str(), "w");
    if (!fp) return set_err(MWDG2_ERR_IO, "cannot write " + path);
    fprintf(fp, "# vtk DataFile Version 3.0\nMultiresolution flow and topo data\nASCII\n\n"
                "DATASET UNSTRUCTURED_GRID\nPOINTS %d float\n", n * 4);
    const T dx = cs_.dx, xmin = cs_.xmin, ymin = cs_.ymin;
    bool ok = write_rows(fp, n, [&](int64_t i, std::string& out) {
        const int l = lvl[i];
        const int code = act[i] - mw::lvl_idx(l);
        const T size = dx * T(1 << (L_ - l));
        const int x = mw::compact(code), y = mw::compact(code >> 1);
        const T xs[4] = {xmin + x * size, xmin + x * size, xmin + (x + 1) * size, xmin + (x + 1) * size};
        const T ys[4] = {ymin + y * size, ymin + (y + 1) * size, ymin + y * size, ymin + (y + 1) * size};
        for (int k = 0; k < 4; ++k)
        {
            append_fmt(out, "%lf ", (double)xs[k]);
            append_fmt(out, "%lf ", (double)ys[k]);
            append_fmt(out, "%lf\n", 1.0);
        }
    });
    fprintf(fp, "\nCELLS %d %d\n", n, n * 5);
    ok = ok && write_rows(fp, n, [&](int64_t i, std::string& out) {
        char tmp[96];
        const int p = (int)i * 4;
        out.append(tmp, (size_t)snprintf(tmp, sizeof(tmp), "4 %d %d %d %d\n", p, p + 1, p + 2, p + 3));
    });
    fprintf(fp, "\nCELL_TYPES %d\n", n);
    for (int i = 0; i < n; ++i) fputs("8\n", fp);
    fprintf(fp, "\nCELL_DATA %d\n", n);
    const size_t N = (size_t)n;
    auto scalars = [&](const char* name, auto value) {
        fprintf(fp, "\nSCALARS %s float 1\nLOOKUP_TABLE default\n", name);
        return write_rows(fp, n, [&](int64_t i, std::string& out) { append_fmt(out, "%lf\n", (double)value(i)); });
    };
    ok = ok && scalars("dt", [&](int64_t i) { return dtl[i]; });
    ok = ok && scalars("h", [&](int64_t i) { return (T)st[0 * N + i]; });
    ok = ok && scalars("qx", [&](int64_t i) { return (T)st[1 * N + i]; });
    ok = ok && scalars("qy", [&](int64_t i) { return (T)st[2 * N + i]; });
    ok = ok && scalars("z", [&](int64_t i) { return (T)st[3 * N + i]; });
    ok = ok && scalars("eta", [&](int64_t i) { return (T)((T)st[0 * N + i] + (T)st[3 * N + i]); });
    fclose(fp);
    if (!ok) return set_err(MWDG2_ERR_IO, "cannot write " + path);
    return MWDG2_OK;
}

// output/write_c_prop_data.cu:3-81 and output/append_reals_to_file.cu:3-48: the cumulative
// line, then one CSV row per save of each discharge mode over the leaves, appended to
// <dirroot><name>.csv (the reference joins the two without a separator).
template <typename T> mwdg2_status Sim<T>::write_c_prop(bool first)
{
    if (mwdg2_status s = write_cumulative(first)) return s;
    const int n = n_leaves_;
    struct Col { const char* name; int k; };
    const Col cols[] = {{"qx0-c-prop", 3}, {"qy0-c-prop", 6}, {"qx1x-c-prop", 4}, {"qx1y-c-prop", 5},
                        {"qy1x-c-prop", 7}, {"qy1y-c-prop", 8}};
    const int ncols = mw_ ? 6 : 2;
    std::vector<T> v(n);
    const std::string vf = std::string(fig_fmt<T>()) + ",";
    for (int c = 0; c < ncols; ++c)
    {
        CU(cudaMemcpyAsync(v.data(), lf_.un[cols[c].k], sizeof(T) * n, cudaMemcpyDeviceToHost, st_));
        CU(cudaStreamSynchronize(st_));
        const std::string path = cs_.dirroot + cols[c].name + ".csv";
        FILE* fp = fopen(path.c_str(), first ? "w" : "a");
        if (!fp) return set_err(MWDG2_ERR_IO, "cannot write " + path);
        const int64_t per = 4096;
        const bool ok = write_rows(fp, (n + per - 1) / per, [&](int64_t r, std::string& out) {
            const int64_t hi = std::min<int64_t>(n, (r + 1) * per);
            for (int64_t i = r * per; i < hi; ++i) append_fmt(out, vf.c_str(), (double)v[i]);
        });
        fputs("\n", fp);
        fclose(fp);
        if (!ok) return set_err(MWDG2_ERR_IO, "cannot write " + path);
    }
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::prepare_outputs()
{
    if (!opts_.write_outputs) return MWDG2_OK;
    // classes/PlottingParams.h:55-60 (mkdir dirroot)
    if (mkdir(cs_.dirroot.c_str(), 0755) != 0 && errno != EEXIST)
        return set_err(MWDG2_ERR_IO, "cannot create output directory " + cs_.dirroot);
    return MWDG2_OK;
}

// Everything the reference's loop does after the solver (run_simulation.cu:656-766): saveint
// writes VTK / raster maps / c-prop data; massint writes res.cumu (if `cumulative`) and the
// stage files; the periodic progress line.
template <typename T> mwdg2_status Sim<T>::after_step(bool first, double dt, int64_t n, double step_seconds)
{
    time_solver_ += step_seconds;
    if (opts_.write_outputs)
    {
        if (time_ >= cs_.saveint * cs_.saveint_count)
        {
            cs_.saveint_count++;
            if (mwdg2_status so = write_saveint(first)) return so;
        }
        if (time_ >= cs_.massint * cs_.massint_count)
        {
            cs_.massint_count++;
            if (mwdg2_status so = write_outputs(first)) return so;
        }
    }
    if (opts_.verbose && (timestep_ - 1) % 10000 == 1)
    {
        const double comp = 100.0 - 100.0 * n / ((double)cs_.xsz * cs_.ysz);
        printf("Elements: %lld, compression: %f%%, time step: %f, timestep: %d, sim time: %f\n", (long long)n, comp,
               dt, timestep_ - 1, (double)time_);
    }
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::run(int64_t max_steps, int64_t* steps, int64_t* updates)
{
    int64_t done = 0, upd = 0;
    if (mwdg2_status s = prepare_outputs()) return s;
    while (max_steps <= 0 || done < max_steps)
    {
        const bool first = first_;
        double dt;
        int64_t n;
        const auto t0 = std::chrono::steady_clock::now();
        mwdg2_status s = step(&dt, &n);
        if (s == MWDG2_DONE) break;
        if (s != MWDG2_OK) return s;
        ++done;
        upd += n;
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (mwdg2_status so = after_step(first, dt, n, secs)) return so;
    }
    if (steps) *steps = done;
    if (updates) *updates = upd;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::info(double* out, int n)
{
    if (!out || n < 14) return set_err(MWDG2_ERR_ARG, "info: need 14 slots");
    const double v[14] = {(double)time_, (double)dt_, (double)timestep_, (double)n_leaves_, (double)L_, (double)cs_.xsz,
                          (double)cs_.ysz, (double)cs_.dx, (double)cs_.epsilon, (double)cs_.solver,
                          (double)(sizeof(T) * 8), (double)cs_.sim_time, (double)n_det_, (double)n_all_};
    for (int i = 0; i < 14; ++i) out[i] = v[i];
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::leaves(int32_t* a, int32_t* l, int32_t* ids, int32_t* lv, int64_t cap)
{
    const int n = n_leaves_;
    if (cap < n) return set_err(MWDG2_ERR_ARG, "get_leaves: capacity below the leaf count");
    CU(cudaSetDevice(device_));
    if (a) CU(cudaMemcpy(a, lf_.act, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> tmp(n);
    if (l)
    {
        CU(cudaMemcpy(tmp.data(), lf_.lvl, n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) l[i] = tmp[i];
    }
    if (lv && !l) CU(cudaMemcpy(tmp.data(), lf_.lvl, n, cudaMemcpyDeviceToHost));
    std::vector<int32_t> nb(lv ? n : 0);
    for (int d = 0; d < 4; ++d)
    {
        int32_t* dst = ids ? ids + (size_t)d * n : (lv ? nb.data() : nullptr);
        if (dst) CU(cudaMemcpy(dst, lf_.nb[d], sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        if (lv)
            for (int i = 0; i < n; ++i) lv[(size_t)d * n + i] = dst[i] == -1 ? (int32_t)tmp[i] : mw::level_of(dst[i]);
    }
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::state(double* out, int64_t cap)
{
    const int n = n_leaves_;
    if (!out || cap < 12LL * n) return set_err(MWDG2_ERR_ARG, "get_state: need 12 x n_leaves doubles");
    CU(cudaSetDevice(device_));
    if (!d_state_scratch_) { if (mwdg2_status s = dalloc(d_state_scratch_, 12 * F_)) return s; }
    mw::k_gather_state<T><<<grid_for(n, 256, 4096), 256, 0, st_>>>(lf_, hr_, sc_, mw_, d_state_scratch_);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, d_state_scratch_, sizeof(double) * 12 * (size_t)n, cudaMemcpyDeviceToHost, st_));
    CU(cudaStreamSynchronize(st_));
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::sig(uint8_t* out, int64_t cap)
{
    if (!out || cap < n_det_) return set_err(MWDG2_ERR_ARG, "get_sig: need n_details bytes");
    CU(cudaSetDevice(device_));
    CU(cudaMemcpy(out, hr_.flags, n_det_, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n_det_; ++i) out[i] = (out[i] & mw::F_SIG) ? 1 : 0;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::hierarchy(int f, int m, double* out, int64_t cap)
{
    if (f < 0 || f > 3 || m < 0 || m > 2 || !out || cap < n_all_) return set_err(MWDG2_ERR_ARG, "get_hierarchy: bad arguments");
    if (!hr_.s[f][m]) return set_err(MWDG2_ERR_ARG, "get_hierarchy: HWFV1 holds mode 0 only");
    CU(cudaSetDevice(device_));
    std::vector<T> tmp(n_all_);
    CU(cudaMemcpy(tmp.data(), hr_.s[f][m], sizeof(T) * n_all_, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n_all_; ++i) out[i] = tmp[i];
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::stage(double* out, int n)
{
    const int np = (int)cs_.stage_codes.size();
    if (!out || n < np) return set_err(MWDG2_ERR_ARG, "read_stage: buffer smaller than the number of stage points");
    CU(cudaSetDevice(device_));
    std::vector<T> v;
    if (mwdg2_status s = sample_stage(v)) return s;
    for (int p = 0; p < np; ++p) out[p] = v[4 * p];
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::timing(double* out, int n)
{
    for (int i = 0; i < n && i < 8; ++i) out[i] = last_ms_[i];
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::set_timing(int mode)
{
    if (mode < 0 || mode > 2) return set_err(MWDG2_ERR_ARG, "set_timing: mode 0, 1 or 2");
    CU(cudaSetDevice(device_));
    if (mode == 2 && !ev_[0])
        for (auto& e : ev_) CU(cudaEventCreate(&e));
    if (mode == 1 && !ev_step_[0])
        for (auto& e : ev_step_) CU(cudaEventCreate(&e));
    timing_mode_ = mode;
    timed_ = (mode == 2);
    for (auto& v : last_ms_) v = 0.0;
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::decode_mode(int mode)
{
    if (mode < 0 || mode > 1) return set_err(MWDG2_ERR_ARG, "set_decode_mode: mode 0 or 1");
    CU(cudaSetDevice(device_));
    if (mode == 1 && mw_ && !d_keep_prop_)
    {
        if (mwdg2_status s = freeze_alloc()) return s;
        const int C = mw::proposal_level(L_);
        const int64_t n = (int64_t)1 << (2 * (C + 1));
        std::vector<uint8_t> mask((size_t)n, 0);
        for (const auto& src : cs_.srcs) mask[(size_t)(src.code >> (2 * (L_ - (C + 1))))] = 1;
        if (mwdg2_status s = dalloc(d_keep_prop_, (size_t)n)) return s;
        CU(cudaMemcpy(d_keep_prop_, mask.data(), (size_t)n, cudaMemcpyHostToDevice));
        prop_C_ = C;
        if (mwdg2_status s = dalloc(hs_tag_, n_all_)) return s;
    }
    keep_ = (mode == 1);
    if (mw_)
    {
        // no slot counts as current from before the switch (on the simulation's stream, ahead
        // of its next step: the legacy stream does not order with a non-blocking stream)
        if (hs_tag_) CU(cudaMemsetAsync(hs_tag_, 0xff, sizeof(uint32_t) * (size_t)n_all_, st_));
        hs_.tag = keep_ ? hs_tag_ : nullptr;
    }
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second.exec);   // they hold the old kernel arguments
    graphs_.clear();
    return MWDG2_OK;
}

template <typename T> mwdg2_status Sim<T>::counters(int64_t* out, int n)
{
    for (int i = 0; i < n && i < 11; ++i) out[i] = last_cnt_[i];
    return MWDG2_OK;
}

} // namespace

// Internal: lets other translation units of the library set the mwdg2_last_error text.
void mwdg2_detail_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

mwdg2_status mwdg2_detail_proposal_samples(mwdg2_sim* sim, const void** feats, const uint8_t** labels, int64_t* n,
                                           int* device);

// ============================================================================ batched ensembles

namespace {

// A size class of batch members (same max_ref_lvl, MWDG2, same precision, past their first
// step): one launch per kernel steps every member of the class (csrc/batch.cuh), the
// launches captured once into one CUDA graph. The members keep their own state, clocks and
// outputs (Sim); the group only replaces their launches.
struct GroupBase
{
    virtual ~GroupBase() = default;
    // Launch one step of the members with stepping[k] (member k of the group; their
    // begin_step has run); the others are skipped by every kernel.
    virtual mwdg2_status launch(const std::vector<uint8_t>& stepping) = 0;
    virtual mwdg2_status wait() = 0;
    std::vector<int> idx;   // the members' indices in the batch
    int key = -1;
};

template <typename T> class Group final : public GroupBase
{
public:
    ~Group() override
    {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (d_on_) cudaFree(d_on_);
        if (d_map_) cudaFree(d_map_);
        if (h_map_) cudaFreeHost(h_map_);
        if (h_active_) cudaFreeHost(h_active_);
        for (auto& e : ev_)
            if (e) cudaEventDestroy(e);
        if (st2_) cudaStreamDestroy(st2_);
        if (st_) cudaStreamDestroy(st_);
    }

    mwdg2_status build(const std::vector<Sim<T>*>& ms)
    {
        ms_ = ms;
        n_ = (int)ms.size();
        const Sim<T>& m0 = *ms[0];
        L_ = m0.L_;
        ntiles_ = m0.ntiles_;
        bands_ = m0.bands_;
        CU(cudaSetDevice(m0.device_));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m0.device_);
        // per-leaf launches: the device's resident blocks of the kernel, shared among the
        // members by the block maps (plus one block per member, the rounding's room)
        auto capacity = [&](auto kernel, int threads) {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0) != cudaSuccess || b < 1) b = 1;
            return sms * b;
        };
        cap_wet_ = capacity(mw::k_members_stage_wet<T, 1>, 256);
        cap_dry_ = capacity(mw::k_members_stage_dry<T, 1>, 256);
        cap_list_ = capacity(mw::k_members_stage_list<T, 1>, mw::kSolverThreads);
        cap_leaf_ = capacity(mw::k_members_stage2_maxh<T>, 256);
        if (n_ > mw::MemberTable<T>::kMax) return set_err(MWDG2_ERR_STATE, "batch group larger than its table");
        tab_ = std::make_unique<mw::MemberTable<T>>();
        for (int k = 0; k < n_; ++k)
        {
            const Sim<T>& m = *ms[k];
            mw::MemberArgs<T>& a = tab_->m[k];
            a.sc = m.sc_;
            a.sc_host = m.sc_host_;
            a.scal_bytes = (int)m.scal_bytes_;
            a.m_args = m.m_args_;
            a.d_args = m.d_args_;
            a.m_src = m.m_src_;
            a.nsrc = (int)m.cs_.srcs.size();
            a.hr = m.hr_;
            a.hs = m.hs_;
            a.lf = m.lf_;
            a.P = m.P_;
            a.dx = m.cs_.dx;
            a.eps = m.cs_.epsilon;
            a.M = m.M_;
            a.xsz = m.cs_.xsz;
            a.ysz = m.cs_.ysz;
            a.tile_counts = m.tile_counts_;
            a.dry1 = m.dry_;
            a.dry2 = m.dry2_;
            a.wet = m.wet_list_;
            a.fric = m.cs_.manning > T(0) ? 1 : 0;
            a.limit = m.cs_.limitslopes ? 1 : 0;
            a.stage_codes = m.d_stage_codes_;
            a.np = (int)m.cs_.stage_codes.size();
            a.stage_out = m.d_stage_out_;
            np_max_ = std::max(np_max_, a.np);
        }
        CU(cudaMalloc(&d_on_, n_));
        const size_t nmap = (size_t)mw::kBlockMaps * (n_ + 1);
        CU(cudaMalloc(&d_map_, sizeof(int32_t) * nmap));
        CU(cudaHostAlloc(&h_map_, sizeof(int32_t) * nmap, cudaHostAllocMapped));
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&m_map_), h_map_, 0));
        CU(cudaHostAlloc(&h_active_, n_, cudaHostAllocMapped));
        CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&m_active_), h_active_, 0));
        CU(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        CU(cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking));
        for (auto& e : ev_) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        return MWDG2_OK;
    }

    mwdg2_status launch(const std::vector<uint8_t>& stepping) override
    {
        CU(cudaSetDevice(ms_[0]->device_));
        for (int k = 0; k < n_; ++k)
        {
            h_active_[k] = stepping[k];
            if (stepping[k]) ms_[k]->prepare_args();
        }
        // the block maps from the members' last step: leaves; wet leaves of stage 1 and 2
        for (int map = 0; map < mw::kBlockMaps; ++map)
        {
            const int cap = map == 0 ? std::min(cap_wet_, std::min(cap_dry_, cap_leaf_)) : cap_list_;
            std::vector<double> w(n_, 0.0);
            double tot = 0;
            for (int k = 0; k < n_; ++k)
                if (stepping[k])
                {
                    const Sim<T>& m = *ms_[k];
                    w[k] = map == 0 ? (double)std::max<int64_t>(1, m.n_leaves_)
                                    : (double)std::max<int64_t>(1, m.wet_prev_[map - 1] + 1);
                    tot += w[k];
                }
            int32_t* first = h_map_ + map * (n_ + 1);
            int32_t b = 0;
            for (int k = 0; k < n_; ++k)
            {
                first[k] = b;
                if (stepping[k]) b += std::max(1, (int)(cap * (w[k] / tot)));
            }
            first[n_] = b;   // at most cap + n_
        }
        if (!exec_)
        {
            cudaGraph_t g = nullptr;
            CU(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
            launches_ = 0;
            enqueue();
            const cudaError_t e = cudaStreamEndCapture(st_, &g);
            if (e != cudaSuccess) return set_err(MWDG2_ERR_CUDA, std::string("batch group capture: ") + cudaGetErrorString(e));
            const cudaError_t e2 = cudaGraphInstantiate(&exec_, g, 0);
            cudaGraphDestroy(g);
            if (e2 != cudaSuccess) return set_err(MWDG2_ERR_CUDA, std::string("batch group graph: ") + cudaGetErrorString(e2));
        }
        for (int k = 0; k < n_; ++k)
            if (stepping[k]) ms_[k]->launches_ = launches_;
        CU(cudaGraphLaunch(exec_, st_));
        return MWDG2_OK;
    }

    mwdg2_status wait() override
    {
        CU(cudaStreamSynchronize(st_));
        return MWDG2_OK;
    }

private:
    static int blocks(int64_t n, int threads)
    {
        const int64_t b = (n + threads - 1) / threads;
        return (int)std::max<int64_t>(1, std::min<int64_t>(b, 1 << 30));
    }
    void fork(cudaEvent_t e)
    {
        cudaEventRecord(e, st_);
        cudaStreamWaitEvent(st2_, e, 0);
    }
    void join(cudaEvent_t e)
    {
        cudaEventRecord(e, st2_);
        cudaStreamWaitEvent(st_, e, 0);
    }
    template <bool FULL> void encode()
    {
        for (int level = L_ - 1; level > mw::kBandMaxLevel; --level)
        {
            mw::k_members_encode_level<T, FULL><<<dim3(blocks((int64_t)1 << (2 * level), 256), n_), 256, 0, st_>>>(
                *tab_, d_on_, L_, level);
            ++launches_;
        }
        for (const auto& b : bands_)
        {
            mw::k_members_encode_band<T, FULL><<<dim3(b.grid, n_), 256, 0, st_>>>(*tab_, d_on_, L_, b.lo, b.depth);
            ++launches_;
        }
    }
    template <int STAGE> void stage()
    {
        const int32_t* leaves = d_map_;
        const int32_t* wet = d_map_ + STAGE * (n_ + 1);
        const int g = std::min(cap_wet_, std::min(cap_dry_, cap_leaf_)) + n_;
        mw::k_members_stage_wet<T, STAGE><<<g, 256, 0, st_>>>(*tab_, d_on_, leaves, n_);
        fork(ev_[2]);
        mw::k_members_stage_list<T, STAGE><<<cap_list_ + n_, mw::kSolverThreads, 0, st2_>>>(*tab_, d_on_, wet, n_);
        mw::k_members_stage_dry<T, STAGE><<<g, 256, 0, st_>>>(*tab_, d_on_, leaves, n_);
        join(ev_[3]);
        launches_ += 3;
    }
    // the launches of one step, in the order of Sim::enqueue_device for a step after the
    // first with every RK stage over the wet list and no sparse level
    void enqueue()
    {
        mw::k_members_open<T><<<dim3(1, n_), 128, 0, st_>>>(*tab_, m_active_, d_on_, L_, m_map_, d_map_, n_);
        ++launches_;
        encode<true>();
        for (size_t k = bands_.size(); k-- > 0;)
        {
            const auto& b = bands_[k];
            mw::k_members_decode_band<T><<<dim3(b.grid, n_), 256, 0, st_>>>(*tab_, d_on_, L_, b.lo, b.depth);
            ++launches_;
        }
        for (int level = mw::kBandMaxLevel + 1; level <= L_ - 2; ++level)
        {
            mw::k_members_extra_sig<T><<<dim3(blocks((int64_t)1 << (2 * level - 2), 256), n_), 256, 0, st_>>>(
                *tab_, d_on_, L_, level);
            ++launches_;
        }
        const bool split = L_ - 1 > mw::kBandMaxLevel;
        if (split)
        {
            fork(ev_[0]);
            for (int level = mw::kBandMaxLevel + 1; level < L_; ++level)
            {
                mw::k_members_decode_level<T><<<dim3(blocks((int64_t)1 << (2 * level), 256), n_), 256, 0, st2_>>>(
                    *tab_, d_on_, L_, level);
                ++launches_;
            }
        }
        mw::k_members_tile_count<T><<<dim3(ntiles_, n_), 96, 0, st_>>>(*tab_, d_on_, L_);
        mw::k_members_tile_scan<T><<<dim3(1, n_), 1024, 0, st_>>>(*tab_, d_on_, ntiles_);
        mw::k_members_tile_emit<T><<<dim3(ntiles_, n_), mw::kTileThreads, 0, st_>>>(*tab_, d_on_, L_);
        launches_ += 3;
        if (split) join(ev_[1]);
        stage<1>();
        encode<false>();
        mw::k_members_stage2_maxh<T><<<std::min(cap_wet_, std::min(cap_dry_, cap_leaf_)) + n_, 256, 0, st_>>>(
            *tab_, d_on_, d_map_, n_);
        ++launches_;
        stage<2>();
        if (np_max_ > 0)
        {
            mw::k_members_sample<T><<<dim3((32 * np_max_ + 127) / 128, n_), 128, 0, st_>>>(*tab_, d_on_, L_, ntiles_);
            ++launches_;
        }
        mw::k_members_scalars_out<T><<<dim3(1, n_), 128, 0, st_>>>(*tab_, d_on_);
        ++launches_;
    }

    std::vector<Sim<T>*> ms_;
    int n_ = 0, L_ = 0, ntiles_ = 0, np_max_ = 0, launches_ = 0;
    int cap_wet_ = 1, cap_dry_ = 1, cap_list_ = 1, cap_leaf_ = 1;
    std::vector<typename Sim<T>::Band> bands_;
    std::unique_ptr<mw::MemberTable<T>> tab_;   // passed by value to every launch
    uint8_t* d_on_ = nullptr;
    uint8_t* h_active_ = nullptr;   // pinned, mapped
    uint8_t* m_active_ = nullptr;   // its device address
    int32_t* h_map_ = nullptr;      // block maps, pinned and mapped (host writes before each launch)
    int32_t* m_map_ = nullptr;      // its device address
    int32_t* d_map_ = nullptr;      // the maps in device memory (k_members_open copies them)
    cudaStream_t st_ = nullptr, st2_ = nullptr;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t exec_ = nullptr;
};

} // namespace

// ============================================================================ C ABI

struct mwdg2_sim
{
    std::unique_ptr<SimBase> impl;
};

struct mwdg2_batch
{
    std::vector<std::unique_ptr<mwdg2_sim>> members;
    std::vector<uint8_t> done;
    // size classes stepped by one launch per kernel (formed once every member is past its
    // first step); group_of[i] = -1: member i steps on its own
    std::vector<std::unique_ptr<GroupBase>> groups;
    std::vector<int> group_of;
    bool grouped = false;
    // Size classes hold members of at most this max_ref_lvl (mwdg2_batch_group_max_level;
    // 0: none). Off by default: on the 64-member ensemble (FP32, 512^2 to 2048^2) the members
    // stepped as their own CUDA graphs on their own streams, launched from host threads, beat
    // one launch per kernel for a whole class at every size (against stepping the members one
    // after another: 512^2 1.68x against 1.46x, 1024^2 1.26x against 1.08x, 2048^2 1.12x
    // against 0.97x): a class launch lasts as long as its slowest member's part, while
    // independent member graphs fill each other's gaps.
    int group_max_level = 0;
};

namespace {

// Runs fn(i) for every member index on up to eight host threads (launching kernels from
// several threads hides the per-launch host cost of many small members); returns the first
// failing member's status, its message recorded for mwdg2_last_error.
template <typename Fn> mwdg2_status for_members(int n, Fn fn)
{
    const int nt = std::max(1, std::min({n, 8, (int)std::max(1u, std::thread::hardware_concurrency())}));
    std::vector<mwdg2_status> st(n, MWDG2_OK);
    std::vector<std::string> msg(n);
    auto work = [&](int t) {
        for (int i = t; i < n; i += nt)
        {
            st[i] = fn(i);
            if (st[i] != MWDG2_OK && st[i] != MWDG2_DONE) msg[i] = g_last_error;
        }
    };
    if (nt == 1) work(0);
    else
    {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
        for (auto& x : th) x.join();
    }
    for (int i = 0; i < n; ++i)
        if (st[i] != MWDG2_OK && st[i] != MWDG2_DONE)
            return set_err(st[i], "batch member " + std::to_string(i) + ": " + msg[i]);
    return MWDG2_OK;
}

// Forms the batch's size classes of two or more members with the same group key (none is
// formed while a member has its first step to take); checks that grouped members still
// qualify and dissolves the groups otherwise (they are formed again at the next step).
mwdg2_status regroup(mwdg2_batch* b)
{
    const int n = (int)b->members.size();
    if (b->grouped)
    {
        bool ok = true;
        for (const auto& g : b->groups)
            for (int i : g->idx)
                if (!b->done[i] && b->members[i]->impl->group_key() != g->key) ok = false;
        if (ok) return MWDG2_OK;
        b->groups.clear();
        b->grouped = false;
    }
    b->group_of.assign(n, -1);
    std::map<int, std::vector<int>> by_key;
    for (int i = 0; i < n; ++i)
    {
        if (b->done[i]) continue;
        if (b->members[i]->impl->first_step()) return MWDG2_OK;   // not yet
        const int k = b->members[i]->impl->group_key();
        if (k >= 0 && (k & 0xff) <= b->group_max_level) by_key[k].push_back(i);
    }
    for (auto& kv : by_key)
    {
        const bool dbl = (kv.first & (1 << 8)) != 0;
        const size_t cap = dbl ? mw::MemberTable<double>::kMax : mw::MemberTable<float>::kMax;
        // a class larger than one table is stepped as several groups
        for (size_t c0 = 0; c0 < kv.second.size(); c0 += cap)
        {
            const std::vector<int> idx(kv.second.begin() + c0, kv.second.begin() + std::min(kv.second.size(), c0 + cap));
            if (idx.size() < 2) continue;
            std::unique_ptr<GroupBase> g;
            if (dbl)
            {
                std::vector<Sim<double>*> ms;
                for (int i : idx) ms.push_back(static_cast<Sim<double>*>(b->members[i]->impl.get()));
                auto* gg = new Group<double>();
                g.reset(gg);
                if (mwdg2_status st = gg->build(ms)) return st;
            }
            else
            {
                std::vector<Sim<float>*> ms;
                for (int i : idx) ms.push_back(static_cast<Sim<float>*>(b->members[i]->impl.get()));
                auto* gg = new Group<float>();
                g.reset(gg);
                if (mwdg2_status st = gg->build(ms)) return st;
            }
            g->idx = idx;
            g->key = kv.first;
            for (int i : idx) b->group_of[i] = (int)b->groups.size();
            b->groups.push_back(std::move(g));
        }
    }
    b->grouped = true;
    return MWDG2_OK;
}

} // namespace

extern "C" {

void mwdg2_default_opts(mwdg2_opts* o)
{
    if (!o) return;
    o->precision = 64;
    o->device = -1;
    o->epsilon = -1.0;
    o->solver = 0;
    o->dirroot = nullptr;
    o->write_outputs = 1;
    o->verbose = 0;
}

const char* mwdg2_last_error(void) { return g_last_error.c_str(); }

mwdg2_status mwdg2_create(const char* par_path, const mwdg2_opts* opts, mwdg2_sim** out)
{
    if (!par_path || !out) return set_err(MWDG2_ERR_ARG, "mwdg2_create: null argument");
    *out = nullptr;
    mwdg2_opts o;
    mwdg2_default_opts(&o);
    if (opts) o = *opts;
    if (o.precision == 0) o.precision = 64;
    if (o.precision != 32 && o.precision != 64) return set_err(MWDG2_ERR_ARG, "precision must be 32 or 64");
    auto* s = new mwdg2_sim();
    if (o.precision == 32) s->impl.reset(new Sim<float>());
    else s->impl.reset(new Sim<double>());
    mwdg2_status st = s->impl->init(par_path, o);
    if (st != MWDG2_OK)
    {
        delete s;
        return st;
    }
    *out = s;
    return MWDG2_OK;
}

mwdg2_status mwdg2_step(mwdg2_sim* s, double* dt, int64_t* n)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->step(dt, n);
}

mwdg2_status mwdg2_run(mwdg2_sim* s, int64_t max_steps, int64_t* steps, int64_t* updates)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->run(max_steps, steps, updates);
}

mwdg2_status mwdg2_info(mwdg2_sim* s, double* out, int n)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->info(out, n);
}

mwdg2_status mwdg2_get_leaves(mwdg2_sim* s, int32_t* a, int32_t* l, int32_t* ids, int32_t* lv, int64_t cap)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->leaves(a, l, ids, lv, cap);
}

mwdg2_status mwdg2_get_state(mwdg2_sim* s, double* out, int64_t cap)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->state(out, cap);
}

mwdg2_status mwdg2_get_sig(mwdg2_sim* s, uint8_t* out, int64_t cap)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->sig(out, cap);
}

mwdg2_status mwdg2_get_hierarchy(mwdg2_sim* s, int f, int m, double* out, int64_t cap)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->hierarchy(f, m, out, cap);
}

mwdg2_status mwdg2_read_stage(mwdg2_sim* s, double* out, int n)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->stage(out, n);
}

mwdg2_status mwdg2_last_step_timing(mwdg2_sim* s, double* out, int n)
{
    if (!s || !out) return set_err(MWDG2_ERR_ARG, "null argument");
    return s->impl->timing(out, n);
}

mwdg2_status mwdg2_set_timing(mwdg2_sim* s, int mode)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->set_timing(mode);
}

mwdg2_status mwdg2_last_step_counters(mwdg2_sim* s, int64_t* out, int n)
{
    if (!s || !out) return set_err(MWDG2_ERR_ARG, "null argument");
    return s->impl->counters(out, n);
}

void mwdg2_destroy(mwdg2_sim* s) { delete s; }

mwdg2_status mwdg2_volume(mwdg2_sim* s, double* out)
{
    if (!s || !out) return set_err(MWDG2_ERR_ARG, "null argument");
    return s->impl->volume(out);
}

mwdg2_status mwdg2_set_decode_mode(mwdg2_sim* s, int mode)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->decode_mode(mode);
}

mwdg2_status mwdg2_proposal_record(mwdg2_sim* s, int on)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->proposal_record(on != 0);
}

mwdg2_status mwdg2_proposal_enable(mwdg2_sim* s, const float* params, int judge_every, float threshold, float miss_bound)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    if (judge_every < 0 || !(miss_bound >= 0.0f)) return set_err(MWDG2_ERR_ARG, "judge_every >= 0 and miss_bound >= 0");
    return s->impl->proposal_enable(params, judge_every, threshold, miss_bound);
}

mwdg2_status mwdg2_proposal_samples(mwdg2_sim* s, float* feats, uint8_t* labels, int64_t cap, int64_t* n)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->proposal_samples_host(feats, labels, cap, n);
}

mwdg2_status mwdg2_proposal_mask(mwdg2_sim* s, uint8_t* out, int64_t cap, int64_t* n)
{
    if (!s) return set_err(MWDG2_ERR_ARG, "null handle");
    return s->impl->proposal_mask(out, cap, n);
}

mwdg2_status mwdg2_proposal_stats(mwdg2_sim* s, double* out, int n)
{
    if (!s || !out) return set_err(MWDG2_ERR_ARG, "null argument");
    return s->impl->proposal_stats(out, n);
}

mwdg2_status mwdg2_batch_create(int n, const char* const* par_paths, const mwdg2_opts* opts, mwdg2_batch** out)
{
    if (!out || !par_paths || n < 1) return set_err(MWDG2_ERR_ARG, "mwdg2_batch_create: need n >= 1 paths and an output");
    *out = nullptr;
    std::unique_ptr<mwdg2_batch> b(new mwdg2_batch());
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return set_err(MWDG2_ERR_IO, "mwdg2_batch_create: getcwd failed");
    for (int i = 0; i < n; ++i)
    {
        if (!par_paths[i]) return set_err(MWDG2_ERR_ARG, "mwdg2_batch_create: null path " + std::to_string(i));
        // relative names in a member's .par (and its dirroot) resolve against its own folder
        const std::string path = par_paths[i];
        const size_t cut = path.find_last_of('/');
        const std::string dir = cut == std::string::npos ? "." : (cut == 0 ? "/" : path.substr(0, cut));
        char absdir[4096];
        if (!realpath(dir.c_str(), absdir) || chdir(absdir) != 0)
            return set_err(MWDG2_ERR_IO, "batch member " + std::to_string(i) + ": cannot enter the folder of " + path);
        mwdg2_sim* s = nullptr;
        const std::string base = cut == std::string::npos ? path : path.substr(cut + 1);
        mwdg2_status st = mwdg2_create(base.c_str(), opts, &s);
        if (chdir(cwd) != 0 && st == MWDG2_OK) st = set_err(MWDG2_ERR_IO, "cannot return to the working directory");
        if (st != MWDG2_OK)
        {
            delete s;
            return set_err(st, "batch member " + std::to_string(i) + ": " + g_last_error);
        }
        b->members.emplace_back(s);
        s->impl->anchor_outputs(absdir);
        if ((st = s->impl->prepare_outputs()) != MWDG2_OK) return st;
    }
    b->done.assign(n, 0);
    *out = b.release();
    return MWDG2_OK;
}

mwdg2_status mwdg2_batch_step(mwdg2_batch* b, double* dts, int64_t* leaves, int32_t* active)
{
    if (!b) return set_err(MWDG2_ERR_ARG, "null batch");
    const int n = (int)b->members.size();
    if (mwdg2_status s = regroup(b)) return s;
    if (b->group_of.size() != (size_t)n) b->group_of.assign(n, -1);
    std::vector<uint8_t> stepped(n, 0), first(n, 0);
    std::vector<std::chrono::steady_clock::time_point> t0(n);
    auto begin = [&](int i) -> mwdg2_status {
        SimBase& m = *b->members[i]->impl;
        first[i] = m.first_step();
        t0[i] = std::chrono::steady_clock::now();
        mwdg2_status s = m.begin_step();
        if (s == MWDG2_DONE) { b->done[i] = 1; return MWDG2_OK; }
        if (s != MWDG2_OK) return s;
        stepped[i] = 1;
        return MWDG2_OK;
    };
    // clock updates and kernels of every member on its own, without waiting
    mwdg2_status st = for_members(n, [&](int i) -> mwdg2_status {
        if (b->done[i] || b->group_of[i] >= 0) return MWDG2_OK;
        if (mwdg2_status s = begin(i)) return s;
        return stepped[i] ? b->members[i]->impl->enqueue_step() : MWDG2_OK;
    });
    // the size classes: one launch per kernel for all their members
    for (auto& g : b->groups)
    {
        if (st != MWDG2_OK) break;
        std::vector<uint8_t> stepping(g->idx.size(), 0);
        for (size_t k = 0; k < g->idx.size() && st == MWDG2_OK; ++k)
        {
            const int i = g->idx[k];
            if (b->done[i]) continue;
            st = begin(i);
            stepping[k] = stepped[i];
        }
        if (st == MWDG2_OK) st = g->launch(stepping);
    }
    for (auto& g : b->groups)
        if (st == MWDG2_OK) st = g->wait();
    // then wait for each member, take its dt and write its outputs
    mwdg2_status st2 = st != MWDG2_OK ? st : for_members(n, [&](int i) -> mwdg2_status {
        double dt = 0;
        int64_t nl = 0;
        if (stepped[i])
        {
            SimBase& m = *b->members[i]->impl;
            mwdg2_status s = m.finish_step(&dt, &nl);
            if (s != MWDG2_OK) return s;
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0[i]).count();
            if ((s = m.after_step(first[i], dt, nl, secs)) != MWDG2_OK) return s;
        }
        if (dts) dts[i] = dt;
        if (leaves) leaves[i] = nl;
        return MWDG2_OK;
    });
    if (st != MWDG2_OK) return st;
    if (st2 != MWDG2_OK) return st2;
    int32_t k = 0;
    for (int i = 0; i < n; ++i) k += stepped[i];
    if (active) *active = k;
    return k ? MWDG2_OK : MWDG2_DONE;
}

mwdg2_status mwdg2_batch_run(mwdg2_batch* b, int64_t max_batch_steps, int64_t* batch_steps, int64_t* member_steps,
                             int64_t* updates)
{
    if (!b) return set_err(MWDG2_ERR_ARG, "null batch");
    const int n = (int)b->members.size();
    std::vector<int64_t> nl(n);
    int64_t bs = 0, ms = 0, upd = 0;
    while (max_batch_steps <= 0 || bs < max_batch_steps)
    {
        int32_t k = 0;
        mwdg2_status st = mwdg2_batch_step(b, nullptr, nl.data(), &k);
        if (st == MWDG2_DONE) break;
        if (st != MWDG2_OK) return st;
        ++bs;
        ms += k;
        for (int i = 0; i < n; ++i) upd += nl[i];
    }
    if (batch_steps) *batch_steps = bs;
    if (member_steps) *member_steps = ms;
    if (updates) *updates = upd;
    return MWDG2_OK;
}

mwdg2_status mwdg2_batch_group_max_level(mwdg2_batch* b, int level)
{
    if (!b) return set_err(MWDG2_ERR_ARG, "null batch");
    b->group_max_level = level;
    b->groups.clear();   // formed again at the next step
    b->grouped = false;
    return MWDG2_OK;
}

mwdg2_status mwdg2_batch_member(mwdg2_batch* b, int i, mwdg2_sim** out)
{
    if (!b || !out || i < 0 || i >= (int)b->members.size()) return set_err(MWDG2_ERR_ARG, "mwdg2_batch_member: bad index");
    *out = b->members[i].get();
    return MWDG2_OK;
}

void mwdg2_batch_destroy(mwdg2_batch* b) { delete b; }

mwdg2_status mwdg2_run_simulation(int argc, char** argv)
{
    // input/read_command_line_params.cpp:12-47; the last argument is the .par file
    if (argc < 2) return set_err(MWDG2_ERR_ARG, "usage: gpu-mwdg2 [-epsilon e] [-solver hwfv1|mwdg2] [-dirroot d] case.par");
    mwdg2_opts o;
    mwdg2_default_opts(&o);
    o.verbose = 1;
    std::string dirroot;
    for (int i = 0; i < argc - 1; ++i)
    {
        const char* flag = argv[i];
        const char* value = argv[i + 1];
        if (!strncmp(flag, "-epsilon", 8)) o.epsilon = atof(value);
        else if (!strncmp(flag, "-solver", 7))
        {
            if (!strncmp(value, "hwfv1", 5)) o.solver = 1;
            else if (!strncmp(value, "mwdg2", 5)) o.solver = 2;
            else return set_err(MWDG2_ERR_ARG, "invalid -solver (use hwfv1 or mwdg2)");
        }
        else if (!strncmp(flag, "-dirroot", 8)) dirroot = value;
        else if (!strncmp(flag, "-precision", 10)) o.precision = atoi(value);
    }
    if (!dirroot.empty()) o.dirroot = dirroot.c_str();
    mwdg2_sim* s = nullptr;
    mwdg2_status st = mwdg2_create(argv[argc - 1], &o, &s);
    if (st != MWDG2_OK) return st;
    const auto t0 = std::chrono::steady_clock::now();
    int64_t steps = 0, upd = 0;
    st = mwdg2_run(s, 0, &steps, &upd);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st == MWDG2_OK) printf("Loop time: %f s (%lld steps, %.4e active-cell updates/s)\n", secs, (long long)steps, upd / secs);
    mwdg2_destroy(s);
    return st;
}

} // extern "C"

mwdg2_status mwdg2_detail_proposal_samples(mwdg2_sim* sim, const void** feats, const uint8_t** labels, int64_t* n,
                                           int* device)
{
    return sim->impl->proposal_samples(feats, labels, n, device);
}
