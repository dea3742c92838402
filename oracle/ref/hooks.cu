/*
 * Observation wrappers around five host functions of the reference time loop
 * (al0vya/gpu-mwdg2 source/run_simulation.cu). Test infrastructure only: these
 * wrappers are linked into the reference build under oracle/_ref and are never
 * part of the product.
 *
 * Each wrapper calls the reference's own function with the same arguments and
 * then (optionally) writes raw little-endian binary arrays:
 *
 *   MWDG2_REF_DUMP_DIR    directory for dumps (unset: no array dumps)
 *   MWDG2_REF_DUMP_STEPS  comma separated step numbers, or "all"
 *   MWDG2_REF_STOP_AFTER  stop the process (exit 0) after this many steps
 *   MWDG2_REF_STEPS_CSV   per-step log "step,dt,n_leaves,wall_s,time" (always written
 *                         when set; time: simulated time at the end of the step)
 *   MWDG2_REF_WINDOW_TIME, MWDG2_REF_WINDOW_STEPS
 *                         when both are set, stop (exit 0) once WINDOW_STEPS steps have
 *                         ended at or after the first step that ended at a simulated time
 *                         >= WINDOW_TIME (a timing window later in the run)
 *   MWDG2_REF_DIGEST_DIR  directory for per-step digests (unset: none): every step,
 *                         digest.csv gets one row "step,name,n,hash" per leaf-list,
 *                         neighbour and significance array (hash: below), and at the
 *                         steps listed in MWDG2_REF_SAMPLE_STEPS sample_step<n>.bin gets
 *                         the leaf state after step n at up to 2048 evenly spaced leaves
 *                         (12 rows of `real`) followed by the float64 sums of the 12 rows
 *
 * Digest of n 8- or 32-bit values v_i (their bit patterns, zero-extended):
 *     n * 0x9E3779B97F4A7C15 + sum_i (v_i + 1) * (splitmix64(i) | 1)   (mod 2^64)
 * with splitmix64 Vigna's finaliser of x + 0x9E3779B97F4A7C15. Every multiplier is odd, so
 * a change in any single value changes the digest; tests/golden/make_golden_digest.py
 * computes the same function in numpy for the product's arrays.
 *
 * Dump points (step n counts from 1, as the reference's `timestep`):
 *   compaction (run_simulation.cu:457)  -> leaf list + neighbours of step n
 *   decoding   (run_simulation.cu:393)  -> significance flags, norms, hierarchy
 *   get_max_scale_coeffs (:247)         -> leaf state after step n-1 and maxes
 *   get_dt_CFL (:650)                   -> dt, leaf count, wall time of step n
 *   project_assem_sol (:725)            -> pass-through
 */
#include "run_simulation.cuh"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

namespace
{
int  g_step_done  = 0;     // number of completed get_dt_CFL calls
int  g_max_calls  = 0;     // number of get_max_scale_coeffs calls
bool g_cfg_loaded = false;
bool g_dump_all   = false;
int  g_stop_after = -1;
double g_window_time = -1.0;   // MWDG2_REF_WINDOW_TIME
int    g_window_steps = 0;     // MWDG2_REF_WINDOW_STEPS
int    g_window_first = -1;    // first step that ended at or after g_window_time
double g_sim_time = 0.0;       // simulated time at the end of the last step
double g_dt_next = 0.001;      // dt of the next step (the reference starts with 0.001)
std::set<int> g_dump_steps;
std::string   g_dump_dir;
FILE*         g_steps_csv = nullptr;
std::chrono::steady_clock::time_point g_t0;
std::string   g_digest_dir;
FILE*         g_digest_csv = nullptr;
std::set<int> g_sample_steps;
constexpr int kSample = 2048;

std::set<int> parse_steps(const char* steps)
{
    std::set<int> out;
    if (!steps) return out;
    std::string s(steps);
    size_t pos = 0;
    while (pos < s.size())
    {
        size_t end = s.find(',', pos);
        if (end == std::string::npos) end = s.size();
        if (end > pos) out.insert(atoi(s.substr(pos, end - pos).c_str()));
        pos = end + 1;
    }
    return out;
}

uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

template <typename T>
uint64_t digest_host(const T* v, size_t n)
{
    static_assert(sizeof(T) == 1 || sizeof(T) == 4, "8- or 32-bit values");
    uint64_t h = (uint64_t)n * 0x9E3779B97F4A7C15ull;
    for (size_t i = 0; i < n; ++i)
    {
        uint64_t bits;
        if (sizeof(T) == 1) bits = *reinterpret_cast<const uint8_t*>(v + i);
        else bits = *reinterpret_cast<const uint32_t*>(v + i);
        h += (bits + 1) * (splitmix64(i) | 1ull);
    }
    return h;
}

template <typename T>
void digest_dev(int step, const char* name, const T* d_ptr, size_t count)
{
    if (!g_digest_csv || d_ptr == nullptr) return;
    std::vector<T> h(count);
    if (count) cudaMemcpy(h.data(), d_ptr, count * sizeof(T), cudaMemcpyDeviceToHost);
    fprintf(g_digest_csv, "%d,%s,%zu,%llu\n", step, name, count,
            (unsigned long long)digest_host(h.data(), count));
}

void load_cfg()
{
    if (g_cfg_loaded) return;
    g_cfg_loaded = true;
    g_t0 = std::chrono::steady_clock::now();
    const char* dir = getenv("MWDG2_REF_DUMP_DIR");
    if (dir) g_dump_dir = dir;
    const char* steps = getenv("MWDG2_REF_DUMP_STEPS");
    if (steps)
    {
        if (!strcmp(steps, "all")) g_dump_all = true;
        else
        {
            std::string s(steps);
            size_t pos = 0;
            while (pos < s.size())
            {
                size_t end = s.find(',', pos);
                if (end == std::string::npos) end = s.size();
                if (end > pos) g_dump_steps.insert(atoi(s.substr(pos, end - pos).c_str()));
                pos = end + 1;
            }
        }
    }
    const char* stop = getenv("MWDG2_REF_STOP_AFTER");
    if (stop) g_stop_after = atoi(stop);
    const char* wt = getenv("MWDG2_REF_WINDOW_TIME");
    const char* ws = getenv("MWDG2_REF_WINDOW_STEPS");
    if (wt && ws) { g_window_time = atof(wt); g_window_steps = atoi(ws); }
    const char* ddir = getenv("MWDG2_REF_DIGEST_DIR");
    if (ddir)
    {
        g_digest_dir = ddir;
        g_digest_csv = fopen((g_digest_dir + "/digest.csv").c_str(), "w");
        if (g_digest_csv) fprintf(g_digest_csv, "step,name,n,hash\n");
        g_sample_steps = parse_steps(getenv("MWDG2_REF_SAMPLE_STEPS"));
    }
    const char* csv = getenv("MWDG2_REF_STEPS_CSV");
    if (csv)
    {
        g_steps_csv = fopen(csv, "w");
        if (g_steps_csv) fprintf(g_steps_csv, "step,dt,n_leaves,wall_s,time\n");
    }
}

bool want(int step)
{
    load_cfg();
    if (g_dump_dir.empty()) return false;
    return g_dump_all || g_dump_steps.count(step) > 0;
}

template <typename T>
void dump_dev(int step, const char* name, const T* d_ptr, size_t count)
{
    if (d_ptr == nullptr || count == 0) return;
    std::vector<T> h(count);
    cudaMemcpy(h.data(), d_ptr, count * sizeof(T), cudaMemcpyDeviceToHost);
    char path[1024];
    snprintf(path, sizeof(path), "%s/step%06d_%s.bin", g_dump_dir.c_str(), step, name);
    FILE* fp = fopen(path, "wb");
    if (!fp) { fprintf(stderr, "ref hooks: cannot open %s\n", path); return; }
    fwrite(h.data(), sizeof(T), count, fp);
    fclose(fp);
}

template <typename T>
void dump_host(int step, const char* name, const T* ptr, size_t count)
{
    char path[1024];
    snprintf(path, sizeof(path), "%s/step%06d_%s.bin", g_dump_dir.c_str(), step, name);
    FILE* fp = fopen(path, "wb");
    if (!fp) return;
    fwrite(ptr, sizeof(T), count, fp);
    fclose(fp);
}

void dump_assem(int step, const AssembledSolution& s)
{
    const size_t n = (size_t)s.length;
    int len = s.length;
    dump_host(step, "len", &len, 1);
    dump_dev(step, "act_idcs", s.act_idcs, n);
    dump_dev(step, "levels",   s.levels,   n);
    dump_dev(step, "h0",  s.h0,  n);
    dump_dev(step, "qx0", s.qx0, n);
    dump_dev(step, "qy0", s.qy0, n);
    dump_dev(step, "z0",  s.z0,  n);
    dump_dev(step, "h1x",  s.h1x,  n);
    dump_dev(step, "qx1x", s.qx1x, n);
    dump_dev(step, "qy1x", s.qy1x, n);
    dump_dev(step, "z1x",  s.z1x,  n);
    dump_dev(step, "h1y",  s.h1y,  n);
    dump_dev(step, "qx1y", s.qx1y, n);
    dump_dev(step, "qy1y", s.qy1y, n);
    dump_dev(step, "z1y",  s.z1y,  n);
}
// State after `step` at up to kSample evenly spaced leaves (index j * n / S), then the
// float64 sums of the 12 rows over all leaves.
void sample_assem(int step, const AssembledSolution& s)
{
    const size_t n = (size_t)s.length;
    const size_t S = n < (size_t)kSample ? n : (size_t)kSample;
    const real* rows[12] = {s.h0, s.qx0, s.qy0, s.z0, s.h1x, s.qx1x, s.qy1x, s.z1x, s.h1y, s.qx1y, s.qy1y, s.z1y};
    std::vector<real> out(12 * S, real(0));
    double sums[12] = {0};
    std::vector<real> h(n);
    for (int r = 0; r < 12; ++r)
    {
        if (rows[r] == nullptr || n == 0) continue;
        cudaMemcpy(h.data(), rows[r], n * sizeof(real), cudaMemcpyDeviceToHost);
        for (size_t j = 0; j < S; ++j) out[r * S + j] = h[j * n / S];
        double acc = 0;
        for (size_t i = 0; i < n; ++i) acc += (double)h[i];
        sums[r] = acc;
    }
    char path[1024];
    snprintf(path, sizeof(path), "%s/sample_step%06d.bin", g_digest_dir.c_str(), step);
    FILE* fp = fopen(path, "wb");
    if (!fp) return;
    fwrite(out.data(), sizeof(real), out.size(), fp);
    fwrite(sums, sizeof(double), 12, fp);
    fclose(fp);
}
} // namespace

__host__
void ref_hook_compaction
(
    AssembledSolution& d_buf_assem_sol,
    AssembledSolution& d_assem_sol,
    Neighbours&        d_buf_neighbours,
    Neighbours&        d_neighbours,
    CompactionFlags&   d_compaction_flags,
    int                num_finest_elems,
    const SolverParams& solver_params
)
{
    compaction(d_buf_assem_sol, d_assem_sol, d_buf_neighbours, d_neighbours,
               d_compaction_flags, num_finest_elems, solver_params);
    const int step = g_step_done + 1;
    load_cfg();
    if (g_digest_csv)
    {
        const size_t m = (size_t)d_assem_sol.length;
        digest_dev(step, "leaf_act", d_assem_sol.act_idcs, m);
        digest_dev(step, "leaf_lvl", d_assem_sol.levels, m);
        digest_dev(step, "nb_n_ids", d_neighbours.north.act_idcs, m);
        digest_dev(step, "nb_e_ids", d_neighbours.east.act_idcs, m);
        digest_dev(step, "nb_s_ids", d_neighbours.south.act_idcs, m);
        digest_dev(step, "nb_w_ids", d_neighbours.west.act_idcs, m);
        if (solver_params.solver_type == MWDG2)
        {
            digest_dev(step, "nb_n_lvls", d_neighbours.north.levels, m);
            digest_dev(step, "nb_e_lvls", d_neighbours.east.levels, m);
            digest_dev(step, "nb_s_lvls", d_neighbours.south.levels, m);
            digest_dev(step, "nb_w_lvls", d_neighbours.west.levels, m);
        }
    }
    if (!want(step)) return;
    const size_t n = (size_t)d_assem_sol.length;
    int len = d_assem_sol.length;
    dump_host(step, "leaf_len", &len, 1);
    dump_dev(step, "leaf_act_idcs", d_assem_sol.act_idcs, n);
    dump_dev(step, "leaf_levels",   d_assem_sol.levels,   n);
    dump_dev(step, "nb_n_ids", d_neighbours.north.act_idcs, n);
    dump_dev(step, "nb_e_ids", d_neighbours.east.act_idcs,  n);
    dump_dev(step, "nb_s_ids", d_neighbours.south.act_idcs, n);
    dump_dev(step, "nb_w_ids", d_neighbours.west.act_idcs,  n);
    if (solver_params.solver_type == MWDG2)
    {
        dump_dev(step, "nb_n_lvls", d_neighbours.north.levels, n);
        dump_dev(step, "nb_e_lvls", d_neighbours.east.levels,  n);
        dump_dev(step, "nb_s_lvls", d_neighbours.south.levels, n);
        dump_dev(step, "nb_w_lvls", d_neighbours.west.levels,  n);
    }
}

void ref_hook_decoding
(
    bool*              d_sig_details,
    real*              d_norm_details,
    Details&           d_details,
    ScaleCoefficients& d_scale_coeffs,
    SolverParams&      solver_params
)
{
    decoding(d_sig_details, d_norm_details, d_details, d_scale_coeffs, solver_params);
    const int step = g_step_done + 1;
    load_cfg();
    digest_dev(step, "sig", reinterpret_cast<unsigned char*>(d_sig_details), (size_t)get_lvl_idx(solver_params.L));
    if (!want(step)) return;
    const size_t n_det = (size_t)get_lvl_idx(solver_params.L);
    const size_t n_all = (size_t)get_lvl_idx(solver_params.L + 1);
    dump_dev(step, "sig",  reinterpret_cast<unsigned char*>(d_sig_details), n_det);
    dump_dev(step, "norm", d_norm_details, n_det);
    dump_dev(step, "hier_eta0", d_scale_coeffs.eta0, n_all);
    dump_dev(step, "hier_qx0",  d_scale_coeffs.qx0,  n_all);
    dump_dev(step, "hier_qy0",  d_scale_coeffs.qy0,  n_all);
    dump_dev(step, "hier_z0",   d_scale_coeffs.z0,   n_all);
    if (solver_params.solver_type == MWDG2)
    {
        dump_dev(step, "hier_eta1x", d_scale_coeffs.eta1x, n_all);
        dump_dev(step, "hier_qx1x",  d_scale_coeffs.qx1x,  n_all);
        dump_dev(step, "hier_qy1x",  d_scale_coeffs.qy1x,  n_all);
        dump_dev(step, "hier_z1x",   d_scale_coeffs.z1x,   n_all);
        dump_dev(step, "hier_eta1y", d_scale_coeffs.eta1y, n_all);
        dump_dev(step, "hier_qx1y",  d_scale_coeffs.qx1y,  n_all);
        dump_dev(step, "hier_qy1y",  d_scale_coeffs.qy1y,  n_all);
        dump_dev(step, "hier_z1y",   d_scale_coeffs.z1y,   n_all);
    }
}

__host__
Maxes ref_hook_get_max_scale_coeffs
(
    AssembledSolution& d_assem_sol,
    real*&             d_eta_temp
)
{
    load_cfg();
    const int call = g_max_calls++;
    // call 0: initialisation (run_simulation.cu:190); call k >= 1: start of step k,
    // when d_assem_sol still holds the state after step k - 1.
    const int prev_step = call - 1;
    const bool dump = (call >= 2) && want(prev_step);
    if (dump) dump_assem(prev_step, d_assem_sol);
    if (call >= 2 && g_digest_csv && g_sample_steps.count(prev_step)) sample_assem(prev_step, d_assem_sol);
    Maxes m = get_max_scale_coeffs(d_assem_sol, d_eta_temp);
    if (call >= 1 && want(call))
    {
        real mx[5] = { m.eta, m.h, m.qx, m.qy, m.z };
        dump_host(call, "maxes", mx, 5);
    }
    return m;
}

__host__
real ref_hook_get_dt_CFL
(
    real*&     d_dt_CFL,
    const int& sol_len
)
{
    load_cfg();
    real dt = get_dt_CFL(d_dt_CFL, sol_len);
    g_step_done++;
    // run_simulation.cu:228-235 advances the clock by the previous step's dt at the start
    // of each step (the last step is clipped to sim_time, which a timing window never reaches)
    g_sim_time += g_dt_next;
    g_dt_next = (double)dt;
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - g_t0).count();
    if (g_steps_csv)
    {
        fprintf(g_steps_csv, "%d,%.17g,%d,%.9f,%.9f\n", g_step_done, (double)dt, sol_len, wall, g_sim_time);
    }
    if (g_window_steps > 0 && g_window_first < 0 && g_sim_time >= g_window_time) g_window_first = g_step_done;
    const bool window_done = g_window_first > 0 && g_step_done >= g_window_first + g_window_steps;
    if (want(g_step_done))
    {
        dump_dev(g_step_done, "dt_cfl", d_dt_CFL, (size_t)sol_len);
        dump_host(g_step_done, "dt", &dt, 1);
    }
    if ((g_stop_after > 0 && g_step_done >= g_stop_after) || window_done)
    {
        if (g_steps_csv) fclose(g_steps_csv);
        if (g_digest_csv) fclose(g_digest_csv);
        cudaDeviceSynchronize();
        fflush(stdout);
        _exit(0);
    }
    return dt;
}

__host__
void ref_hook_project_assem_sol
(
    const int&               mesh_dim,
    bool*&                   d_sig_details,
    const ScaleCoefficients& d_scale_coeffs,
    AssembledSolution        d_buf_assem_sol,
    const SolverParams&      solver_params,
    MortonCode*              d_rev_z_order,
    MortonCode*              d_indices,
    AssembledSolution        d_assem_sol,
    AssembledSolution        d_plot_assem_sol
)
{
    project_assem_sol(mesh_dim, d_sig_details, d_scale_coeffs, d_buf_assem_sol, solver_params,
                      d_rev_z_order, d_indices, d_assem_sol, d_plot_assem_sol);
}

void ref_hooks_finish()
{
    if (g_steps_csv) { fclose(g_steps_csv); g_steps_csv = nullptr; }
    if (g_digest_csv) { fclose(g_digest_csv); g_digest_csv = nullptr; }
}
