// CPU oracle for one adaptive MWDG2/HWFV1 time step (al0vya/gpu-mwdg2).
//
// TEST INFRASTRUCTURE ONLY: a restatement of the reference algorithm on the CPU,
// used by tests/ as the checker and by bench.py as the timed CPU baseline ("port").
// It keeps the reference's data layout (all finest-grid work arrays, hierarchy arrays
// indexed by get_lvl_idx) and its per-step sequence (source/run_simulation.cu:226-774),
// including the O(F) tree traversal, neighbour search and compaction passes.
// Loops over independent elements run under OpenMP.
//
// Built by oracle/Makefile into oracle/liboracle_mwdg2.so; C API at the end of file.

#include "oracle_io.hpp"

#include <algorithm>
#include <cfloat>
#include <memory>
#include <omp.h>

namespace oracle {

template <typename T> struct LeafArrays
{
    // classes/AssembledSolution.h:15-101 (h0..z1y, act_idcs, levels, length)
    std::vector<T> h0, qx0, qy0, z0, h1x, qx1x, qy1x, z1x, h1y, qx1y, qy1y, z1y;
    std::vector<int> act, lvl;
    int length = 0;
    void alloc(size_t n, bool coeffs)
    {
        act.assign(n, 0);
        lvl.assign(n, 0);
        if (!coeffs) return;
        for (auto* v : {&h0, &qx0, &qy0, &z0, &h1x, &qx1x, &qy1x, &z1x, &h1y, &qx1y, &qy1y, &z1y})
            v->assign(n, T(0));
    }
};

template <typename T> struct Boundary
{
    // classes/Boundary.h:17-502
    int start = 0, end = 0;
    int bdytype = CLOSED;
    T inlet = T(0);
    std::string series;
    std::vector<T> tdata, vdata;
    int row = 0;
    std::vector<int> codes;
    bool bound(int c) const { return c >= start && c <= end; }
    T q_src(T dt, T dx) const { return inlet * dt / dx; }
};

template <typename T> struct Maxes { T eta, h, qx, qy, z; };

template <typename T> class Sim
{
public:
    // ---- parameters (classes/SolverParams.h:10-36, classes/SimulationParams.h:8-32)
    int L = 0, solver = MWDG2, test_case = 0;
    T initial_tstep = T(0), epsilon = T(0), tol_h = T(1e-3), tol_q = T(0), tol_s = T(1e-9);
    T wall_height = T(0), CFL = T(0), tol_Krivo = T(9999.0);
    bool limitslopes = false, refine_wall = false, startq2d = false;
    int ref_thickness = 0;
    T xmin = T(0), xmax = T(0), ymin = T(0), ymax = T(0), g = T(9.80665), sim_time = T(0), manning = T(0);
    int xsz = 0, ysz = 0;
    bool is_monai = false, is_oregon = false;
    std::string par;

    int M = 0, F = 0, n_all = 0, n_det = 0;
    T dx = T(0), dy = T(0), dt = T(0.001), current_time = T(0);
    bool first = true;
    int timestep = 1;
    Maxes<T> maxes{T(1), T(1), T(1), T(1), T(1)};

    Boundary<T> bnd[4];   // north, east, south, west
    std::vector<int> src_codes, src_types, src_rows;
    std::vector<T> srcs;
    std::vector<std::vector<T>> src_t, src_v;
    std::vector<int> stage_codes;

    // ---- arrays (run_simulation.cu:74-99)
    std::vector<T> eta0, qx0, qy0, z0, eta1x, qx1x, qy1x, z1x, eta1y, qx1y, qy1y, z1y; // hierarchy
    std::vector<T> det[4][3][3];  // field (eta,qx,qy,z) x (alpha,beta,gamma) x mode (0,1x,1y)
    std::vector<T> norm;
    std::vector<unsigned char> sig, preflag;
    // Decode mode of the library's keep-values option (not in the reference): the children
    // of a parent that this step's encode visited keep the values the encode read, and
    // only parents made significant without an encode (refined this step) are decoded.
    // enc[p]: parent p was visited by this step's encode (it was significant at the start).
    bool keep_values = false;
    std::vector<unsigned char> enc;
    LeafArrays<T> assem, buf;
    LeafArrays<T> nb[4], buf_nb[4];
    std::vector<unsigned char> flag_ne, flag_sw;
    std::vector<int> rev_z_order, rev_row_major;
    std::vector<T> dt_cfl;

    std::string error;

    bool init(const char* par_path, double eps_override, int solver_override);
    bool step();
    // Leaf list and neighbours of the tree given by significance flags `s` (get_lvl_idx(L)
    // bytes), with no simulation around it: the traversal and neighbour/compaction passes of
    // a step (mra/traverse_tree_of_sig_details.cu, neighbours/find_neighbours.cu,
    // neighbours/compaction.cu) on an MWDG2 grid of 2^L x 2^L cells whose DEM is xsz x ysz.
    int topology_from_sig(const unsigned char* s, int L_, int xsz_, int ysz_);

    T* hier(int field, int mode)
    {
        static T* none = nullptr;
        std::vector<T>* tab[4][3] = {{&eta0, &eta1x, &eta1y}, {&qx0, &qx1x, &qx1y},
                                     {&qy0, &qy1x, &qy1y}, {&z0, &z1x, &z1y}};
        auto* v = tab[field][mode];
        return v->empty() ? none : v->data();
    }

private:
    bool read_params(double eps_override, int solver_override);
    bool read_boundaries();
    bool read_point_sources();
    void read_stage_points();
    void update_srcs(T now);
    void build_preflags();
    bool initial_modes(LeafArrays<T>& rm);
    void topo_encode();
    Maxes<T> get_maxes(const LeafArrays<T>& s);
    T abs_max(const std::vector<T>& a, int n);
    void zero_details();
    void reinsert(const LeafArrays<T>& s);
    void reinsert_point_srcs();
    void encode_flow(bool for_nghbrs);
    void regularisation();
    void extra_significance();
    void decoding();
    void traverse();
    void neighbours_and_compaction();
    void load_soln(LeafArrays<T>& s);
    void add_ghost_cells(LeafArrays<T>& s);
    void friction_implicit();
    void limit_slopes(LeafArrays<T>& s, T max_h);
    void dg2_update(LeafArrays<T>& ld, LeafArrays<T>& st, bool rkdg2);
    void fv1_update();
    T min_dt();
};

// ============================================================================ init

template <typename T>
bool Sim<T>::read_params(double eps_override, int solver_override)
{
    const char* p = par.c_str();
    // input/read_test_case.cpp:3-17
    test_case = read_kw_int(p, "test_case");
    if (test_case != 0) { error = "only raster-based cases (test_case 0) are supported"; return false; }
    // classes/SolverParams.cu:5-48
    L = read_kw_int(p, "max_ref_lvl");
    initial_tstep = read_kw_real<T>(p, "initial_tstep");
    epsilon = read_kw_real<T>(p, "epsilon");
    wall_height = read_kw_real<T>(p, "wall_height");
    if (read_kw_bool(p, "hwfv1")) { solver = HWFV1; CFL = T(0.5); }
    else if (read_kw_bool(p, "mwdg2")) { solver = MWDG2; CFL = T(0.3); }
    else { error = "no solver keyword (hwfv1 or mwdg2)"; return false; }
    limitslopes = read_kw_bool(p, "limitslopes");
    if (limitslopes) tol_Krivo = read_kw_real<T>(p, "tol_Krivo");
    refine_wall = read_kw_bool(p, "refine_wall");
    if (refine_wall) ref_thickness = read_kw_int(p, "ref_thickness");
    startq2d = read_kw_bool(p, "startq2d");
    // CLI overrides (input/read_command_line_params.cpp:12-47)
    if (eps_override >= 0) epsilon = T(eps_override);
    if (solver_override == HWFV1) { solver = HWFV1; CFL = T(0.5); }
    if (solver_override == MWDG2) { solver = MWDG2; CFL = T(0.3); }
    // optional CFL keyword (not read by the reference, whose CFL is fixed)
    bool has_cfl = false;
    T cfl = read_kw_real<T>(p, "CFL", &has_cfl);
    if (has_cfl && cfl > T(0)) CFL = cfl;
    if (L < 6 || L > 14) { error = "max_ref_lvl must be in [6, 14]"; return false; }
    // classes/SimulationParams.cpp:15-33
    std::string dem = read_kw_str(p, "DEMfile");
    if (dem.empty()) { error = "no DEMfile"; return false; }
    FILE* fp = fopen(dem.c_str(), "r");
    if (!fp) { error = "cannot open DEM " + dem; return false; }
    fclose(fp);
    xsz = read_kw_int(dem.c_str(), "ncols");
    ysz = read_kw_int(dem.c_str(), "nrows");
    xmin = read_kw_real<T>(dem.c_str(), "xllcorner");
    ymin = read_kw_real<T>(dem.c_str(), "yllcorner");
    T cellsize = read_kw_real<T>(dem.c_str(), "cellsize");
    xmax = xmin + xsz * cellsize;
    ymax = ymin + ysz * cellsize;
    sim_time = read_kw_real<T>(p, "sim_time");
    manning = read_kw_real<T>(p, "fpfric");
    is_monai = read_kw_bool(p, "monai");
    is_oregon = read_kw_bool(p, "oregon-seaside");
    if (is_monai || is_oregon) { error = "monai/oregon-seaside boundary specials are not supported"; return false; }
    M = 1 << L;
    if (xsz > M || ysz > M || xsz <= 0 || ysz <= 0) { error = "DEM larger than 2^max_ref_lvl"; return false; }
    F = M * M;
    n_all = lvl_idx(L + 1);
    n_det = lvl_idx(L);
    // run_simulation.cu:34-35
    dx = read_cell_size<T>(p);
    dy = dx;
    return true;
}

template <typename T>
bool Sim<T>::read_boundaries()
{
    // classes/Boundary.h:92-371 (read_num_cells, read_bdy_conds, gen_bdy_morton_codes)
    const char* p = par.c_str();
    std::string bci = read_kw_str(p, "bcifile");
    const char dirs[4] = {'N', 'E', 'S', 'W'};
    for (int b = 0; b < 4; ++b)
    {
        Boundary<T>& B = bnd[b];
        if (bci.empty()) continue;
        FILE* fp = fopen(bci.c_str(), "r");
        if (!fp) { error = "cannot open bcifile " + bci; return false; }
        T origin = (b == 0 || b == 2) ? xmin : ymin;
        char line[255] = {0};
        char filedir = '\0';
        char type[8] = {0};
        T lower = T(0), upper = T(0);
        std::string fmt = std::string("%c ") + real_fmt<T>() + " " + real_fmt<T>() + " %7s";
        bool found = false;
        while (fgets(line, sizeof(line), fp))
        {
            sscanf(line, fmt.c_str(), &filedir, &lower, &upper, type);
            if (filedir == dirs[b]) { found = true; break; }
        }
        fclose(fp);
        if (!found) continue;
        int bt = CLOSED;
        T inlet = T(0);
        char series[32] = {0};
        if (!strncmp(type, "CLOSED", 6)) bt = CLOSED;
        else if (!strncmp(type, "FREE", 4)) bt = FREE;
        else if (!strncmp(type, "HFIX", 4)) { bt = HFIX; sscanf(line, (fmt + " " + real_fmt<T>()).c_str(), &filedir, &lower, &upper, type, &inlet); }
        else if (!strncmp(type, "HVAR", 4)) { bt = HVAR; sscanf(line, (fmt + " %31s").c_str(), &filedir, &lower, &upper, type, series); }
        else if (!strncmp(type, "QFIX", 4)) { bt = QFIX; sscanf(line, (fmt + " " + real_fmt<T>()).c_str(), &filedir, &lower, &upper, type, &inlet); }
        else if (!strncmp(type, "QVAR", 4)) { bt = QVAR; sscanf(line, (fmt + " %31s").c_str(), &filedir, &lower, &upper, type, series); }
        B.start = (int)((lower - origin) / dx);
        B.end = (int)((upper - origin) / dx - T(1));
        B.bdytype = bt;
        B.inlet = inlet;
        B.series = series;
        const int ncells = std::max(0, B.end - B.start + 1);
        B.codes.resize(ncells);
        for (int i = 0; i < ncells; ++i)
        {
            const int c = B.start + i;
            switch (b)
            {
                case 0: B.codes[i] = morton(c, ysz - 1); break;
                case 1: B.codes[i] = morton(xsz - 1, c); break;
                case 2: B.codes[i] = morton(c, 0); break;
                default: B.codes[i] = morton(0, c); break;
            }
        }
        if (bt == HVAR || bt == QVAR)
        {
            if (!read_series<T>(p, series, B.tdata, B.vdata)) { error = std::string("missing time series ") + series; return false; }
        }
    }
    return true;
}

template <typename T>
bool Sim<T>::read_point_sources()
{
    // classes/PointSources.h:117-279
    const char* p = par.c_str();
    std::string bci = read_kw_str(p, "bcifile");
    if (bci.empty()) return true;
    FILE* fp = fopen(bci.c_str(), "r");
    if (!fp) { error = "cannot open bcifile " + bci; return false; }
    char line[255];
    std::string fmt = std::string("%c ") + real_fmt<T>() + " " + real_fmt<T>() + " %7s";
    while (fgets(line, sizeof(line), fp))
    {
        char point = 0;
        T xs = T(0), ys = T(0);
        char type[8] = {0};
        sscanf(line, fmt.c_str(), &point, &xs, &ys, type);
        if (point != 'P') continue;
        const int x = (int)((xs - xmin) / dx);
        const int y = (int)((ys - ymin) / dx);
        src_codes.push_back(morton(x, y));
        T val = T(0);
        char series[32] = {0};
        int t = 0;
        if (!strncmp(type, "HFIX", 4)) { t = HFIX; sscanf(line, (fmt + " " + real_fmt<T>()).c_str(), &point, &xs, &ys, type, &val); }
        else if (!strncmp(type, "HVAR", 4)) { t = HVAR; sscanf(line, (fmt + " %31s").c_str(), &point, &xs, &ys, type, series); }
        else if (!strncmp(type, "QFIX", 4)) { t = QFIX; sscanf(line, (fmt + " " + real_fmt<T>()).c_str(), &point, &xs, &ys, type, &val); }
        else if (!strncmp(type, "QVAR", 4)) { t = QVAR; sscanf(line, (fmt + " %31s").c_str(), &point, &xs, &ys, type, series); }
        src_types.push_back(t);
        srcs.push_back(val);
        src_rows.push_back(0);
        src_t.emplace_back();
        src_v.emplace_back();
        if (t == HVAR || t == QVAR)
        {
            if (!read_series<T>(p, series, src_t.back(), src_v.back())) { fclose(fp); error = std::string("missing time series ") + series; return false; }
        }
    }
    fclose(fp);
    return true;
}

template <typename T>
void Sim<T>::read_stage_points()
{
    // classes/StagePoints.h:66-139
    std::string stage = read_kw_str(par.c_str(), "stagefile");
    if (stage.empty()) return;
    FILE* fp = fopen(stage.c_str(), "r");
    if (!fp) return;
    int n = 0;
    if (fscanf(fp, "%d", &n) != 1) n = 0;
    std::string fmt = std::string(real_fmt<T>()) + " " + real_fmt<T>();
    for (int i = 0; i < n; ++i)
    {
        T xs = T(0), ys = T(0);
        if (fscanf(fp, fmt.c_str(), &xs, &ys) != 2) break;
        stage_codes.push_back(morton((int)((xs - xmin) / dx), (int)((ys - ymin) / dx)));
    }
    fclose(fp);
}

template <typename T>
void Sim<T>::update_srcs(T now)
{
    // classes/PointSources.h:400-472
    for (size_t i = 0; i < srcs.size(); ++i)
        if (src_types[i] == HVAR || src_types[i] == QVAR)
            srcs[i] = interp_series(now, src_rows[i], src_t[i], src_v[i]);
}

template <typename T>
void Sim<T>::build_preflags()
{
    // mra/preflag_details.cu:3-93, mra/refine_high_wall.cu:3-57
    preflag.assign(n_det, 0);
    const int base = lvl_idx(L - 1);
    auto mark = [&](int code) {
        const long i = (long)base + code / 4;
        if (i >= 0 && i < n_det) preflag[i] = 1;
    };
    for (int c : stage_codes) mark(c);
    for (int b = 0; b < 4; ++b) for (int c : bnd[b].codes) mark(c);
    for (int c : src_codes) mark(c);
    if (refine_wall)
    {
        for (int j = 0; j < ref_thickness; ++j)
            for (int i = 0; i < xsz; ++i) mark(morton(i, ysz - 1 - j));
        for (int j = 0; j < ref_thickness; ++j)
            for (int i = 0; i < ysz; ++i) mark(morton(xsz - 1 - j, i));
    }
}

template <typename T>
bool Sim<T>::initial_modes(LeafArrays<T>& rm)
{
    // input/read_and_project_modes_dg2.cu:3-107, input/read_and_project_modes_fv1.cu:3-60,
    // mra/modal_projections.cu:28-88. Output: row-major finest modes in `rm`.
    const char* p = par.c_str();
    std::string dem = read_kw_str(p, "DEMfile");
    std::string start = read_kw_str(p, "startfile");
    std::vector<T> hr(F, T(0)), qxr(F, T(0)), qyr(F, T(0)), zr(F, wall_height);
    if (!start.empty()) read_raster<T>(start.c_str(), hr, M, wall_height);
    if (!read_raster<T>(dem.c_str(), zr, M, wall_height)) { error = "cannot read DEM"; return false; }
    if (startq2d)
    {
        read_raster<T>((start + ".Qx").c_str(), qxr, M, wall_height);
        read_raster<T>((start + ".Qy").c_str(), qyr, M, wall_height);
    }
    if (solver == HWFV1)
    {
        rm.h0 = hr; rm.qx0 = qxr; rm.qy0 = qyr; rm.z0 = zr;
        return true;
    }
    const int ID = M + 1;
    std::vector<T> hn((size_t)ID * ID), qxn((size_t)ID * ID), qyn((size_t)ID * ID), zn((size_t)ID * ID);
    const int ix = xsz + 1, iy = ysz + 1;
    for (int y = 0; y < ID; ++y)
        for (int x = 0; x < ID; ++x)
        {
            const bool bx = (x == ix - 1 || x == ID - 1);
            const bool by = (y == iy - 1 || y == ID - 1);
            const int i = bx ? x - 1 : x;
            const int j = by ? y - 1 : y;
            const size_t ni = (size_t)(ID - 1 - y) * ID + x;
            const size_t mi = (size_t)(M - 1 - j) * M + i;
            hn[ni] = hr[mi]; qxn[ni] = qxr[mi]; qyn[ni] = qyr[mi]; zn[ni] = zr[mi];
        }
    const T s3x4 = T(4.0) * std::sqrt(T(3.0));
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < F; ++idx)
    {
        const int x = idx % M, y = idx / M;
        const size_t SW = (size_t)y * ID + x, SE = (size_t)y * ID + x + 1;
        const size_t NW = (size_t)(y + 1) * ID + x, NE = (size_t)(y + 1) * ID + x + 1;
        auto avg = [&](const std::vector<T>& a) { return T(0.25) * (a[NW] + a[NE] + a[SE] + a[SW]); };
        auto sx = [&](const std::vector<T>& a) { return (a[NE] - a[NW] + a[SE] - a[SW]) / s3x4; };
        auto sy = [&](const std::vector<T>& a) { return (a[NE] - a[SE] + a[NW] - a[SW]) / s3x4; };
        rm.h0[idx] = avg(hn); rm.qx0[idx] = avg(qxn); rm.qy0[idx] = avg(qyn); rm.z0[idx] = avg(zn);
        rm.h1x[idx] = sx(hn); rm.qx1x[idx] = sx(qxn); rm.qy1x[idx] = sx(qyn); rm.z1x[idx] = sx(zn);
        rm.h1y[idx] = sy(hn); rm.qx1y[idx] = sy(qxn); rm.qy1y[idx] = sy(qyn); rm.z1y[idx] = sy(zn);
    }
    return true;
}

template <typename T>
void Sim<T>::topo_encode()
{
    // mra/preflag_topo.cu:3-43, mra/encode_topography_kernel_mw.cu:3-57, _hw.cu:3-51
    for (int level = L - 1; level >= 0; --level)
    {
        const int nthr = 1 << (2 * level);
        const int curr = lvl_idx(level), next = lvl_idx(level + 1);
        const T eps_local = epsilon / T(1 << (L - level));
        #pragma omp parallel for schedule(static)
        for (int idx = 0; idx < nthr; ++idx)
        {
            const int p = curr + idx, c = next + 4 * idx;
            T mx;
            if (solver == MWDG2)
            {
                Kids<T> k;
                for (int i = 0; i < 4; ++i) { k.u[0][i] = z0[c + i]; k.u[1][i] = z1x[c + i]; k.u[2][i] = z1y[c + i]; }
                z0[p] = encode_scale_mw(0, k);
                z1x[p] = encode_scale_mw(1, k);
                z1y[p] = encode_scale_mw(2, k);
                Det9<T> d = encode_details_mw(k);
                for (int t = 0; t < 3; ++t) for (int m = 0; m < 3; ++m) det[3][t][m][p] = d.d[t][m];
                mx = det9_max(d);
            }
            else
            {
                const T ch[4] = {z0[c], z0[c + 1], z0[c + 2], z0[c + 3]};
                const T a = hw_alpha(ch), b = hw_beta(ch), gm = hw_gamma(ch);
                det[3][0][0][p] = a; det[3][1][0][p] = b; det[3][2][0][p] = gm;
                z0[p] = hw_scale(ch);
                T m1 = std::fmax(std::fabs(a), std::fabs(b));
                mx = std::fmax(std::fabs(gm), m1);
            }
            if ((mx / maxes.z) >= eps_local) preflag[p] = 1;
        }
    }
}

template <typename T>
bool Sim<T>::init(const char* par_path, double eps_override, int solver_override)
{
    par = par_path;
    if (!read_params(eps_override, solver_override)) return false;
    read_stage_points();
    if (!read_boundaries()) return false;
    if (!read_point_sources()) return false;
    update_srcs(dt);  // PointSources constructor (classes/PointSources.h:84)
    build_preflags();

    const bool mw = (solver == MWDG2);
    for (auto* v : {&eta0, &qx0, &qy0, &z0}) v->assign(n_all, T(0));
    if (mw) for (auto* v : {&eta1x, &qx1x, &qy1x, &z1x, &eta1y, &qx1y, &qy1y, &z1y}) v->assign(n_all, T(0));
    for (int f = 0; f < 4; ++f) for (int t = 0; t < 3; ++t) for (int m = 0; m < 3; ++m)
        if (m == 0 || mw) det[f][t][m].assign(n_det, T(0));
    norm.assign(n_det, T(0));
    sig.assign(n_det, 1);  // mra/init_sig_details.cu
    enc.assign(n_det, 0);
    assem.alloc(F, true);
    buf.alloc(F, true);
    for (int d = 0; d < 4; ++d) { nb[d].alloc(F, true); buf_nb[d].alloc(F, false); }
    flag_ne.assign(F, 0);
    flag_sw.assign(F, 0);
    dt_cfl.assign(F, T(0));

    // modal values, row-major (buf plays d_buf_assem_sol at run_simulation.cu:127)
    if (!initial_modes(buf)) return false;
    // zorder/generate_all_morton_codes.cu, zorder/get_sorting_indices.cu:3-62
    rev_z_order.assign(F, 0);
    rev_row_major.assign(F, 0);
    for (int idx = 0; idx < F; ++idx)
    {
        const int code = morton(idx % M, idx / M);
        rev_z_order[code] = idx;
        rev_row_major[idx] = code;
    }
    // zorder/sort_finest_scale_coeffs_z_order.cu:3-35
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < F; ++k)
    {
        const int s = rev_z_order[k];
        assem.h0[k] = buf.h0[s]; assem.qx0[k] = buf.qx0[s]; assem.qy0[k] = buf.qy0[s]; assem.z0[k] = buf.z0[s];
        if (mw)
        {
            assem.h1x[k] = buf.h1x[s]; assem.qx1x[k] = buf.qx1x[s]; assem.qy1x[k] = buf.qy1x[s]; assem.z1x[k] = buf.z1x[s];
            assem.h1y[k] = buf.h1y[s]; assem.qx1y[k] = buf.qx1y[s]; assem.qy1y[k] = buf.qy1y[s]; assem.z1y[k] = buf.z1y[s];
        }
    }
    assem.length = F;
    // zorder/copy_finest_coefficients.cu:3-35
    const int fin = lvl_idx(L);
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < F; ++k)
    {
        const int h = fin + k;
        eta0[h] = assem.h0[k] + assem.z0[k]; qx0[h] = assem.qx0[k]; qy0[h] = assem.qy0[k]; z0[h] = assem.z0[k];
        if (mw)
        {
            eta1x[h] = assem.h1x[k] + assem.z1x[k]; qx1x[h] = assem.qx1x[k]; qy1x[h] = assem.qy1x[k]; z1x[h] = assem.z1x[k];
            eta1y[h] = assem.h1y[k] + assem.z1y[k]; qx1y[h] = assem.qx1y[k]; qy1y[h] = assem.qy1y[k]; z1y[h] = assem.z1y[k];
        }
    }
    // mra/insert_point_srcs.cu:3-29 (HFIX/HVAR subtract z0 at the source's index, as the reference does)
    for (size_t i = 0; i < srcs.size(); ++i)
    {
        const int code = src_codes[i];
        if (src_types[i] == HFIX || src_types[i] == HVAR) assem.h0[code] = srcs[i] - assem.z0[i];
        else if (src_types[i] == QFIX || src_types[i] == QVAR) assem.h0[code] += srcs[i] * dt / dx;
    }
    maxes = get_maxes(assem);   // run_simulation.cu:190
    topo_encode();              // run_simulation.cu:203
    return true;
}

// ============================================================================ step parts

template <typename T>
T Sim<T>::abs_max(const std::vector<T>& a, int n)
{
    // utilities/get_max_from_array.cu:3-64 (AbsMax reduction, initial value 0)
    T m = T(0);
    #pragma omp parallel for reduction(max : m) schedule(static)
    for (int i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
    return m;
}

template <typename T>
Maxes<T> Sim<T>::get_maxes(const LeafArrays<T>& s)
{
    // mra/get_max_scale_coeffs.cu:3-27 (qy max taken over qx0, as in the reference)
    const int n = s.length;
    T me = T(0), mh = T(0), mq = T(0), mz = T(0);
    #pragma omp parallel for reduction(max : me, mh, mq, mz) schedule(static)
    for (int i = 0; i < n; ++i)
    {
        me = std::max(me, std::fabs(s.h0[i] + s.z0[i]));  // mra/init_eta_temp.cu:3-15
        mh = std::max(mh, std::fabs(s.h0[i]));
        mq = std::max(mq, std::fabs(s.qx0[i]));
        mz = std::max(mz, std::fabs(s.z0[i]));
    }
    Maxes<T> r;
    r.eta = std::max(T(1), me);
    r.h = std::max(T(1), mh);
    r.qx = std::max(T(1), mq);
    r.qy = std::max(T(1), mq);
    r.z = std::max(T(1), mz);
    return r;
}

template <typename T>
void Sim<T>::zero_details()
{
    // mra/zero_details.cu:3-53
    for (int f = 0; f < 3; ++f) for (int t = 0; t < 3; ++t) for (int m = 0; m < 3; ++m)
        if (!det[f][t][m].empty()) std::fill(det[f][t][m].begin(), det[f][t][m].end(), T(0));
    std::fill(norm.begin(), norm.end(), T(0));
}

template <typename T>
void Sim<T>::reinsert(const LeafArrays<T>& s)
{
    // mra/reinsert_assem_sol.cu:3-32
    const bool mw = (solver == MWDG2);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        const int a = s.act[i];
        eta0[a] = s.h0[i] + s.z0[i]; qx0[a] = s.qx0[i]; qy0[a] = s.qy0[i];
        if (mw)
        {
            eta1x[a] = s.h1x[i] + s.z1x[i]; qx1x[a] = s.qx1x[i]; qy1x[a] = s.qy1x[i];
            eta1y[a] = s.h1y[i] + s.z1y[i]; qx1y[a] = s.qx1y[i]; qy1y[a] = s.qy1y[i];
        }
    }
}

template <typename T>
void Sim<T>::reinsert_point_srcs()
{
    // mra/reinsert_point_srcs.cu:3-29
    for (size_t i = 0; i < srcs.size(); ++i)
    {
        const int h = lvl_idx(L) + src_codes[i];
        if (src_types[i] == HFIX || src_types[i] == HVAR) eta0[h] = srcs[i];
        else if (src_types[i] == QFIX || src_types[i] == QVAR) eta0[h] += srcs[i] * dt / dx;
    }
}

template <typename T>
void Sim<T>::encode_flow(bool for_nghbrs)
{
    // mra/encode_flow.cu:3-92 with encode_flow_kernel_{mw,hw}.cu and the single-block
    // variants (levels 3..0 use epsilon / 2^(L-3): encode_flow_kernel_single_block_mw.cu:48)
    const bool mw = (solver == MWDG2);
    std::vector<T>* fld0[3] = {&eta0, &qx0, &qy0};
    std::vector<T>* fld1x[3] = {&eta1x, &qx1x, &qy1x};
    std::vector<T>* fld1y[3] = {&eta1y, &qx1y, &qy1y};
    const T fmax_[3] = {maxes.eta, maxes.qx, maxes.qy};
    for (int level = L - 1; level >= 0; --level)
    {
        const int eps_level = (level >= 4) ? level : 3;
        const T eps_local = epsilon / T(1 << (L - eps_level));
        const int nthr = 1 << (2 * level);
        const int curr = lvl_idx(level), next = lvl_idx(level + 1);
        #pragma omp parallel for schedule(static)
        for (int idx = 0; idx < nthr; ++idx)
        {
            const int p = curr + idx;
            const bool was_sig = sig[p] != 0;
            // the multi-block kernel clears the flag of every parent it visits unless it
            // only re-encodes scale coefficients (encode_flow_kernel_mw.cu:78)
            if (!for_nghbrs) { sig[p] = 0; enc[p] = was_sig ? 1 : 0; }
            if (!was_sig) continue;
            const int c = next + 4 * idx;
            T nd = T(0);
            for (int f = 0; f < 3; ++f)
            {
                if (mw)
                {
                    Kids<T> k;
                    for (int i = 0; i < 4; ++i)
                    {
                        k.u[0][i] = (*fld0[f])[c + i]; k.u[1][i] = (*fld1x[f])[c + i]; k.u[2][i] = (*fld1y[f])[c + i];
                    }
                    (*fld0[f])[p] = encode_scale_mw(0, k);
                    (*fld1x[f])[p] = encode_scale_mw(1, k);
                    (*fld1y[f])[p] = encode_scale_mw(2, k);
                    if (!for_nghbrs)
                    {
                        Det9<T> d = encode_details_mw(k);
                        for (int t = 0; t < 3; ++t) for (int m = 0; m < 3; ++m) det[f][t][m][p] = d.d[t][m];
                        nd = std::fmax(nd, det9_max(d) / fmax_[f]);
                    }
                }
                else
                {
                    const T ch[4] = {(*fld0[f])[c], (*fld0[f])[c + 1], (*fld0[f])[c + 2], (*fld0[f])[c + 3]};
                    (*fld0[f])[p] = hw_scale(ch);
                    const T a = hw_alpha(ch), b = hw_beta(ch), gm = hw_gamma(ch);
                    det[f][0][0][p] = a; det[f][1][0][p] = b; det[f][2][0][p] = gm;
                    T m1 = std::fmax(std::fabs(a), std::fabs(b));
                    m1 = std::fmax(std::fabs(gm), m1);
                    nd = std::fmax(nd, m1 / fmax_[f]);
                }
            }
            if (!for_nghbrs || !mw)
            {
                norm[p] = nd;
                sig[p] = (nd >= eps_local || preflag[p]) ? 1 : 0;
            }
        }
    }
}

template <typename T>
void Sim<T>::regularisation()
{
    // mra/regularisation.cu:3-27 (levels L-2 .. 0)
    for (int level = L - 2; level >= 0; --level)
    {
        const int nthr = 1 << (2 * level);
        const int curr = lvl_idx(level), next = lvl_idx(level + 1);
        #pragma omp parallel for schedule(static)
        for (int idx = 0; idx < nthr; ++idx)
        {
            const int c = next + 4 * idx;
            if (sig[c] || sig[c + 1] || sig[c + 2] || sig[c + 3]) sig[curr + idx] = 1;
        }
    }
}

template <typename T>
void Sim<T>::extra_significance()
{
    // mra/extra_significance.cu:3-33, mra/extra_significance_kernel.cu:3-42 (levels 0 .. L-2)
    for (int level = 0; level <= L - 2; ++level)
    {
        const int nthr = 1 << (2 * level);
        const int curr = lvl_idx(level), next = lvl_idx(level + 1);
        const T eps_local = epsilon / T(1 << (L - level));
        const T eps_extra = eps_local * std::pow(T(2.0), T(1.5) + T(1));
        #pragma omp parallel for schedule(static)
        for (int idx = 0; idx < nthr; ++idx)
        {
            const int p = curr + idx;
            if (sig[p] && norm[p] >= eps_extra)
            {
                const int c = next + 4 * idx;
                sig[c] = sig[c + 1] = sig[c + 2] = sig[c + 3] = 1;
            }
        }
    }
}

template <typename T>
void Sim<T>::decoding()
{
    // mra/decoding.cu:3-67, mra/decoding_kernel_mw.cu:3-142, mra/decoding_kernel_hw.cu:3-108
    const bool mw = (solver == MWDG2);
    std::vector<T>* fld0[3] = {&eta0, &qx0, &qy0};
    std::vector<T>* fld1x[3] = {&eta1x, &qx1x, &qy1x};
    std::vector<T>* fld1y[3] = {&eta1y, &qx1y, &qy1y};
    for (int level = 0; level < L; ++level)
    {
        const int nthr = 1 << (2 * level);
        const int curr = lvl_idx(level), next = lvl_idx(level + 1);
        #pragma omp parallel for schedule(static)
        for (int idx = 0; idx < nthr; ++idx)
        {
            const int p = curr + idx;
            if (!sig[p]) continue;
            // keep-values mode: an encoded parent's children already hold the values its
            // details were computed from (the decode would return them up to rounding)
            if (keep_values && enc[p]) continue;
            const int c = next + 4 * idx;
            for (int f = 0; f < 3; ++f)
            {
                if (mw)
                {
                    const T s[3] = {(*fld0[f])[p], (*fld1x[f])[p], (*fld1y[f])[p]};
                    Det9<T> d;
                    for (int t = 0; t < 3; ++t) for (int m = 0; m < 3; ++m) d.d[t][m] = det[f][t][m][p];
                    T out[3][4];
                    for (int ch = 0; ch < 4; ++ch) for (int k = 0; k < 3; ++k) out[k][ch] = decode_mw(ch, k, s, d);
                    for (int ch = 0; ch < 4; ++ch)
                    {
                        (*fld0[f])[c + ch] = out[0][ch]; (*fld1x[f])[c + ch] = out[1][ch]; (*fld1y[f])[c + ch] = out[2][ch];
                    }
                }
                else
                {
                    T out[4];
                    hw_decode((*fld0[f])[p], det[f][0][0][p], det[f][1][0][p], det[f][2][0][p], out);
                    for (int ch = 0; ch < 4; ++ch) (*fld0[f])[c + ch] = out[ch];
                }
            }
        }
    }
}

template <typename T>
void Sim<T>::traverse()
{
    // mra/traverse_tree_of_sig_details.cu:3-101 -> buf.act/lvl in Z-order
    const int nq = F / 4;
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < nq; ++idx)
    {
        const int fine = 4 * idx;
        int level = 0;
        int ind[4], lv[4];
        while (true)
        {
            const int code = fine >> (2 * (L - level));
            const int h = lvl_idx(level) + code;
            if (!sig[h])
            {
                for (int i = 0; i < 4; ++i) { ind[i] = h; lv[i] = level; }
                break;
            }
            level++;
            if (level == L)
            {
                const int child = lvl_idx(level) + 4 * code;
                for (int i = 0; i < 4; ++i) { ind[i] = child + i; lv[i] = level; }
                break;
            }
        }
        for (int i = 0; i < 4; ++i) { buf.act[fine + i] = ind[i]; buf.lvl[fine + i] = lv[i]; }
    }
}

template <typename T>
void Sim<T>::neighbours_and_compaction()
{
    const bool mw = (solver == MWDG2);
    // zorder/rev_z_order_act_idcs.cu:3-20 (Z-order -> row-major)
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < F; ++idx)
    {
        const int s = rev_row_major[idx];
        assem.act[idx] = buf.act[s];
        assem.lvl[idx] = buf.lvl[s];
    }
    // neighbours/find_neighbours.cu:3-430 (row-major)
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < F; ++idx)
    {
        const int x = idx % M, y = idx / M;
        const int lvl_local = assem.lvl[idx];
        const bool northern = (y == M - 1 || y == ysz - 1);
        const bool eastern = (x == M - 1 || x == xsz - 1);
        const bool southern = (y == 0);
        const bool western = (x == 0);
        const int h_dir = western ? WEST : eastern ? EAST : 0;
        const int v_dir = southern ? SOUTH : northern ? NORTH : 0;
        const int pos = v_dir | h_dir;
        const int li_local = lvl_idx(lvl_local);
        const int offs[4] = {M, 1, -M, -1};
        for (int d = 0; d < 4; ++d)
        {
            const int bit = (d == 0) ? NORTH : (d == 1) ? EAST : (d == 2) ? SOUTH : WEST;
            if (pos & bit)
            {
                nb[d].act[idx] = -1;
                nb[d].lvl[idx] = lvl_local;
                continue;
            }
            const int n = idx + offs[d];
            const int act_n = assem.act[n];
            const int lvl_n = assem.lvl[n];
            const int li_n = lvl_idx(lvl_n);
            const int code_n = act_n - li_n;
            const int diff = std::max(0, lvl_n - lvl_local);
            nb[d].act[idx] = std::min(li_local, li_n) + (code_n >> (2 * diff));
            nb[d].lvl[idx] = std::min(lvl_local, lvl_n);
        }
    }
    // neighbours/get_compaction_flags.cu:3-38 (on the Z-ordered traversal output)
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < F; ++idx)
    {
        const int cur = buf.act[idx];
        flag_ne[idx] = (idx < F - 1) ? (cur != buf.act[idx + 1]) : 1;
        flag_sw[idx] = (idx > 0) ? (cur != buf.act[idx - 1]) : 1;
    }
    // zorder/sort_neighbours_z_order.cu:3-31 (row-major -> Z-order)
    #pragma omp parallel for schedule(static)
    for (int idx = 0; idx < F; ++idx)
    {
        const int s = rev_z_order[idx];
        for (int d = 0; d < 4; ++d)
        {
            buf_nb[d].act[idx] = nb[d].act[s];
            if (mw) buf_nb[d].lvl[idx] = nb[d].lvl[s];
        }
    }
    // neighbours/compaction.cu:3-203 (stable selection by flag; parallel two-pass)
    auto select = [&](const std::vector<unsigned char>& flag, const std::vector<int>& in, std::vector<int>& out) {
        const int nt = omp_get_max_threads();
        std::vector<long> cnt(nt + 1, 0);
        #pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num(), nth = omp_get_num_threads();
            const long lo = (long)F * t / nth, hi = (long)F * (t + 1) / nth;
            long c = 0;
            for (long i = lo; i < hi; ++i) c += flag[i];
            cnt[t + 1] = c;
            #pragma omp barrier
            #pragma omp single
            for (int k = 1; k <= nth; ++k) cnt[k] += cnt[k - 1];
            long o = cnt[t];
            for (long i = lo; i < hi; ++i) if (flag[i]) out[o++] = in[i];
        }
        return (int)cnt[nt];
    };
    const int n = select(flag_ne, buf.act, assem.act);
    select(flag_ne, buf.lvl, assem.lvl);
    select(flag_ne, buf_nb[0].act, nb[0].act);
    select(flag_ne, buf_nb[1].act, nb[1].act);
    select(flag_sw, buf_nb[2].act, nb[2].act);
    select(flag_sw, buf_nb[3].act, nb[3].act);
    if (mw)
    {
        select(flag_ne, buf_nb[0].lvl, nb[0].lvl);
        select(flag_ne, buf_nb[1].lvl, nb[1].lvl);
        select(flag_sw, buf_nb[2].lvl, nb[2].lvl);
        select(flag_sw, buf_nb[3].lvl, nb[3].lvl);
    }
    assem.length = n;
}

template <typename T>
int Sim<T>::topology_from_sig(const unsigned char* s, int L_, int xsz_, int ysz_)
{
    L = L_;
    M = 1 << L;
    F = M * M;
    xsz = xsz_;
    ysz = ysz_;
    solver = MWDG2;
    n_det = lvl_idx(L);
    sig.assign(s, s + n_det);
    assem.alloc(F, false);
    buf.alloc(F, false);
    for (int d = 0; d < 4; ++d) { nb[d].alloc(F, false); buf_nb[d].alloc(F, false); }
    flag_ne.assign(F, 0);
    flag_sw.assign(F, 0);
    rev_z_order.assign(F, 0);
    rev_row_major.assign(F, 0);
    for (int idx = 0; idx < F; ++idx)
    {
        const int code = morton(idx % M, idx / M);
        rev_z_order[code] = idx;
        rev_row_major[idx] = code;
    }
    traverse();
    neighbours_and_compaction();
    return assem.length;
}

template <typename T>
void Sim<T>::load_soln(LeafArrays<T>& s)
{
    // neighbours/load_soln_and_nghbr_coeffs.cu:3-104
    const bool mw = (solver == MWDG2);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        auto fill = [&](LeafArrays<T>& o, int a) {
            o.h0[i] = eta0[a] - z0[a]; o.qx0[i] = qx0[a]; o.qy0[i] = qy0[a]; o.z0[i] = z0[a];
            if (mw)
            {
                o.h1x[i] = eta1x[a] - z1x[a]; o.qx1x[i] = qx1x[a]; o.qy1x[i] = qy1x[a]; o.z1x[i] = z1x[a];
                o.h1y[i] = eta1y[a] - z1y[a]; o.qx1y[i] = qx1y[a]; o.qy1y[i] = qy1y[a]; o.z1y[i] = z1y[a];
            }
        };
        fill(s, s.act[i]);
        for (int d = 0; d < 4; ++d)
        {
            const int a = nb[d].act[i];
            fill(nb[d], a == -1 ? 0 : a);
        }
    }
}

template <typename T>
void Sim<T>::add_ghost_cells(LeafArrays<T>& s)
{
    // neighbours/add_ghost_cells.cu:3-500, raster cases (test_case 0) only
    const bool mw = (solver == MWDG2);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        const int level = s.lvl[i];
        const int code = s.act[i] - lvl_idx(level);
        const int x = compact(code), y = compact(code >> 1);
        const bool finest = (level == L);
        for (int d = 0; d < 4; ++d)
        {
            if (nb[d].act[i] != -1) continue;
            LeafArrays<T>& G = nb[d];
            G.h0[i] = s.h0[i];
            G.qx0[i] = (d == 1 || d == 3) ? T(0) : s.qx0[i];
            G.qy0[i] = (d == 0 || d == 2) ? T(0) : s.qy0[i];
            G.z0[i] = s.z0[i];
            if (mw)
            {
                G.h1x[i] = T(0); G.qx1x[i] = T(0); G.qy1x[i] = T(0); G.z1x[i] = T(0);
                G.h1y[i] = T(0); G.qx1y[i] = T(0); G.qy1y[i] = T(0); G.z1y[i] = T(0);
            }
            const Boundary<T>& B = bnd[d];
            const bool bound = B.bound((d == 0 || d == 2) ? x : y);
            const bool border = (d == 0) ? (y == ysz - 1) : (d == 1) ? (x == xsz - 1) : (d == 2) ? (y == 0) : (x == 0);
            if (!(finest && bound && border)) continue;
            if (B.bdytype == FREE)
            {
                const T q = (d == 0 || d == 2) ? s.qy0[i] : s.qx0[i];
                G.h0[i] = std::pow((q * q) / g, T(1.0) / T(3.0));
                G.qx0[i] = s.qx0[i];
                G.qy0[i] = s.qy0[i];
            }
            else if (B.bdytype == HFIX || B.bdytype == HVAR)
            {
                s.h0[i] = B.inlet - s.z0[i];
                G.h0[i] = s.h0[i];
            }
            else if (B.bdytype == QFIX || B.bdytype == QVAR)
            {
                s.h0[i] = B.q_src(dt, dx);
                G.h0[i] = s.h0[i];
            }
        }
    }
}

// operators/apply_friction.cuh:7-53
template <typename T>
inline void apply_friction(T h, T tol_h, T tol_s, T& qx, T& qy, T n, T g, T dt)
{
    if (h < tol_h) { qx = T(0); qy = T(0); return; }
    const T ux = qx / h;
    const T uy = qy / h;
    if (std::fabs(ux) < tol_s && std::fabs(uy) < tol_s) { qx = T(0); qy = T(0); return; }
    const T Cf = g * n * n / std::pow(h, T(1.0) / T(3.0));
    const T speed = std::sqrt(ux * ux + uy * uy);
    const T Sf_x = -Cf * ux * speed;
    const T Sf_y = -Cf * uy * speed;
    const T D_x = T(1.0) + dt * Cf / h * (T(2.0) * ux * ux + uy * uy) / speed;
    const T D_y = T(1.0) + dt * Cf / h * (T(2.0) * uy * uy + ux * ux) / speed;
    qx += dt * Sf_x / D_x;
    qy += dt * Sf_y / D_y;
}

template <typename T>
void Sim<T>::friction_implicit()
{
    // operators/friction_implicit.cu:3-265
    const bool mw = (solver == MWDG2);
    LeafArrays<T>& s = assem;
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        {
            const T h = s.h0[i];
            const bool below_depth = (h < tol_h);
            const T ux = below_depth ? T(0) : s.qx0[i] / h;
            const T uy = below_depth ? T(0) : s.qy0[i] / h;
            const bool below_speed = (std::fabs(ux) < tol_s && std::fabs(uy) < tol_s);
            if (below_depth || below_speed) { s.qx0[i] = T(0); s.qy0[i] = T(0); continue; }
        }
        LeafArrays<T>* cells[5] = {&s, &nb[0], &nb[1], &nb[2], &nb[3]};
        if (!mw)
        {
            for (auto* c : cells) apply_friction(c->h0[i], tol_h, tol_s, c->qx0[i], c->qy0[i], manning, g, dt);
            continue;
        }
        // Gauss-point values are formed before the centre values are updated
        T hlx[5], hux[5], hly[5], huy[5], qxlx[5], qxux[5], qxly[5], qxuy[5], qylx[5], qyux[5], qyly[5], qyuy[5];
        for (int k = 0; k < 5; ++k)
        {
            LeafArrays<T>& c = *cells[k];
            hlx[k] = c.h0[i] - c.h1x[i]; hux[k] = c.h0[i] + c.h1x[i];
            hly[k] = c.h0[i] - c.h1y[i]; huy[k] = c.h0[i] + c.h1y[i];
            qxlx[k] = c.qx0[i] - c.qx1x[i]; qxux[k] = c.qx0[i] + c.qx1x[i];
            qxly[k] = c.qx0[i] - c.qx1y[i]; qxuy[k] = c.qx0[i] + c.qx1y[i];
            qylx[k] = c.qy0[i] - c.qy1x[i]; qyux[k] = c.qy0[i] + c.qy1x[i];
            qyly[k] = c.qy0[i] - c.qy1y[i]; qyuy[k] = c.qy0[i] + c.qy1y[i];
        }
        for (int k = 0; k < 5; ++k) apply_friction(cells[k]->h0[i], tol_h, tol_s, cells[k]->qx0[i], cells[k]->qy0[i], manning, g, dt);
        for (int k = 0; k < 5; ++k) apply_friction(hlx[k], tol_h, tol_s, qxlx[k], qylx[k], manning, g, dt);
        for (int k = 0; k < 5; ++k) apply_friction(hux[k], tol_h, tol_s, qxux[k], qyux[k], manning, g, dt);
        for (int k = 0; k < 5; ++k) apply_friction(hly[k], tol_h, tol_s, qxly[k], qyly[k], manning, g, dt);
        for (int k = 0; k < 5; ++k) apply_friction(huy[k], tol_h, tol_s, qxuy[k], qyuy[k], manning, g, dt);
        for (int k = 0; k < 5; ++k)
        {
            LeafArrays<T>& c = *cells[k];
            c.qx1x[i] = T(0.5) * (qxux[k] - qxlx[k]);
            c.qx1y[i] = T(0.5) * (qxuy[k] - qxly[k]);
            c.qy1x[i] = T(0.5) * (qyux[k] - qylx[k]);
            c.qy1y[i] = T(0.5) * (qyuy[k] - qyly[k]);
        }
    }
}

template <typename T> struct Planar { T _0, _1x, _1y; };
template <typename T> struct Vec3 { T h, qx, qy; };

// classes/FlowVector.h
template <typename T> inline Vec3<T> operator+(const Vec3<T>& a, const Vec3<T>& b) { return {a.h + b.h, a.qx + b.qx, a.qy + b.qy}; }
template <typename T> inline Vec3<T> operator-(const Vec3<T>& a, const Vec3<T>& b) { return {a.h - b.h, a.qx - b.qx, a.qy - b.qy}; }
template <typename T> inline Vec3<T> operator*(T s, const Vec3<T>& a) { return {s * a.h, s * a.qx, s * a.qy}; }
template <typename T> inline Vec3<T> operator/(const Vec3<T>& a, T s) { return {a.h / s, a.qx / s, a.qy / s}; }

template <typename T> inline T face_val(const Planar<T>& s, const Planar<T>& b)
{
    // operators/eval_loc_face_val_dg2.cuh:7-15
    return s._0 * b._0 + s._1x * b._1x + s._1y * b._1y;
}

template <typename T> inline Vec3<T> get_star(const Vec3<T>& U, T z, T z_inter, T tol_h)
{
    // classes/FlowVector.h:13-48
    const T eta = U.h + z;
    const T h_star = std::max(T(0), eta - z_inter);
    const T ux = (U.h < tol_h) ? T(0) : U.qx / U.h;
    const T uy = (U.h < tol_h) ? T(0) : U.qy / U.h;
    return {h_star, h_star * ux, h_star * uy};
}

template <typename T> inline Vec3<T> phys_flux_x(const Vec3<T>& U, T tol_h, T g)
{
    if (U.h < tol_h) return {T(0), T(0), T(0)};
    return {U.qx, U.qx * U.qx / U.h + g * U.h * U.h / T(2.0), U.qx * U.qy / U.h};
}
template <typename T> inline Vec3<T> phys_flux_y(const Vec3<T>& U, T tol_h, T g)
{
    if (U.h < tol_h) return {T(0), T(0), T(0)};
    return {U.qy, U.qx * U.qy / U.h, U.qy * U.qy / U.h + g * U.h * U.h / T(2.0)};
}

// operators/flux_HLL.cuh:9-111
template <typename T> inline Vec3<T> flux_hll_x(const Vec3<T>& Un, const Vec3<T>& Up, T tol_h, T g)
{
    if (Un.h < tol_h && Up.h < tol_h) return {T(0), T(0), T(0)};
    const T h_neg = (Un.h < tol_h) ? T(0) : Un.h;
    const T u_neg = (Un.h < tol_h) ? T(0) : Un.qx / Un.h;
    const T v_neg = (Un.h < tol_h) ? T(0) : Un.qy / Un.h;
    const T h_pos = (Up.h < tol_h) ? T(0) : Up.h;
    const T u_pos = (Up.h < tol_h) ? T(0) : Up.qx / Up.h;
    const T v_pos = (Up.h < tol_h) ? T(0) : Up.qy / Up.h;
    const T a_neg = std::sqrt(g * h_neg);
    const T a_pos = std::sqrt(g * h_pos);
    const T A = T(0.5) * (a_neg + a_pos) + T(0.25) * (u_neg - u_pos);
    const T h_star = A * A / g;
    const T u_star = T(0.5) * (u_neg + u_pos) + a_neg - a_pos;
    const T a_star = std::sqrt(g * h_star);
    const T s_neg = (h_neg < tol_h) ? u_pos - T(2.0) * a_pos : std::min(u_neg - a_neg, u_star - a_star);
    const T s_pos = (h_pos < tol_h) ? u_neg + T(2.0) * a_neg : std::max(u_pos + a_pos, u_star + a_star);
    const Vec3<T> F_neg = {Un.qx, u_neg * Un.qx + T(0.5) * g * h_neg * h_neg, Un.qy * u_neg};
    const Vec3<T> F_pos = {Up.qx, u_pos * Up.qx + T(0.5) * g * h_pos * h_pos, Up.qy * u_pos};
    if (s_neg >= T(0)) return F_neg;
    if (s_neg < T(0) && s_pos >= T(0))
    {
        Vec3<T> Fv;
        Fv.h = (s_pos * F_neg.h - s_neg * F_pos.h + s_neg * s_pos * (h_pos - h_neg)) / (s_pos - s_neg);
        Fv.qx = (s_pos * F_neg.qx - s_neg * F_pos.qx + s_neg * s_pos * (Up.qx - Un.qx)) / (s_pos - s_neg);
        const T s_mid = (s_neg * h_pos * (u_pos - s_pos) - s_pos * h_neg * (u_neg - s_neg)) /
                        (h_pos * (u_pos - s_pos) - h_neg * (u_neg - s_neg));
        Fv.qy = (s_neg < T(0) && s_mid >= T(0)) ? Fv.h * v_neg : Fv.h * v_pos;
        return Fv;
    }
    return F_pos;
}
template <typename T> inline Vec3<T> flux_hll_y(const Vec3<T>& Un, const Vec3<T>& Up, T tol_h, T g)
{
    const Vec3<T> rn = {Un.h, Un.qy, -Un.qx};
    const Vec3<T> rp = {Up.h, Up.qy, -Up.qx};
    const Vec3<T> Fr = flux_hll_x(rn, rp, tol_h, g);
    return {Fr.h, -Fr.qy, Fr.qx};
}

// zorder/get_x_coord.cuh, zorder/get_y_coord.cuh, zorder/get_spatial_coord.cuh
template <typename T> inline T cell_x(int h_idx, int level, int L, T dxf)
{
    const T dl = dxf * T(1 << (L - level));
    const int i = compact(h_idx - lvl_idx(level));
    return i * dl + dl / T(2.0);
}
template <typename T> inline T cell_y(int h_idx, int level, int L, T dyf)
{
    const T dl = dyf * T(1 << (L - level));
    const int j = compact((h_idx - lvl_idx(level)) >> 1);
    return j * dl + dl / T(2.0);
}

// operators/get_leg_basis.cuh:12-40 with get_{x,y}_face_{coord,unit}.cuh
template <typename T>
inline Planar<T> leg_basis(int h_idx_nb, int level_nb, int L, T x, T y, T dx_loc, T dy_loc, T dxf, T dyf, int dir)
{
    (void)h_idx_nb;
    T x_face = T(0), y_face = T(0);
    switch (dir)
    {
        case NORTH: x_face = x - dx_loc / T(2.0) + T(0.5) * dx_loc; y_face = y - dy_loc / T(2.0) + T(1.0) * dy_loc; break;
        case SOUTH: x_face = x - dx_loc / T(2.0) + T(0.5) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.0) * dy_loc; break;
        case EAST:  x_face = x - dx_loc / T(2.0) + T(1.0) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.5) * dy_loc; break;
        default:    x_face = x - dx_loc / T(2.0) + T(0.0) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.5) * dy_loc; break;
    }
    T xu, yu;
    if (h_idx_nb == -1)
    {
        xu = (dir == NORTH || dir == SOUTH) ? T(0.5) : (dir == EAST) ? T(0.0) : T(1.0);
        yu = (dir == EAST || dir == WEST) ? T(0.5) : (dir == NORTH) ? T(0.0) : T(1.0);
    }
    else
    {
        const T dxn = dxf * T(1 << (L - level_nb));
        const T xn = cell_x(h_idx_nb, level_nb, L, dxf);
        xu = (x_face - (xn - dxn / T(2.0))) / dxn;
        const T dyn = dyf * T(1 << (L - level_nb));
        const T yn = cell_y(h_idx_nb, level_nb, L, dyf);
        yu = (y_face - (yn - dyn / T(2.0))) / dyn;
    }
    const T s3 = std::sqrt(T(3.0));
    return {T(1.0), s3 * (T(2.0) * xu - T(1.0)), s3 * (T(2.0) * yu - T(1.0))};
}

// operators/minmod.cuh:7-24
template <typename T> inline T minmod(T a, T b, T c)
{
    if ((a * b > T(0)) && (a * c > T(0)))
    {
        const T sign_a = T((a > T(0)) - (a < T(0)));
        return std::min(std::fabs(a), std::min(std::fabs(b), std::fabs(c))) * sign_a;
    }
    return T(0);
}

// operators/get_limited_slopes.cuh:10-78
template <typename T>
inline void limited_slopes(const Planar<T>& u, const Planar<T>& un, const Planar<T>& ue, const Planar<T>& us,
                           const Planar<T>& uw, const Planar<T>& bn, const Planar<T>& be, const Planar<T>& bs,
                           const Planar<T>& bw, T dxf, T dyf, T tolK, T& out1x, T& out1y)
{
    const T s3 = std::sqrt(T(3.0));
    const T u_n_pos = face_val(un, bn);
    const T u_e_pos = face_val(ue, be);
    const T u_s_neg = face_val(us, bs);
    const T u_w_neg = face_val(uw, bw);
    const T u_n_neg = face_val(u, Planar<T>{T(1.0), T(0.0), s3});
    const T u_e_neg = face_val(u, Planar<T>{T(1.0), s3, T(0.0)});
    const T u_s_pos = face_val(u, Planar<T>{T(1.0), T(0.0), -s3});
    const T u_w_pos = face_val(u, Planar<T>{T(1.0), -s3, T(0.0)});
    const T jn = std::fabs(u_n_pos - u_n_neg);
    const T je = std::fabs(u_e_pos - u_e_neg);
    const T js = std::fabs(u_s_pos - u_s_neg);
    const T jw = std::fabs(u_w_pos - u_w_neg);
    const T norm_x = std::max(std::fabs(u._0 - u._1x), std::fabs(u._0 + u._1x));
    const T norm_y = std::max(std::fabs(u._0 - u._1y), std::fabs(u._0 + u._1y));
    const T DS_e = (norm_x > T(1e-12)) ? je / (T(0.5) * dxf * norm_x) : T(0.0);
    const T DS_w = (norm_x > T(1e-12)) ? jw / (T(0.5) * dxf * norm_x) : T(0.0);
    const T DS_n = (norm_y > T(1e-12)) ? jn / (T(0.5) * dyf * norm_y) : T(0.0);
    const T DS_s = (norm_y > T(1e-12)) ? js / (T(0.5) * dyf * norm_y) : T(0.0);
    out1x = (std::max(DS_e, DS_w) < tolK) ? u._1x : minmod(u._1x, (u._0 - uw._0) / s3, (ue._0 - u._0) / s3);
    out1y = (std::max(DS_n, DS_s) < tolK) ? u._1y : minmod(u._1y, (u._0 - us._0), (un._0 - u._0));
}

template <typename T>
void Sim<T>::limit_slopes(LeafArrays<T>& s, T max_h)
{
    // operators/limit_slopes.cu:3-238 (finest-level cells only)
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        const int level = s.lvl[i];
        if (level != L) continue;
        const T dxl = dx * T(1 << (L - level));
        const T dyl = dy * T(1 << (L - level));
        const int h_idx = s.act[i];
        const T x = cell_x(h_idx, level, L, dx);
        const T y = cell_y(h_idx, level, L, dy);
        if ((x >= xsz * dx) || (y >= ysz * dy)) continue;
        auto pl = [&](const std::vector<T>& a0, const std::vector<T>& a1, const std::vector<T>& a2) {
            return Planar<T>{a0[i], a1[i], a2[i]};
        };
        const Planar<T> h = pl(s.h0, s.h1x, s.h1y), qx = pl(s.qx0, s.qx1x, s.qx1y), qy = pl(s.qy0, s.qy1x, s.qy1y);
        Planar<T> hn[4], qxn[4], qyn[4], zn[4], eta_n[4], bas[4];
        const Planar<T> z = pl(s.z0, s.z1x, s.z1y);
        const int dirs[4] = {NORTH, EAST, SOUTH, WEST};
        for (int d = 0; d < 4; ++d)
        {
            hn[d] = pl(nb[d].h0, nb[d].h1x, nb[d].h1y);
            qxn[d] = pl(nb[d].qx0, nb[d].qx1x, nb[d].qx1y);
            qyn[d] = pl(nb[d].qy0, nb[d].qy1x, nb[d].qy1y);
            zn[d] = pl(nb[d].z0, nb[d].z1x, nb[d].z1y);
            eta_n[d] = {zn[d]._0 + hn[d]._0, zn[d]._1x + hn[d]._1x, zn[d]._1y + hn[d]._1y};
            bas[d] = leg_basis(nb[d].act[i], nb[d].lvl[i], L, x, y, dxl, dyl, dx, dy, dirs[d]);
        }
        const Planar<T> eta = {z._0 + h._0, z._1x + h._1x, z._1y + h._1y};
        T e1x, e1y, qx1x_, qx1y_, qy1x_, qy1y_;
        limited_slopes(eta, eta_n[0], eta_n[1], eta_n[2], eta_n[3], bas[0], bas[1], bas[2], bas[3], dx, dy, tol_Krivo, e1x, e1y);
        limited_slopes(qx, qxn[0], qxn[1], qxn[2], qxn[3], bas[0], bas[1], bas[2], bas[3], dx, dy, tol_Krivo, qx1x_, qx1y_);
        limited_slopes(qy, qyn[0], qyn[1], qyn[2], qyn[3], bas[0], bas[1], bas[2], bas[3], dx, dy, tol_Krivo, qy1x_, qy1y_);
        const bool ax = (T(0.05) * max_h < std::min(h._0, std::min(hn[1]._0, hn[3]._0)));
        const bool ay = (T(0.05) * max_h < std::min(h._0, std::min(hn[0]._0, hn[2]._0)));
        if (ax) { s.h1x[i] = e1x - z._1x; s.qx1x[i] = qx1x_; s.qy1x[i] = qy1x_; }
        if (ay) { s.h1y[i] = e1y - z._1y; s.qx1y[i] = qx1y_; s.qy1y[i] = qy1y_; }
    }
}

template <typename T>
void Sim<T>::dg2_update(LeafArrays<T>& ld, LeafArrays<T>& st, bool rkdg2)
{
    // operators/dg2_update.cu:3-359
    const T s3 = std::sqrt(T(3.0));
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < ld.length; ++i)
    {
        const T zc = ld.z0[i];
        const bool highwall = (std::fabs(zc - wall_height) < T(1e-10)) && (test_case == 0);
        const bool wet = (ld.h0[i] >= tol_h || nb[0].h0[i] >= tol_h || nb[1].h0[i] >= tol_h ||
                          nb[2].h0[i] >= tol_h || nb[3].h0[i] >= tol_h) && !highwall;
        dt_cfl[i] = initial_tstep;
        if (!wet) continue;
        const int level = ld.lvl[i];
        const T dxl = dx * T(1 << (L - level));
        const T dyl = dy * T(1 << (L - level));
        const int h_idx = ld.act[i];
        const T x = cell_x(h_idx, level, L, dx);
        const T y = cell_y(h_idx, level, L, dy);
        if ((x >= xsz * dx) || (y >= ysz * dy)) continue;
        const int dirs[4] = {NORTH, EAST, SOUTH, WEST};
        Planar<T> bas[4];
        for (int d = 0; d < 4; ++d) bas[d] = leg_basis(nb[d].act[i], nb[d].lvl[i], L, x, y, dxl, dyl, dx, dy, dirs[d]);
        const Planar<T> bn_loc = {T(1.0), T(0.0), s3};
        const Planar<T> be_loc = {T(1.0), s3, T(0.0)};
        const Planar<T> bs_loc = {T(1.0), T(0.0), -s3};
        const Planar<T> bw_loc = {T(1.0), -s3, T(0.0)};
        auto pl = [&](const std::vector<T>& a0, const std::vector<T>& a1, const std::vector<T>& a2) {
            return Planar<T>{a0[i], a1[i], a2[i]};
        };
        Planar<T> ch = pl(ld.h0, ld.h1x, ld.h1y), cqx = pl(ld.qx0, ld.qx1x, ld.qx1y), cqy = pl(ld.qy0, ld.qy1x, ld.qy1y);
        Planar<T> nh[4], nqx[4], nqy[4], nz[4];
        for (int d = 0; d < 4; ++d)
        {
            nh[d] = pl(nb[d].h0, nb[d].h1x, nb[d].h1y);
            nqx[d] = pl(nb[d].qx0, nb[d].qx1x, nb[d].qx1y);
            nqy[d] = pl(nb[d].qy0, nb[d].qy1x, nb[d].qy1y);
            nz[d] = pl(nb[d].z0, nb[d].z1x, nb[d].z1y);
        }
        const Planar<T> zp = pl(ld.z0, ld.z1x, ld.z1y);
        auto lfv = [&](const Planar<T>& h, const Planar<T>& qx, const Planar<T>& qy, const Planar<T>& b) {
            return Vec3<T>{face_val(h, b), face_val(qx, b), face_val(qy, b)};
        };
        const T z_n_pos = face_val(nz[0], bas[0]);
        const T z_e_pos = face_val(nz[1], bas[1]);
        const T z_s_neg = face_val(nz[2], bas[2]);
        const T z_w_neg = face_val(nz[3], bas[3]);
        const T z_n_neg = face_val(zp, bn_loc);
        const T z_e_neg = face_val(zp, be_loc);
        const T z_s_pos = face_val(zp, bs_loc);
        const T z_w_pos = face_val(zp, bw_loc);
        const T zi_n = std::max(z_n_neg, z_n_pos);
        const T zi_e = std::max(z_e_neg, z_e_pos);
        const T zi_s = std::max(z_s_neg, z_s_pos);
        const T zi_w = std::max(z_w_neg, z_w_pos);
        const Vec3<T> Us_n_pos = get_star(lfv(nh[0], nqx[0], nqy[0], bas[0]), z_n_pos, zi_n, tol_h);
        const Vec3<T> Us_e_pos = get_star(lfv(nh[1], nqx[1], nqy[1], bas[1]), z_e_pos, zi_e, tol_h);
        const Vec3<T> Us_s_neg = get_star(lfv(nh[2], nqx[2], nqy[2], bas[2]), z_s_neg, zi_s, tol_h);
        const Vec3<T> Us_w_neg = get_star(lfv(nh[3], nqx[3], nqy[3], bas[3]), z_w_neg, zi_w, tol_h);
        const Vec3<T> Us_n_neg = get_star(lfv(ch, cqx, cqy, bn_loc), z_n_neg, zi_n, tol_h);
        const Vec3<T> Us_e_neg = get_star(lfv(ch, cqx, cqy, be_loc), z_e_neg, zi_e, tol_h);
        const Vec3<T> Us_s_pos = get_star(lfv(ch, cqx, cqy, bs_loc), z_s_pos, zi_s, tol_h);
        const Vec3<T> Us_w_pos = get_star(lfv(ch, cqx, cqy, bw_loc), z_w_pos, zi_w, tol_h);
        const Vec3<T> F_n = flux_hll_y(Us_n_neg, Us_n_pos, tol_h, g);
        const Vec3<T> F_e = flux_hll_x(Us_e_neg, Us_e_pos, tol_h, g);
        const Vec3<T> F_s = flux_hll_y(Us_s_neg, Us_s_pos, tol_h, g);
        const Vec3<T> F_w = flux_hll_x(Us_w_neg, Us_w_pos, tol_h, g);
        const Vec3<T> U0x = (Us_e_neg + Us_w_pos) / T(2.0);
        const Vec3<T> U1x = (Us_e_neg - Us_w_pos) / (T(2.0) * s3);
        // Lx (coefficients h, qx, qy x modes 0, 1x, 1y)
        Vec3<T> Lx0 = (T(-1.0) * (F_e - F_w)) / dxl;
        Vec3<T> Lx1x = (-s3 / dxl) * (F_e + F_w - phys_flux_x(U0x - U1x, tol_h, g) - phys_flux_x(U0x + U1x, tol_h, g));
        // operators/get_bed_src.cuh:46-72
        {
            const T eta_e_neg = face_val(ch, be_loc) + z_e_neg;
            const T eta_w_pos = face_val(ch, bw_loc) + z_w_pos;
            const T zse = zi_e - std::max(T(0.0), -(eta_e_neg - zi_e));
            const T zsw = zi_w - std::max(T(0.0), -(eta_w_pos - zi_w));
            const T z1x_star = (zse - zsw) / (T(2.0) * s3);
            const T S0 = T(-2.0) * s3 * g * U0x.h * z1x_star / dxl;
            const T S1 = T(-2.0) * s3 * g * U1x.h * z1x_star / dxl;
            Lx0.qx = Lx0.qx + S0;
            Lx1x.qx = Lx1x.qx + S1;
            Lx0.h = Lx0.h + T(0); Lx0.qy = Lx0.qy + T(0);
            Lx1x.h = Lx1x.h + T(0); Lx1x.qy = Lx1x.qy + T(0);
        }
        const Vec3<T> U0y = (Us_n_neg + Us_s_pos) / T(2.0);
        const Vec3<T> U1y = (Us_n_neg - Us_s_pos) / (T(2.0) * s3);
        Vec3<T> Ly0 = (T(-1.0) * (F_n - F_s)) / dyl;
        Vec3<T> Ly1y = (-s3 / dyl) * (F_s + F_n - phys_flux_y(U0y - U1y, tol_h, g) - phys_flux_y(U0y + U1y, tol_h, g));
        {
            const T eta_n_neg = face_val(ch, bn_loc) + z_n_neg;
            const T eta_s_pos = face_val(ch, bs_loc) + z_s_pos;
            const T zsn = zi_n - std::max(T(0.0), -(eta_n_neg - zi_n));
            const T zss = zi_s - std::max(T(0.0), -(eta_s_pos - zi_s));
            const T z1y_star = (zsn - zss) / (T(2.0) * s3);
            const T S0 = T(-2.0) * s3 * g * U0y.h * z1y_star / dyl;
            const T S1 = T(-2.0) * s3 * g * U1y.h * z1y_star / dyl;
            Ly0.qy = Ly0.qy + S0;
            Ly1y.qy = Ly1y.qy + S1;
            Ly0.h = Ly0.h + T(0); Ly0.qx = Ly0.qx + T(0);
            Ly1y.h = Ly1y.h + T(0); Ly1y.qx = Ly1y.qx + T(0);
        }
        // FlowCoeffs sum: Lx has modes (0, 1x, 0), Ly has modes (0, 0, 1y)
        auto upd = [&](T c, T lx, T ly) { return c + dt * (lx + ly); };
        const T nh0 = upd(ch._0, Lx0.h, Ly0.h), nh1x = upd(ch._1x, Lx1x.h, T(0)), nh1y = upd(ch._1y, T(0), Ly1y.h);
        const T nqx0 = upd(cqx._0, Lx0.qx, Ly0.qx), nqx1x = upd(cqx._1x, Lx1x.qx, T(0)), nqx1y = upd(cqx._1y, T(0), Ly1y.qx);
        const T nqy0 = upd(cqy._0, Lx0.qy, Ly0.qy), nqy1x = upd(cqy._1x, Lx1x.qy, T(0)), nqy1y = upd(cqy._1y, T(0), Ly1y.qy);
        T& h0 = st.h0[i]; T& h1x = st.h1x[i]; T& h1y = st.h1y[i];
        T& q0 = st.qx0[i]; T& q1x = st.qx1x[i]; T& q1y = st.qx1y[i];
        T& r0 = st.qy0[i]; T& r1x = st.qy1x[i]; T& r1y = st.qy1y[i];
        h0 = rkdg2 ? T(0.5) * (nh0 + h0) : nh0;
        h1x = rkdg2 ? T(0.5) * (nh1x + h1x) : nh1x;
        h1y = rkdg2 ? T(0.5) * (nh1y + h1y) : nh1y;
        q0 = rkdg2 ? T(0.5) * (nqx0 + q0) : nqx0;
        q1x = rkdg2 ? T(0.5) * (nqx1x + q1x) : nqx1x;
        q1y = rkdg2 ? T(0.5) * (nqx1y + q1y) : nqx1y;
        r0 = rkdg2 ? T(0.5) * (nqy0 + r0) : nqy0;
        r1x = rkdg2 ? T(0.5) * (nqy1x + r1x) : nqy1x;
        r1y = rkdg2 ? T(0.5) * (nqy1y + r1y) : nqy1y;
        const bool below = (h0 < tol_h);
        if (below) { q0 = q1x = q1y = r0 = r1x = r1y = T(0); }
        else
        {
            const T ux = q0 / h0, uy = r0 / h0;
            const T dtx = CFL * dxl / (std::fabs(ux) + std::sqrt(g * h0));
            const T dty = CFL * dyl / (std::fabs(uy) + std::sqrt(g * h0));
            dt_cfl[i] = std::min(dtx, dty);
        }
    }
}

template <typename T>
void Sim<T>::fv1_update()
{
    // operators/fv1_update.cu:3-243
    LeafArrays<T>& s = assem;
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < s.length; ++i)
    {
        const bool wet = (s.h0[i] >= tol_h || nb[0].h0[i] >= tol_h || nb[1].h0[i] >= tol_h ||
                          nb[2].h0[i] >= tol_h || nb[3].h0[i] >= tol_h);
        dt_cfl[i] = initial_tstep;
        if (!wet) continue;
        const int level = s.lvl[i];
        const T dxl = dx * T(1 << (L - level));
        const T dyl = dy * T(1 << (L - level));
        const T z = s.z0[i];
        T h = s.h0[i], qx = s.qx0[i], qy = s.qy0[i];
        const T eta_loc = h + z;
        const T zn = nb[0].z0[i], ze = nb[1].z0[i], zs = nb[2].z0[i], zw = nb[3].z0[i];
        const T zin = std::max(z, zn), zie = std::max(z, ze), zis = std::max(z, zs), ziw = std::max(z, zw);
        const Vec3<T> U = {h, qx, qy};
        auto nv = [&](int d) { return Vec3<T>{nb[d].h0[i], nb[d].qx0[i], nb[d].qy0[i]}; };
        const Vec3<T> Usnn = get_star(U, z, zin, tol_h), Usnp = get_star(nv(0), zn, zin, tol_h);
        const Vec3<T> F_n = flux_hll_y(Usnn, Usnp, tol_h, g);
        const Vec3<T> Usen = get_star(U, z, zie, tol_h), Usep = get_star(nv(1), ze, zie, tol_h);
        const Vec3<T> F_e = flux_hll_x(Usen, Usep, tol_h, g);
        const Vec3<T> Ussn = get_star(nv(2), zs, zis, tol_h), Ussp = get_star(U, z, zis, tol_h);
        const Vec3<T> F_s = flux_hll_y(Ussn, Ussp, tol_h, g);
        const Vec3<T> Uswn = get_star(nv(3), zw, ziw, tol_h), Uswp = get_star(U, z, ziw, tol_h);
        const Vec3<T> F_w = flux_hll_x(Uswn, Uswp, tol_h, g);
        // operators/get_bed_src.cuh:7-44
        const T zsw = ziw - std::max(T(0.0), -(eta_loc - ziw));
        const T zse = zie - std::max(T(0.0), -(eta_loc - zie));
        const T bx = g * T(0.5) * (Uswp.h + Usen.h) * (zse - zsw) / dxl;
        const T zss = zis - std::max(T(0.0), -(eta_loc - zis));
        const T zsn = zin - std::max(T(0.0), -(eta_loc - zin));
        const T by = g * T(0.5) * (Ussp.h + Usnn.h) * (zsn - zss) / dyl;
        h = h - dt * (F_e.h - F_w.h) / dxl;
        qx = qx - dt * ((F_e.qx - F_w.qx) / dxl + bx);
        qy = qy - dt * (F_e.qy - F_w.qy) / dxl;
        h = h - dt * (F_n.h - F_s.h) / dyl;
        qx = qx - dt * (F_n.qx - F_s.qx) / dyl;
        qy = qy - dt * ((F_n.qy - F_s.qy) / dyl + by);
        const bool below_depth = (h < tol_h);
        const bool below_disch = (std::fabs(qx) < tol_q && std::fabs(qy) < tol_q);
        if (below_depth || below_disch) { qx = T(0); qy = T(0); }
        if (!below_depth)
        {
            const T ux = qx / h, uy = qy / h;
            const T dtx = CFL * dxl / (std::fabs(ux) + std::sqrt(g * h));
            const T dty = CFL * dyl / (std::fabs(uy) + std::sqrt(g * h));
            dt_cfl[i] = std::min(dtx, dty);
        }
        s.h0[i] = h;
        s.qx0[i] = qx;
        s.qy0[i] = qy;
    }
}

template <typename T>
T Sim<T>::min_dt()
{
    // operators/get_dt_CFL.cu:3-50
    T m = FLT_MAX;
    if (sizeof(T) == 8) m = T(DBL_MAX);
    const int n = assem.length;
    #pragma omp parallel for reduction(min : m) schedule(static)
    for (int i = 0; i < n; ++i) m = std::min(m, dt_cfl[i]);
    return m;
}

template <typename T>
bool Sim<T>::step()
{
    // source/run_simulation.cu:226-774
    if (!(current_time < sim_time)) return false;
    current_time += dt;
    if ((current_time - sim_time) > T(0))
    {
        current_time -= dt;
        dt = sim_time - current_time;
        current_time += dt;
    }
    zero_details();
    maxes = get_maxes(assem);
    if (!first) reinsert(assem);
    update_srcs(current_time);
    reinsert_point_srcs();
    if (epsilon > T(0) || first)
    {
        encode_flow(false);
        regularisation();
        extra_significance();
        decoding();
        traverse();
        neighbours_and_compaction();
    }
    load_soln(assem);
    for (int b = 0; b < 4; ++b)
        if (bnd[b].bdytype == HVAR || bnd[b].bdytype == QVAR)
            bnd[b].inlet = interp_series(current_time, bnd[b].row, bnd[b].tdata, bnd[b].vdata);
    add_ghost_cells(assem);
    if (manning > T(0)) friction_implicit();
    if (solver == HWFV1) fv1_update();
    else
    {
        // operators/copy_to_buf_assem_sol.cu:3-30
        buf.h0 = assem.h0; buf.h1x = assem.h1x; buf.h1y = assem.h1y;
        buf.qx0 = assem.qx0; buf.qx1x = assem.qx1x; buf.qx1y = assem.qx1y;
        buf.qy0 = assem.qy0; buf.qy1x = assem.qy1x; buf.qy1y = assem.qy1y;
        buf.z0 = assem.z0; buf.z1x = assem.z1x; buf.z1y = assem.z1y;
        buf.lvl = assem.lvl; buf.act = assem.act; buf.length = assem.length;
        if (limitslopes) limit_slopes(assem, maxes.h);
        dg2_update(assem, buf, false);
        reinsert(buf);
        if (epsilon > T(0)) encode_flow(true);
        load_soln(buf);
        add_ghost_cells(buf);
        if (limitslopes)
        {
            const T mh = abs_max(buf.h0, buf.length);
            maxes.h = mh;
            limit_slopes(buf, mh);
        }
        dg2_update(buf, assem, true);
    }
    dt = min_dt();
    timestep++;
    first = false;
    return true;
}

} // namespace oracle

// ============================================================================ C API

using namespace oracle;

struct OracleHandle
{
    int precision = 64;
    std::unique_ptr<Sim<double>> d;
    std::unique_ptr<Sim<float>> f;
    std::string err;
};

template <typename S> static void copy_leaves(S& s, int* act, int* lvl, int* nb_ids, int* nb_lvls)
{
    const int n = s.assem.length;
    for (int i = 0; i < n; ++i)
    {
        if (act) act[i] = s.assem.act[i];
        if (lvl) lvl[i] = s.assem.lvl[i];
        for (int d = 0; d < 4; ++d)
        {
            if (nb_ids) nb_ids[(size_t)d * n + i] = s.nb[d].act[i];
            if (nb_lvls) nb_lvls[(size_t)d * n + i] = s.nb[d].lvl[i];
        }
    }
}

template <typename S> static void copy_state(S& s, double* out)
{
    // 12 rows: h0 qx0 qy0 z0 h1x qx1x qy1x z1x h1y qx1y qy1y z1y (HWFV1: rows 4..11 = 0)
    const int n = s.assem.length;
    auto& a = s.assem;
    const decltype(&a.h0) rows[12] = {&a.h0, &a.qx0, &a.qy0, &a.z0, &a.h1x, &a.qx1x, &a.qy1x, &a.z1x,
                                      &a.h1y, &a.qx1y, &a.qy1y, &a.z1y};
    for (int r = 0; r < 12; ++r)
        for (int i = 0; i < n; ++i)
            out[(size_t)r * n + i] = rows[r]->empty() ? 0.0 : (double)(*rows[r])[i];
}

extern "C" {

void* oracle_create(const char* par, int precision, double eps_override, int solver_override, char* err, int errlen)
{
    auto* h = new OracleHandle();
    h->precision = precision;
    bool ok;
    std::string e;
    if (precision == 32)
    {
        h->f.reset(new Sim<float>());
        ok = h->f->init(par, eps_override, solver_override);
        e = h->f->error;
    }
    else
    {
        h->d.reset(new Sim<double>());
        ok = h->d->init(par, eps_override, solver_override);
        e = h->d->error;
    }
    if (!ok)
    {
        if (err && errlen > 0) snprintf(err, errlen, "%s", e.c_str());
        delete h;
        return nullptr;
    }
    return h;
}

void oracle_destroy(void* p) { delete static_cast<OracleHandle*>(p); }

// info: [L, xsz, ysz, solver, n_leaves, timestep, current_time, dt, dx, epsilon, n_det, n_all]
void oracle_info(void* p, double* info)
{
    auto* h = static_cast<OracleHandle*>(p);
    auto fill = [&](auto& s) {
        const double v[12] = {(double)s.L, (double)s.xsz, (double)s.ysz, (double)s.solver, (double)s.assem.length,
                              (double)s.timestep, (double)s.current_time, (double)s.dt, (double)s.dx,
                              (double)s.epsilon, (double)s.n_det, (double)s.n_all};
        for (int i = 0; i < 12; ++i) info[i] = v[i];
    };
    if (h->f) fill(*h->f); else fill(*h->d);
}

// Advances one step; returns 1 if a step was taken, 0 at the end of the simulation.
int oracle_step(void* p, double* dt_out, int* n_leaves_out)
{
    auto* h = static_cast<OracleHandle*>(p);
    int r;
    if (h->f) { r = h->f->step(); if (dt_out) *dt_out = h->f->dt; if (n_leaves_out) *n_leaves_out = h->f->assem.length; }
    else { r = h->d->step(); if (dt_out) *dt_out = h->d->dt; if (n_leaves_out) *n_leaves_out = h->d->assem.length; }
    return r;
}

int oracle_num_threads(void) { return omp_get_max_threads(); }

// Keep-values decode (the library's mwdg2_set_decode_mode 1) from the next step on.
void oracle_set_keep_values(void* p, int on)
{
    auto* h = static_cast<OracleHandle*>(p);
    if (h->f) h->f->keep_values = on != 0; else h->d->keep_values = on != 0;
}

void oracle_get_leaves(void* p, int* act, int* lvl, int* nb_ids, int* nb_lvls)
{
    auto* h = static_cast<OracleHandle*>(p);
    if (h->f) copy_leaves(*h->f, act, lvl, nb_ids, nb_lvls); else copy_leaves(*h->d, act, lvl, nb_ids, nb_lvls);
}

void oracle_get_state(void* p, double* out)
{
    auto* h = static_cast<OracleHandle*>(p);
    if (h->f) copy_state(*h->f, out); else copy_state(*h->d, out);
}

void oracle_get_sig(void* p, unsigned char* out)
{
    auto* h = static_cast<OracleHandle*>(p);
    if (h->f) memcpy(out, h->f->sig.data(), h->f->sig.size()); else memcpy(out, h->d->sig.data(), h->d->sig.size());
}

// field: 0 eta, 1 qx, 2 qy, 3 z; mode: 0, 1 (1x), 2 (1y); n_all values
int oracle_get_hier(void* p, int field, int mode, double* out)
{
    auto* h = static_cast<OracleHandle*>(p);
    auto get = [&](auto& s) {
        auto* v = s.hier(field, mode);
        if (!v) return 0;
        for (int i = 0; i < s.n_all; ++i) out[i] = (double)v[i];
        return 1;
    };
    return h->f ? get(*h->f) : get(*h->d);
}

// Leaf list and neighbours of a flag tree alone (Sim::topology_from_sig). Outputs hold up to
// 4^L leaves (nb_ids / nb_lvls laid out [4][4^L]); returns the number of leaves.
int oracle_leaf_topology(const unsigned char* sig, int L, int xsz, int ysz, int* act, int* lvl, int* nb_ids,
                         int* nb_lvls)
{
    Sim<double> s;
    const int n = s.topology_from_sig(sig, L, xsz, ysz);
    const size_t cap = (size_t)1 << (2 * L);
    for (int i = 0; i < n; ++i)
    {
        act[i] = s.assem.act[i];
        lvl[i] = s.assem.lvl[i];
        for (int d = 0; d < 4; ++d)
        {
            nb_ids[d * cap + i] = s.nb[d].act[i];
            nb_lvls[d * cap + i] = s.nb[d].lvl[i];
        }
    }
    return n;
}

void oracle_get_maxes(void* p, double* out)
{
    auto* h = static_cast<OracleHandle*>(p);
    auto get = [&](auto& s) { out[0] = s.maxes.eta; out[1] = s.maxes.h; out[2] = s.maxes.qx; out[3] = s.maxes.qy; out[4] = s.maxes.z; };
    if (h->f) get(*h->f); else get(*h->d);
}

} // extern "C"

template class oracle::Sim<double>;
template class oracle::Sim<float>;
