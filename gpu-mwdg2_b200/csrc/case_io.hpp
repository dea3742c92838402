// Host-side reading of a case in the reference's input formats and construction of the
// initial state (al0vya/gpu-mwdg2: source/input/*, source/classes/{SolverParams,
// SimulationParams,Boundary,PointSources,StagePoints,PlottingParams,SaveInterval}.h,
// source/mra/preflag_details.cu, source/input/read_and_project_modes_{dg2,fv1}.cu,
// source/mra/modal_projections.cu, source/zorder/*).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mwio {

// Text-keyword access to a parameter file, with the reference's matching rule: a line
// matches when its first token starts with the keyword; the first matching line wins.
class KeywordFile
{
public:
    bool load(const std::string& path, size_t max_lines = (size_t)-1);
    bool has(const char* kw) const;                       // read_keyword_bool.cpp
    std::string str(const char* kw) const;                // read_keyword_str.cpp
    int integer(const char* kw) const;                    // read_keyword_int.cpp
    template <typename T> T real(const char* kw, bool* found = nullptr) const;  // read_keyword_real.cpp
private:
    std::vector<std::string> lines_;
    int find(const char* kw) const;
};

template <typename T> struct Series
{
    std::vector<T> t, v;  // time (s), value
    int row = 0;
    // classes/Boundary.h:471-500 -- linear interpolation with a one-row advance per call
    T at(T now);
};

template <typename T> struct BoundarySide
{
    int start = 0, end = 0, type = 1 /*CLOSED*/;
    T inlet = T(0);
    bool varying = false;
    Series<T> series;
    std::vector<int> codes;  // Morton codes of the boundary cells (preflags)
};

template <typename T> struct PointSource
{
    int code = 0, type = 0;
    T value = T(0);
    bool varying = false;
    Series<T> series;
};

template <typename T> struct Case
{
    // classes/SolverParams.h:10-36
    int L = 0, solver = 2;
    T initial_tstep = T(0), epsilon = T(0), tol_h = T(1e-3), tol_q = T(0), tol_s = T(1e-9);
    T wall_height = T(0), CFL = T(0.3), tol_Krivo = T(9999.0);
    bool limitslopes = false, refine_wall = false, startq2d = false;
    int west_special = 0;             // west HFIX/HVAR ghost: 1 monai, 2 oregon-seaside (SimulationParams.h:29-30)
    int ref_thickness = 0;
    // classes/SimulationParams.h:8-32
    T xmin = T(0), ymin = T(0), xmax = T(0), ymax = T(0), g = T(9.80665), sim_time = T(0), manning = T(0);
    int xsz = 0, ysz = 0;
    T dx = T(0);
    // boundaries N, E, S, W; point sources; stage points
    BoundarySide<T> bnd[4];
    std::vector<PointSource<T>> srcs;
    std::vector<int> stage_codes;
    // outputs (classes/PlottingParams.h:20-53, classes/SaveInterval.h)
    std::string dirroot = "res", resroot = "res";
    bool cumulative = false, voutput_stage = false;
    bool vtk = false, c_prop = false, raster_out = false, voutput = false, qoutput = false, elevoff = false,
         depthoff = false;
    T massint = T(9999.0), saveint = T(9999.0);
    int massint_count = 9999, saveint_count = 9999;

    // initial state
    std::vector<uint8_t> preflag;     // get_lvl_idx(L) bytes
    std::vector<T> raster[4];         // h, qx, qy, z as read: row-major M x M (k_init_finest projects them)

    std::string error;
    int error_kind = 0;               // 1 IO, 2 PARSE

    // Reads everything; eps_override < 0 and solver_override 0 mean "from the file".
    bool read(const std::string& par, double eps_override, int solver_override);
};

// Fast ESRI-ASCII reader; values convert exactly as fscanf("%lf"/"%f") would.
template <typename T>
bool read_raster(const std::string& path, std::vector<T>& arr, int mesh_dim, T wall_height, std::string& err);

} // namespace mwio
