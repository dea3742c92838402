// Host-side case reading and initial-state construction (see case_io.hpp).
#include "case_io.hpp"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace mwio {

namespace {

int dil(int c)
{
    c &= 0x0000ffff;
    c = (c ^ (c << 8)) & 0x00ff00ff;
    c = (c ^ (c << 4)) & 0x0f0f0f0f;
    c = (c ^ (c << 2)) & 0x33333333;
    c = (c ^ (c << 1)) & 0x55555555;
    return c;
}
int morton(int x, int y) { return dil(x) | (dil(y) << 1); }
int lvl_idx(int level) { return ((1 << (2 * level)) - 1) / 3 + 3; }

template <typename T> const char* rfmt();
template <> const char* rfmt<double>() { return "%lf"; }
template <> const char* rfmt<float>() { return "%f"; }

template <typename T> T to_real(const char* s, char** end);
template <> double to_real<double>(const char* s, char** end) { return strtod(s, end); }
template <> float to_real<float>(const char* s, char** end) { return strtof(s, end); }

// Read a whole small text file as fgets-sized chunks (the reference reads with a
// 255-byte fgets buffer, so very long lines continue as further "lines").
bool load_chunks(const std::string& path, std::vector<std::string>& out, size_t max_lines = (size_t)-1)
{
    FILE* fp = fopen(path.c_str(), "r");
    if (!fp) return false;
    char buf[255];
    out.clear();
    while (out.size() < max_lines && fgets(buf, sizeof(buf), fp)) out.emplace_back(buf);
    fclose(fp);
    return true;
}

bool read_file(const std::string& path, std::string& out)
{
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) return false;
    fseek(fp, 0, SEEK_END);
    long n = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    size_t got = n > 0 ? fread(&out[0], 1, (size_t)n, fp) : 0;
    fclose(fp);
    out.resize(got);
    return true;
}

} // namespace

// ------------------------------------------------------------------- KeywordFile

bool KeywordFile::load(const std::string& path, size_t max_lines) { return load_chunks(path, lines_, max_lines); }

int KeywordFile::find(const char* kw) const
{
    const size_t n = strlen(kw);
    char tok[128];
    for (size_t i = 0; i < lines_.size(); ++i)
    {
        tok[0] = '\0';
        if (sscanf(lines_[i].c_str(), "%127s", tok) == 1 && strncmp(tok, kw, n) == 0) return (int)i;
    }
    return -1;
}

bool KeywordFile::has(const char* kw) const { return find(kw) >= 0; }

std::string KeywordFile::str(const char* kw) const
{
    // the value buffer keeps the last second token seen on any line up to the match
    const int m = find(kw);
    if (m < 0) return "";
    char tok[128], val[128] = {0};
    for (int i = 0; i <= m; ++i) sscanf(lines_[i].c_str(), "%127s %127s", tok, val);
    return val;
}

int KeywordFile::integer(const char* kw) const
{
    const int m = find(kw);
    if (m < 0) return 0;
    char tok[128];
    int v = 0;
    for (int i = 0; i <= m; ++i) sscanf(lines_[i].c_str(), "%127s %d", tok, &v);
    return v;
}

template <typename T> T KeywordFile::real(const char* kw, bool* found) const
{
    const int m = find(kw);
    if (found) *found = (m >= 0);
    if (m < 0) return T(0);
    char tok[128];
    T v = T(0);
    std::string f = std::string("%127s ") + rfmt<T>();
    for (int i = 0; i <= m; ++i) sscanf(lines_[i].c_str(), f.c_str(), tok, &v);
    return v;
}

// ------------------------------------------------------------------- Series

template <typename T> T Series<T>::at(T now)
{
    const int len = (int)t.size();
    auto cl = [&](int i) { return i < 0 ? 0 : (i >= len ? len - 1 : i); };
    if ((row - 1) < len)
    {
        T t1 = t[cl(row)], t2 = t[cl(row + 1)];
        if (now > t2)
        {
            row++;
            t1 = t[cl(row)];
            t2 = t[cl(row + 1)];
        }
        const T v1 = v[cl(row)], v2 = v[cl(row + 1)];
        return v1 + (v2 - v1) / (t2 - t1) * (now - t1);
    }
    return v[len - 1];
}

// Time series "name" of the .bdy file (classes/Boundary.h:427-466)
template <typename T>
static bool read_series(const std::string& bdy, const char* name, Series<T>& s, std::string& err)
{
    std::vector<std::string> lines;
    if (!load_chunks(bdy, lines)) { err = "cannot open bdyfile " + bdy; return false; }
    const size_t n = strlen(name);
    char tok[128];
    size_t i = 0;
    for (; i < lines.size(); ++i)
        if (sscanf(lines[i].c_str(), "%127s", tok) == 1 && !strncmp(tok, name, n)) break;
    if (i >= lines.size()) { err = std::string("time series ") + name + " not found in " + bdy; return false; }
    int rows = 0;
    char unit[128] = {0};
    if (i + 1 >= lines.size() || sscanf(lines[i + 1].c_str(), "%d %127s", &rows, unit) < 1 || rows <= 0)
    {
        err = std::string("time series ") + name + ": bad row count";
        return false;
    }
    const int mult = !strncmp(unit, "seconds", 7) ? 1 : !strncmp(unit, "minutes", 7) ? 60 : 3600;
    s.t.assign(rows, T(0));
    s.v.assign(rows, T(0));
    std::string f = std::string(rfmt<T>()) + " " + rfmt<T>();
    for (int r = 0; r < rows; ++r)
    {
        if (i + 2 + r >= lines.size()) { err = std::string("time series ") + name + ": too few rows"; return false; }
        sscanf(lines[i + 2 + r].c_str(), f.c_str(), &s.v[r], &s.t[r]);
        s.t[r] *= mult;
    }
    s.row = 0;
    return true;
}

// ------------------------------------------------------------------- rasters

template <typename T>
bool read_raster(const std::string& path, std::vector<T>& arr, int mesh_dim, T wall_height, std::string& err)
{
    // input/read_raster_file.cpp:3-48: six header pairs, then nrows x ncols values,
    // first row northernmost; stored south-up with row stride mesh_dim.
    std::string text;
    if (!read_file(path, text)) { err = "cannot open raster " + path; return false; }
    const char* p = text.c_str();
    char* e = nullptr;
    int ncols = 0, nrows = 0;
    for (int h = 0; h < 6; ++h)
    {
        while (*p && isspace((unsigned char)*p)) ++p;
        while (*p && !isspace((unsigned char)*p)) ++p;    // key
        if (h < 2)
        {
            long v = strtol(p, &e, 10);
            if (e == p) { err = "bad raster header in " + path; return false; }
            (h == 0 ? ncols : nrows) = (int)v;
        }
        else
        {
            to_real<T>(p, &e);
            if (e == p) { err = "bad raster header in " + path; return false; }
        }
        p = e;
    }
    if (ncols <= 0 || nrows <= 0 || ncols > mesh_dim || nrows > mesh_dim)
    {
        err = "raster " + path + " does not fit the 2^max_ref_lvl mesh";
        return false;
    }
    for (int j = 0; j < nrows; ++j)
    {
        T* row = arr.data() + (size_t)(nrows - 1 - j) * mesh_dim;
        for (int i = 0; i < ncols; ++i)
        {
            const T v = to_real<T>(p, &e);
            if (e == p) { err = "raster " + path + " has too few values"; return false; }
            p = e;
            const bool nodata = std::fabs(v + T(9999.0)) < T(1e-10);
            row[i] = nodata ? wall_height : v;
        }
    }
    return true;
}

// ------------------------------------------------------------------- Case

template <typename T>
bool Case<T>::read(const std::string& par, double eps_override, int solver_override)
{
    auto fail = [&](int kind, const std::string& msg) { error = msg; error_kind = kind; return false; };
    KeywordFile kf;
    if (!kf.load(par)) return fail(1, "cannot open parameter file " + par);
    if (kf.integer("test_case") != 0) return fail(2, "built-in test cases (test_case != 0) are not supported; use rasters");
    // classes/SolverParams.cu:5-48
    L = kf.integer("max_ref_lvl");
    initial_tstep = kf.real<T>("initial_tstep");
    epsilon = kf.real<T>("epsilon");
    wall_height = kf.real<T>("wall_height");
    if (kf.has("hwfv1")) { solver = 1; CFL = T(0.5); }
    else if (kf.has("mwdg2")) { solver = 2; CFL = T(0.3); }
    else return fail(2, "no solver keyword (hwfv1 or mwdg2) in " + par);
    limitslopes = kf.has("limitslopes");
    if (limitslopes) tol_Krivo = kf.real<T>("tol_Krivo");
    refine_wall = kf.has("refine_wall");
    if (refine_wall) ref_thickness = kf.integer("ref_thickness");
    startq2d = kf.has("startq2d");
    // command-line overrides (input/read_command_line_params.cpp:12-47)
    if (eps_override >= 0) epsilon = T(eps_override);
    if (solver_override == 1) { solver = 1; CFL = T(0.5); }
    if (solver_override == 2) { solver = 2; CFL = T(0.3); }
    bool has_cfl = false;
    const T cfl = kf.real<T>("CFL", &has_cfl);  // extension: the reference's CFL is fixed
    if (has_cfl && cfl > T(0)) CFL = cfl;
    // 14 at most: the hierarchy's slot count (4^(L+1) - 1) / 3 + 3 is formed in 32-bit ints,
    // and a level-15 mesh would not fit in one GPU's memory anyway
    if (L < 6 || L > 14) return fail(2, "max_ref_lvl must be between 6 and 14");
    // classes/SimulationParams.cpp:15-33
    const std::string dem = kf.str("DEMfile");
    if (dem.empty()) return fail(2, "no DEMfile in " + par);
    KeywordFile df;  // header keywords only: the first lines of the raster
    if (!df.load(dem, 16)) return fail(1, "cannot open DEM " + dem);
    xsz = df.integer("ncols");
    ysz = df.integer("nrows");
    xmin = df.real<T>("xllcorner");
    ymin = df.real<T>("yllcorner");
    const T cellsize = df.real<T>("cellsize");
    xmax = xmin + xsz * cellsize;
    ymax = ymin + ysz * cellsize;
    sim_time = kf.real<T>("sim_time");
    manning = kf.real<T>("fpfric");
    // classes/SimulationParams.cpp:31-32 (monai wins when both are present, as in
    // neighbours/add_ghost_cells.cu:450-471)
    west_special = kf.has("monai") ? 1 : (kf.has("oregon-seaside") ? 2 : 0);
    const int M = 1 << L;
    if (xsz <= 0 || ysz <= 0 || xsz > M || ysz > M) return fail(2, "DEM size must be within 2^max_ref_lvl");
    // input/read_cell_size.cpp:5-41 (fifth header value)
    {
        FILE* fp = fopen(dem.c_str(), "r");
        if (!fp) return fail(1, "cannot open DEM " + dem);
        char b[128];
        int d = 0;
        T cs = T(0);
        std::string f = std::string("%127s ") + rfmt<T>();
        if (fscanf(fp, "%127s %d", b, &d) != 2 || fscanf(fp, "%127s %d", b, &d) != 2) { fclose(fp); return fail(2, "bad DEM header"); }
        for (int k = 0; k < 3; ++k) if (fscanf(fp, f.c_str(), b, &cs) != 2) { fclose(fp); return fail(2, "bad DEM header"); }
        fclose(fp);
        dx = cs;
    }
    if (!(dx > T(0))) return fail(2, "non-positive cellsize");
    // classes/PlottingParams.h:20-53, classes/SaveInterval.h:10-50
    cumulative = kf.has("cumulative");
    voutput_stage = kf.has("voutput_stage");
    vtk = kf.has("vtk");
    c_prop = kf.has("c_prop");
    raster_out = kf.has("raster_out");
    voutput = kf.has("voutput");   // a `voutput_stage` line also matches, as in the reference
    qoutput = kf.has("qoutput");
    elevoff = kf.has("elevoff");
    depthoff = kf.has("depthoff");
    { std::string s = kf.str("resroot"); if (!s.empty()) resroot = s; }
    { std::string s = kf.str("dirroot"); if (!s.empty()) dirroot = s; }
    { bool f = false; T v = kf.real<T>("massint", &f); if (f) { massint = v; massint_count = 0; } }
    { bool f = false; T v = kf.real<T>("saveint", &f); if (f) { saveint = v; saveint_count = 0; } }

    const std::string bci = kf.str("bcifile");
    const std::string bdy = kf.str("bdyfile");
    // classes/StagePoints.h:66-139
    const std::string stage = kf.str("stagefile");
    if (!stage.empty())
    {
        FILE* fp = fopen(stage.c_str(), "r");
        if (!fp) return fail(1, "cannot open stagefile " + stage);
        int n = 0;
        if (fscanf(fp, "%d", &n) != 1) n = 0;
        std::string f = std::string(rfmt<T>()) + " " + rfmt<T>();
        for (int i = 0; i < n; ++i)
        {
            T xs = T(0), ys = T(0);
            if (fscanf(fp, f.c_str(), &xs, &ys) != 2) { fclose(fp); return fail(2, "stagefile has too few points"); }
            stage_codes.push_back(morton((int)((xs - xmin) / dx), (int)((ys - ymin) / dx)));
        }
        fclose(fp);
    }
    // classes/Boundary.h:92-371 and classes/PointSources.h:117-279 (one .bci file)
    if (!bci.empty())
    {
        std::vector<std::string> lines;
        if (!load_chunks(bci, lines)) return fail(1, "cannot open bcifile " + bci);
        const std::string f4 = std::string("%c ") + rfmt<T>() + " " + rfmt<T>() + " %7s";
        const char dirs[4] = {'N', 'E', 'S', 'W'};
        for (int b = 0; b < 4; ++b)
        {
            BoundarySide<T>& B = bnd[b];
            const T origin = (b == 0 || b == 2) ? xmin : ymin;
            for (const std::string& ln : lines)
            {
                char d = 0, type[8] = {0};
                T lo = T(0), hi = T(0);
                sscanf(ln.c_str(), f4.c_str(), &d, &lo, &hi, type);
                if (d != dirs[b]) continue;
                char series[32] = {0};
                T inlet = T(0);
                int bt = 1;
                if (!strncmp(type, "CLOSED", 6)) bt = 1;
                else if (!strncmp(type, "FREE", 4)) bt = 2;
                else if (!strncmp(type, "HFIX", 4)) { bt = 4; sscanf(ln.c_str(), (f4 + " " + rfmt<T>()).c_str(), &d, &lo, &hi, type, &inlet); }
                else if (!strncmp(type, "HVAR", 4)) { bt = 8; sscanf(ln.c_str(), (f4 + " %31s").c_str(), &d, &lo, &hi, type, series); }
                else if (!strncmp(type, "QFIX", 4)) { bt = 16; sscanf(ln.c_str(), (f4 + " " + rfmt<T>()).c_str(), &d, &lo, &hi, type, &inlet); }
                else if (!strncmp(type, "QVAR", 4)) { bt = 32; sscanf(ln.c_str(), (f4 + " %31s").c_str(), &d, &lo, &hi, type, series); }
                B.start = (int)((lo - origin) / dx);
                B.end = (int)((hi - origin) / dx - T(1));
                B.type = bt;
                B.inlet = inlet;
                const int nc = std::max(0, B.end - B.start + 1);
                B.codes.resize(nc);
                for (int i = 0; i < nc; ++i)
                {
                    const int c = B.start + i;
                    B.codes[i] = (b == 0) ? morton(c, ysz - 1) : (b == 1) ? morton(xsz - 1, c)
                               : (b == 2) ? morton(c, 0) : morton(0, c);
                }
                if (bt == 8 || bt == 32)
                {
                    B.varying = true;
                    if (!read_series<T>(bdy, series, B.series, error)) { error_kind = 2; return false; }
                }
                break;
            }
        }
        for (const std::string& ln : lines)
        {
            char pch = 0, type[8] = {0};
            T xs = T(0), ys = T(0);
            sscanf(ln.c_str(), f4.c_str(), &pch, &xs, &ys, type);
            if (pch != 'P') continue;
            PointSource<T> s;
            s.code = morton((int)((xs - xmin) / dx), (int)((ys - ymin) / dx));
            char series[32] = {0};
            if (!strncmp(type, "HFIX", 4)) { s.type = 4; sscanf(ln.c_str(), (f4 + " " + rfmt<T>()).c_str(), &pch, &xs, &ys, type, &s.value); }
            else if (!strncmp(type, "HVAR", 4)) { s.type = 8; sscanf(ln.c_str(), (f4 + " %31s").c_str(), &pch, &xs, &ys, type, series); }
            else if (!strncmp(type, "QFIX", 4)) { s.type = 16; sscanf(ln.c_str(), (f4 + " " + rfmt<T>()).c_str(), &pch, &xs, &ys, type, &s.value); }
            else if (!strncmp(type, "QVAR", 4)) { s.type = 32; sscanf(ln.c_str(), (f4 + " %31s").c_str(), &pch, &xs, &ys, type, series); }
            if (s.code < 0 || s.code >= M * M) return fail(2, "point source outside the mesh");
            if (s.type == 8 || s.type == 32)
            {
                s.varying = true;
                if (!read_series<T>(bdy, series, s.series, error)) { error_kind = 2; return false; }
            }
            srcs.push_back(s);
        }
    }
    // PointSources constructor: values at t = dt = 0.001 (classes/PointSources.h:84)
    const T dt0 = T(0.001);
    for (auto& s : srcs) if (s.varying) s.value = s.series.at(dt0);

    // preflags (mra/preflag_details.cu:3-93, mra/refine_high_wall.cu:3-57)
    const int n_det = lvl_idx(L);
    preflag.assign(n_det, 0);
    const int base = lvl_idx(L - 1);
    auto mark = [&](int code) { const long i = (long)base + code / 4; if (i >= base && i < n_det) preflag[i] = 1; };
    for (int c : stage_codes) mark(c);
    for (int b = 0; b < 4; ++b) for (int c : bnd[b].codes) mark(c);
    for (auto& s : srcs) mark(s.code);
    if (refine_wall)
    {
        for (int j = 0; j < ref_thickness; ++j) for (int i = 0; i < xsz; ++i) mark(morton(i, ysz - 1 - j));
        for (int j = 0; j < ref_thickness; ++j) for (int i = 0; i < ysz; ++i) mark(morton(xsz - 1 - j, i));
    }

    // initial rasters (h, qx, qy, z), row-major as read
    const size_t F = (size_t)M * M;
    std::vector<T> hr(F, T(0)), qxr(F, T(0)), qyr(F, T(0)), zr(F, wall_height);
    const std::string start = kf.str("startfile");
    std::string e2;
    if (!start.empty() && !read_raster<T>(start, hr, M, wall_height, e2))
    {
        FILE* fp = fopen(start.c_str(), "r");
        if (fp) { fclose(fp); return fail(2, e2); }   // unreadable content is an error; a missing file means "defaults"
    }
    if (!read_raster<T>(dem, zr, M, wall_height, e2)) return fail(2, e2);
    if (startq2d)
    {
        read_raster<T>(start + ".Qx", qxr, M, wall_height, e2);
        read_raster<T>(start + ".Qy", qyr, M, wall_height, e2);
    }
    // the modal projection, Z-order placement and initial point-source insertion run on the
    // device (init.cuh)
    raster[0].swap(hr); raster[1].swap(qxr); raster[2].swap(qyr); raster[3].swap(zr);
    return true;
}

template struct Series<double>;
template struct Series<float>;
template struct Case<double>;
template struct Case<float>;
template bool read_raster<double>(const std::string&, std::vector<double>&, int, double, std::string&);
template bool read_raster<float>(const std::string&, std::vector<float>&, int, float, std::string&);
template double KeywordFile::real<double>(const char*, bool*) const;
template float KeywordFile::real<float>(const char*, bool*) const;

} // namespace mwio
