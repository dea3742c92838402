// CPU oracle: input readers restating the reference's parsers.
//
// TEST INFRASTRUCTURE ONLY (see oracle_common.hpp). Relative file names are opened
// relative to the current working directory, as the reference does.
#pragma once

#include "oracle_common.hpp"

namespace oracle {

template <typename T> inline const char* real_fmt();
template <> inline const char* real_fmt<double>() { return "%lf"; }
template <> inline const char* real_fmt<float>() { return "%f"; }

// input/read_keyword_real.cpp:3-45 (first token prefix-matched against keyword)
template <typename T>
T read_kw_real(const char* file, const char* kw, bool* found = nullptr)
{
    if (found) *found = false;
    FILE* fp = fopen(file, "r");
    if (!fp) return T(0);
    const size_t n = strlen(kw);
    T value = T(0);
    char kwbuf[128] = {0};
    char line[255] = {0};
    std::string fmt = std::string("%127s ") + real_fmt<T>();
    while (strncmp(kwbuf, kw, n))
    {
        if (!fgets(line, sizeof(line), fp)) { fclose(fp); return T(0); }
        sscanf(line, fmt.c_str(), kwbuf, &value);
    }
    fclose(fp);
    if (found) *found = true;
    return value;
}

// input/read_keyword_int.cpp:3-41
inline int read_kw_int(const char* file, const char* kw)
{
    FILE* fp = fopen(file, "r");
    if (!fp) return 0;
    const size_t n = strlen(kw);
    int value = 0;
    char kwbuf[128] = {0};
    char line[255] = {0};
    while (strncmp(kwbuf, kw, n))
    {
        if (!fgets(line, sizeof(line), fp)) { fclose(fp); return 0; }
        sscanf(line, "%127s %d", kwbuf, &value);
    }
    fclose(fp);
    return value;
}

// input/read_keyword_bool.cpp:3-43 -- true if any line's first token starts with kw
inline bool read_kw_bool(const char* file, const char* kw)
{
    FILE* fp = fopen(file, "r");
    if (!fp) return false;
    const size_t n = strlen(kw);
    char kwbuf[128] = {0};
    char line[255] = {0};
    while (strncmp(kwbuf, kw, n))
    {
        if (!fgets(line, sizeof(line), fp)) { fclose(fp); return false; }
        sscanf(line, "%127s", kwbuf);
    }
    fclose(fp);
    return true;
}

// input/read_keyword_str.cpp:3-41
inline std::string read_kw_str(const char* file, const char* kw)
{
    FILE* fp = fopen(file, "r");
    if (!fp) return "";
    const size_t n = strlen(kw);
    char kwbuf[128] = {0};
    char val[128] = {0};
    char line[255] = {0};
    while (strncmp(kwbuf, kw, n))
    {
        if (!fgets(line, sizeof(line), fp)) { fclose(fp); return ""; }
        sscanf(line, "%127s %127s", kwbuf, val);
    }
    fclose(fp);
    return std::string(val);
}

// input/read_cell_size.cpp:5-41 -- fifth header value of the DEM
template <typename T> T read_cell_size(const char* par)
{
    std::string dem = read_kw_str(par, "DEMfile");
    FILE* fp = fopen(dem.c_str(), "r");
    if (!fp) return T(0);
    char buf[128];
    int dummy = 0;
    T cs = T(0);
    std::string fmt = std::string("%127s ") + real_fmt<T>();
    if (fscanf(fp, "%127s %d", buf, &dummy) != 2) {}
    if (fscanf(fp, "%127s %d", buf, &dummy) != 2) {}
    if (fscanf(fp, fmt.c_str(), buf, &cs) != 2) {}
    if (fscanf(fp, fmt.c_str(), buf, &cs) != 2) {}
    if (fscanf(fp, fmt.c_str(), buf, &cs) != 2) {}
    fclose(fp);
    return cs;
}

// input/read_raster_file.cpp:3-48 -- south-up row-major into a mesh_dim-wide array;
// -9999 (|v + 9999| < 1e-10) becomes wall_height.
template <typename T>
bool read_raster(const char* path, std::vector<T>& arr, int mesh_dim, T wall_height)
{
    FILE* fp = fopen(path, "r");
    if (!fp) return false;
    char buf[255];
    int nrows = 0, ncols = 0;
    T dummy = T(0);
    std::string fmt = std::string("%254s ") + real_fmt<T>();
    if (fscanf(fp, "%254s %d", buf, &ncols) != 2) {}
    if (fscanf(fp, "%254s %d", buf, &nrows) != 2) {}
    for (int i = 0; i < 4; ++i) if (fscanf(fp, fmt.c_str(), buf, &dummy) != 2) {}
    const char* vfmt = real_fmt<T>();
    for (int j = 0; j < nrows; ++j)
        for (int i = 0; i < ncols; ++i)
        {
            if (fscanf(fp, vfmt, &dummy) != 1) {}
            const bool nodata = std::fabs(dummy + T(9999.0)) < T(1e-10);
            const long idx = (long)(nrows - 1 - j) * mesh_dim + i;
            if (idx >= 0 && idx < (long)arr.size()) arr[idx] = nodata ? wall_height : dummy;
        }
    fclose(fp);
    return true;
}

// One time series of a .bdy file (classes/Boundary.h:427-466,
// classes/PointSources.h:300-360): "name" line, then "n units", then n rows "value time".
template <typename T>
bool read_series(const char* par, const char* name, std::vector<T>& t, std::vector<T>& v)
{
    std::string bdy = read_kw_str(par, "bdyfile");
    FILE* fp = fopen(bdy.c_str(), "r");
    if (!fp) return false;
    char line[255] = {0};
    char buf[128] = {0};
    const size_t n = strlen(name);
    while (strncmp(buf, name, n))
    {
        if (!fgets(line, sizeof(line), fp)) { fclose(fp); return false; }
        sscanf(line, "%127s", buf);
    }
    int rows = 0;
    if (!fgets(line, sizeof(line), fp)) { fclose(fp); return false; }
    sscanf(line, "%d %127s", &rows, buf);
    const int mult = !strncmp(buf, "seconds", 7) ? 1 : !strncmp(buf, "minutes", 7) ? 60 : 3600;
    if (rows <= 0) { fclose(fp); return false; }
    t.assign(rows, T(0));
    v.assign(rows, T(0));
    std::string fmt = std::string(real_fmt<T>()) + " " + real_fmt<T>();
    for (int i = 0; i < rows; ++i)
    {
        if (!fgets(line, sizeof(line), fp)) break;
        sscanf(line, fmt.c_str(), &v[i], &t[i]);
        t[i] *= mult;
    }
    fclose(fp);
    return true;
}

// classes/Boundary.h:471-500 / classes/PointSources.h:429-450 -- linear interpolation
// with a one-step row advance. Rows past the end are clamped (the reference reads past
// the series end there; inputs are padded so that this never happens).
template <typename T>
T interp_series(T now, int& row, const std::vector<T>& t, const std::vector<T>& v)
{
    const int len = (int)t.size();
    auto at = [&](const std::vector<T>& a, int i) { return a[i < len ? (i < 0 ? 0 : i) : len - 1]; };
    if ((row - 1) < len)
    {
        T t1 = at(t, row), t2 = at(t, row + 1);
        if (now > t2)
        {
            row++;
            t1 = at(t, row);
            t2 = at(t, row + 1);
        }
        T v1 = at(v, row), v2 = at(v, row + 1);
        return v1 + (v2 - v1) / (t2 - t1) * (now - t1);
    }
    return v[len - 1];
}

} // namespace oracle
