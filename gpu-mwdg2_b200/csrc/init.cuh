// Initial finest level on the device: the rasters read on the host (row-major M x M per
// field, the reader's layout) become the hierarchy's finest scale coefficients and the
// initial leaf state, in Z order.
#pragma once

#include "kernels.cuh"

namespace mw {

// a + b rounded on its own (never fused with the product that made a)
template <typename T> __device__ __forceinline__ T add_rounded(T a, T b)
{
    if constexpr (sizeof(T) == 4) return __fadd_rn(a, b);
    else return __dadd_rn(a, b);
}

// Rasters h, qx, qy, z (field f at raster + f * M * M) -> finest level (hierarchy slot fin +
// morton(x, y)) and leaf state (leaf morton(x, y), every finest cell a leaf).
// MWDG2 (input/read_and_project_modes_dg2.cu:60-78, mra/modal_projections.cu:28-88): node
// values come from the raster cells, the last node row and column of the DEM extent and of
// the mesh repeating the neighbouring cell; a cell's three modes are the average of its four
// nodes and the two nodal differences over 4 sqrt(3). HWFV1: the raster values directly
// (zorder/sort_finest_scale_coeffs_z_order.cu). Depths enter the hierarchy as eta = h + z.
// The sums and differences keep the order of the reference's projection, which fuses
// nothing, so the host restatement and this kernel give the same bits.
template <typename T, bool MW>
__global__ void __launch_bounds__(256) k_init_finest(const T* raster, int M, int xsz, int ysz, Hier<T> hr, Leaves<T> lf,
                                                     int fin)
{
    const int64_t F = (int64_t)M * M;
    const int ID = M + 1, ix = xsz + 1, iy = ysz + 1;
    // node (x, y) of the reference's node array
    auto node = [&](const T* r, int x, int y) -> T {
        const int i = (x == ix - 1 || x == ID - 1) ? x - 1 : x;
        const int j = (y == iy - 1 || y == ID - 1) ? y - 1 : y;
        return r[(int64_t)(M - 1 - j) * M + i];
    };
    const T s3x4 = T(4.0) * sqrt(T(3.0));
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < F; t += (int64_t)gridDim.x * blockDim.x)
    {
        const int X = (int)(t % M), Y = (int)(t / M);
        const int zi = morton(X, Y);
        T v[4][3];   // [field h, qx, qy, z][mode]
#pragma unroll
        for (int f = 0; f < 4; ++f)
        {
            const T* r = raster + f * F;
            if (MW)
            {
                // the projection's SW, SE, NW, NE entries of the node array (rows from the north)
                const T sw = node(r, X, ID - 1 - Y), se = node(r, X + 1, ID - 1 - Y);
                const T nw = node(r, X, ID - 2 - Y), ne = node(r, X + 1, ID - 2 - Y);
                v[f][0] = T(0.25) * (nw + ne + se + sw);
                v[f][1] = (ne - nw + se - sw) / s3x4;
                v[f][2] = (ne - se + nw - sw) / s3x4;
            }
            else
            {
                v[f][0] = r[t];
                v[f][1] = v[f][2] = T(0.0);
            }
        }
#pragma unroll
        for (int m = 0; m < (MW ? 3 : 1); ++m)
        {
            hr.s[0][m][fin + zi] = add_rounded(v[0][m], v[3][m]);
            hr.s[1][m][fin + zi] = v[1][m];
            hr.s[2][m][fin + zi] = v[2][m];
            hr.s[3][m][fin + zi] = v[3][m];
            lf.un[0 + m][zi] = v[0][m];
            lf.un[3 + m][zi] = v[1][m];
            lf.un[6 + m][zi] = v[2][m];
        }
    }
}

// Initial point-source insertion into the leaf depths (mra/insert_point_srcs.cu:3-29), which
// only the first step's maxima see; one thread, in source order. The HFIX/HVAR branch takes
// the bed of the finest slot whose Z index equals the source's position in the list, as the
// reference does.
template <typename T>
__global__ void k_init_point_srcs(Leaves<T> lf, Hier<T> hr, const Src<T>* src, int n, T dt0, T dx, int fin)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < n; ++i)
    {
        const int t = src[i].type;
        if (t == HFIX || t == HVAR) lf.un[0][src[i].code] = src[i].value - hr.s[3][0][fin + i];
        else if (t == QFIX || t == QVAR) lf.un[0][src[i].code] += src[i].value * dt0 / dx;
    }
}

} // namespace mw
