// Kernels behind the saveint outputs (run_simulation.cu:656-703): raster maps of the
// solution on the finest grid. The text itself is written on the host.
#pragma once

#include "kernels.cuh"

namespace mw {

// Explicitly rounded arithmetic: the reference evaluates its raster maps on the host,
// where no multiply-add is fused, so every product and sum is rounded on its own.
template <typename T> struct Rn;
template <> struct Rn<double>
{
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <> struct Rn<float>
{
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};

// Raster fields, one row of nx * ny values each (x fastest, y from the south edge).
enum RasterField { R_ETA = 0, R_H, R_Z, R_QX, R_QY, R_VX, R_VY, R_COUNT };

// Index of the leaf holding finest cell `code`: the last leaf (Z order) whose first finest
// cell is at or before it.
template <typename T> __device__ __forceinline__ int leaf_of_cell(const Leaves<T>& lf, int n, int L, int code)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        const int l = lf.lvl[mid];
        const int start = (lf.act[mid] - lvl_idx(l)) << (2 * (L - l));
        if (start <= code) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Every cell of the nx x ny DEM gets its leaf's solution at the cell centre
// (output/write_all_raster_maps_dg2.cu:59-131: the leaf's planar DG2 modes evaluated with
// the Legendre basis at the cell's local coordinates; output/write_all_raster_maps_fv1.cu:
// the leaf's average). `fields` selects rows of `out` (bit k: RasterField k).
template <typename T, bool MW>
__global__ void __launch_bounds__(256) k_raster(Leaves<T> lf, Hier<T> hr, const Scalars<T>* sc, int L, int nx, int ny,
                                                T tol_h, unsigned fields, T* out)
{
    using R = Rn<T>;
    const int n = sc->n_leaves;
    const int64_t total = (int64_t)nx * ny;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(t % nx), j = (int)(t / nx);
        const int e = leaf_of_cell(lf, n, L, morton(i, j));
        const int a = lf.act[e];
        const int sh = L - lf.lvl[e];
        T h, z, qx, qy;
        if (MW)
        {
            // local coordinates of the cell centre in the leaf: exact binary fractions
            const T du = T(1.0) / T(1 << sh);
            const T xu = R::add(R::mul(T(i - ((i >> sh) << sh)), du), du / T(2.0));
            const T yu = R::add(R::mul(T(j - ((j >> sh) << sh)), du), du / T(2.0));
            const T s3 = sqrt(T(3.0));
            const T b1 = R::mul(s3, R::sub(R::mul(T(2.0), xu), T(1.0)));
            const T b2 = R::mul(s3, R::sub(R::mul(T(2.0), yu), T(1.0)));
            // operators/eval_loc_face_val_dg2.cuh: s0 * 1 + s1x * b1 + s1y * b2, left to right
            auto ev = [&](T c0, T c1, T c2) { return R::add(R::add(R::mul(c0, T(1.0)), R::mul(c1, b1)), R::mul(c2, b2)); };
            h = ev(lf.un[0][e], lf.un[1][e], lf.un[2][e]);
            qx = ev(lf.un[3][e], lf.un[4][e], lf.un[5][e]);
            qy = ev(lf.un[6][e], lf.un[7][e], lf.un[8][e]);
            z = ev(hr.s[3][0][a], hr.s[3][1][a], hr.s[3][2][a]);
        }
        else
        {
            h = lf.un[0][e];
            qx = lf.un[3][e];
            qy = lf.un[6][e];
            z = hr.s[3][0][a];
        }
        const size_t N = (size_t)total;
        if (fields & (1u << R_ETA)) out[R_ETA * N + t] = R::add(h, z);
        if (fields & (1u << R_H)) out[R_H * N + t] = h;
        if (fields & (1u << R_Z)) out[R_Z * N + t] = z;
        if (fields & (1u << R_QX)) out[R_QX * N + t] = qx;
        if (fields & (1u << R_QY)) out[R_QY * N + t] = qy;
        if (fields & (1u << R_VX)) out[R_VX * N + t] = (h > tol_h) ? R::div(qx, h) : T(0.0);
        if (fields & (1u << R_VY)) out[R_VY * N + t] = (h > tol_h) ? R::div(qy, h) : T(0.0);
    }
}

} // namespace mw
