// Numerical kernels of the adaptive MWDG2/HWFV1 step, shared by all CUDA kernels.
//
// Every formula keeps the operand order and parenthesisation of the reference
// (al0vya/gpu-mwdg2) so that nvcc forms the same fused multiply-adds and results agree
// bit for bit with the reference's own CUDA build. Citations give the reference file.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mw {

#define MW_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------- enums
enum Solver : int { HWFV1 = 1, MWDG2 = 2 };            // types/SolverTypes.h
enum Inlet : int { CLOSED = 1, FREE = 2, HFIX = 4, HVAR = 8, QFIX = 16, QVAR = 32 };  // types/InletTypes.h

// Flag byte per parent slot of the hierarchy.
enum : uint8_t {
    F_SIG = 1,   // significant: the node is refined (its children exist in the tree)
    F_ENC = 2,   // details of this node were computed by this step's encode
    F_PRE = 4,   // preflagged: always significant once encoded (mra/preflag_*.cu)
    F_XS = 8     // encoded this step with details reaching the extra-significance threshold
                 // (mra/extra_significance_kernel.cu): a significant parent with F_XS makes
                 // its four children significant
};

// ---------------------------------------------------------------- indexing
// utilities/get_lvl_idx.cuh:11-24 -- first slot of level n (3 padding slots)
// (level <= 15: the library allows max_ref_lvl <= 14 and indexes levels up to L + 1)
MW_HD int lvl_idx(int level) { return ((1 << (2 * level)) - 1) / 3 + 3; }

// Level of a hierarchy index h >= 3 (inverse of lvl_idx): 3 (h - 3) + 1 lies in
// [4^l, 4^(l+1)), so l is half the position of its highest set bit (32 bits hold it for
// l <= 15).
MW_HD int level_of(int h)
{
    const unsigned v = 3u * (unsigned)(h - 3) + 1u;
#ifdef __CUDA_ARCH__
    return (31 - __clz((int)v)) >> 1;
#else
    return (31 - __builtin_clz(v)) >> 1;
#endif
}

// zorder/dilate.cuh:25-41, zorder/compact.cuh:9-21, zorder/generate_morton_code.cuh:7-16
MW_HD int dilate(int c)
{
    c &= 0x0000ffff;
    c = (c ^ (c << 8)) & 0x00ff00ff;
    c = (c ^ (c << 4)) & 0x0f0f0f0f;
    c = (c ^ (c << 2)) & 0x33333333;
    c = (c ^ (c << 1)) & 0x55555555;
    return c;
}
MW_HD int compact(int code)
{
    int c = code & 0x55555555;
    c = (c ^ (c >> 1)) & 0x33333333;
    c = (c ^ (c >> 2)) & 0x0f0f0f0f;
    c = (c ^ (c >> 4)) & 0x00ff00ff;
    c = (c ^ (c >> 8)) & 0x0000ffff;
    return c;
}
MW_HD int morton(int x, int y) { return dilate(x) | (dilate(y) << 1); }

// ---------------------------------------------------------------- filters
// Multiwavelet (DG2 basis) two-scale filters. tab[f][r][m]: filter f (f -> child
// {0, 2, 1, 3}), output row r, input mode m (0, 1x, 1y). These numbers must equal the
// reference's (mra/Filters.h:202-397) for bit-exact trees.
struct Filt
{
    static constexpr double H[4][3][3] = {
        {{0.5, 0.0, 0.0}, {-0.4330127018922193, 0.25, 0.0}, {-0.4330127018922193, 0.0, 0.25}},
        {{0.5, 0.0, 0.0}, {-0.4330127018922193, 0.25, 0.0}, {0.4330127018922193, 0.0, 0.25}},
        {{0.5, 0.0, 0.0}, {0.4330127018922193, 0.25, 0.0}, {-0.4330127018922193, 0.0, 0.25}},
        {{0.5, 0.0, 0.0}, {0.4330127018922193, 0.25, 0.0}, {0.4330127018922193, 0.0, 0.25}}};
    static constexpr double GA[4][3][3] = {
        {{-0.2672612419124244, -0.4629100498862757, -0.4629100498862757}, {0.0, 0.0, -0.7071067811865476}, {0.0, -0.7071067811865476, 0.0}},
        {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
        {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
        {{0.2672612419124244, -0.4629100498862757, -0.4629100498862757}, {0.0, 0.0, 0.7071067811865476}, {0.0, 0.7071067811865476, 0.0}}};
    static constexpr double GB[4][3][3] = {
        {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
        {{-0.2672612419124244, -0.4629100498862757, 0.46291004988627577}, {0.0, 0.0, -0.7071067811865476}, {0.0, -0.7071067811865476, 0.0}},
        {{0.2672612419124244, -0.4629100498862757, 0.46291004988627577}, {0.0, 0.0, 0.7071067811865476}, {0.0, 0.7071067811865476, 0.0}},
        {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}}};
    static constexpr double GC[4][3][3] = {
        {{0.5, 0.0, 0.0}, {-0.1636634176769942, -0.2834733547569204, 0.37796447300922725}, {-0.1636634176769942, 0.37796447300922725, -0.2834733547569204}},
        {{-0.5, 0.0, 0.0}, {-0.1636634176769942, -0.2834733547569204, -0.3779644730092272}, {0.16366341767699427, -0.3779644730092272, -0.2834733547569204}},
        {{-0.5, 0.0, 0.0}, {0.16366341767699427, -0.2834733547569204, -0.3779644730092272}, {-0.1636634176769942, -0.3779644730092272, -0.2834733547569204}},
        {{0.5, 0.0, 0.0}, {0.16366341767699427, -0.2834733547569204, 0.37796447300922725}, {0.16366341767699427, 0.37796447300922725, -0.2834733547569204}}};
    // Haar pair (FV1)
    static constexpr double h0 = 0.7071067811865475, h1 = 0.7071067811865475;
    static constexpr double g0 = 0.7071067811865475, g1 = -0.7071067811865475;
};

// Compile-time filter tap as an immediate of type T.
template <typename T, int Tab, int f, int r, int m> MW_HD constexpr T tap()
{
    constexpr double v = (Tab == 0) ? Filt::H[f][r][m] : (Tab == 1) ? Filt::GA[f][r][m]
                       : (Tab == 2) ? Filt::GB[f][r][m] : Filt::GC[f][r][m];
    return static_cast<T>(v);
}

// One 12-tap row of the analysis filter, summed in the reference's order
// (mra/encode_scale.cuh:13-38, mra/encode_details.cuh:65-188): filter 0 on child 0,
// filter 1 on child 2, filter 2 on child 1, filter 3 on child 3; modes 0, 1x, 1y.
// c[m][k]: mode m of child k (Morton order).
template <typename T, int Tab, int r> MW_HD T analyse(const T (&c)[3][4])
{
    return (tap<T, Tab, 0, r, 0>() * c[0][0] + tap<T, Tab, 0, r, 1>() * c[1][0] + tap<T, Tab, 0, r, 2>() * c[2][0] +
            tap<T, Tab, 1, r, 0>() * c[0][2] + tap<T, Tab, 1, r, 1>() * c[1][2] + tap<T, Tab, 1, r, 2>() * c[2][2] +
            tap<T, Tab, 2, r, 0>() * c[0][1] + tap<T, Tab, 2, r, 1>() * c[1][1] + tap<T, Tab, 2, r, 2>() * c[2][1] +
            tap<T, Tab, 3, r, 0>() * c[0][3] + tap<T, Tab, 3, r, 1>() * c[1][3] + tap<T, Tab, 3, r, 2>() * c[2][3]) / T(2.0);
}

// Synthesis of mode k of the child that filter f maps to, from the parent's scale modes
// s[3] and details a/b/g[3] (mra/decode_scale_children.cuh:81-395).
template <typename T, int f, int k>
MW_HD T synthesise(const T (&s)[3], const T (&a)[3], const T (&b)[3], const T (&g)[3])
{
    return (tap<T, 0, f, 0, k>() * s[0] + tap<T, 0, f, 1, k>() * s[1] + tap<T, 0, f, 2, k>() * s[2] +
            tap<T, 1, f, 0, k>() * a[0] + tap<T, 1, f, 1, k>() * a[1] + tap<T, 1, f, 2, k>() * a[2] +
            tap<T, 2, f, 0, k>() * b[0] + tap<T, 2, f, 1, k>() * b[1] + tap<T, 2, f, 2, k>() * b[2] +
            tap<T, 3, f, 0, k>() * g[0] + tap<T, 3, f, 1, k>() * g[1] + tap<T, 3, f, 2, k>() * g[2]) * T(2.0);
}

// Encode one field: parent scale modes s[3] and nine details d[t][m] (t: alpha, beta,
// gamma; m: 0, 1x, 1y) from the 12 child coefficients.
template <typename T> MW_HD void mw_encode_scale(const T (&c)[3][4], T (&s)[3])
{
    s[0] = analyse<T, 0, 0>(c);
    s[1] = analyse<T, 0, 1>(c);
    s[2] = analyse<T, 0, 2>(c);
}
template <typename T> MW_HD void mw_encode_details(const T (&c)[3][4], T (&d)[3][3])
{
    d[0][0] = analyse<T, 1, 0>(c); d[1][0] = analyse<T, 2, 0>(c); d[2][0] = analyse<T, 3, 0>(c);
    d[0][1] = analyse<T, 1, 1>(c); d[1][1] = analyse<T, 2, 1>(c); d[2][1] = analyse<T, 3, 1>(c);
    d[0][2] = analyse<T, 1, 2>(c); d[1][2] = analyse<T, 2, 2>(c); d[2][2] = analyse<T, 3, 2>(c);
}

// classes/SubDetail.h:12-46 -- max |detail| over one field's nine details
template <typename T> MW_HD T mw_detail_max(const T (&d)[3][3])
{
    T m0 = fmax(fabs(d[0][0]), fabs(d[1][0])); m0 = fmax(fabs(d[2][0]), m0);
    T m1 = fmax(fabs(d[0][1]), fabs(d[1][1])); m1 = fmax(fabs(d[2][1]), m1);
    T m2 = fmax(fabs(d[0][2]), fabs(d[1][2])); m2 = fmax(fabs(d[2][2]), m2);
    T m = fmax(m0, m1);
    return fmax(m2, m);
}

// Decode one field: children c[m][k] from parent scale s and details d[t][m].
template <typename T> MW_HD void mw_decode(const T (&s)[3], const T (&d)[3][3], T (&c)[3][4])
{
    const T a[3] = {d[0][0], d[0][1], d[0][2]};
    const T b[3] = {d[1][0], d[1][1], d[1][2]};
    const T g[3] = {d[2][0], d[2][1], d[2][2]};
    c[0][0] = synthesise<T, 0, 0>(s, a, b, g); c[0][1] = synthesise<T, 2, 0>(s, a, b, g);
    c[0][2] = synthesise<T, 1, 0>(s, a, b, g); c[0][3] = synthesise<T, 3, 0>(s, a, b, g);
    c[1][0] = synthesise<T, 0, 1>(s, a, b, g); c[1][1] = synthesise<T, 2, 1>(s, a, b, g);
    c[1][2] = synthesise<T, 1, 1>(s, a, b, g); c[1][3] = synthesise<T, 3, 1>(s, a, b, g);
    c[2][0] = synthesise<T, 0, 2>(s, a, b, g); c[2][1] = synthesise<T, 2, 2>(s, a, b, g);
    c[2][2] = synthesise<T, 1, 2>(s, a, b, g); c[2][3] = synthesise<T, 3, 2>(s, a, b, g);
}

// Haar filters (mra/encode_scale.cuh:7-11, mra/encode_details.cuh:7-23,
// mra/decode_scale_children.cuh:38-76); children in Morton order.
template <typename T> MW_HD T hw_scale(const T (&c)[4])
{
    return T(0.5) * (T(Filt::h0) * (T(Filt::h0) * c[0] + T(Filt::h1) * c[2]) + T(Filt::h1) * (T(Filt::h0) * c[1] + T(Filt::h1) * c[3]));
}
template <typename T> MW_HD T hw_alpha(const T (&c)[4])
{
    return T(0.5) * (T(Filt::h0) * (T(Filt::g0) * c[0] + T(Filt::g1) * c[2]) + T(Filt::h1) * (T(Filt::g0) * c[1] + T(Filt::g1) * c[3]));
}
template <typename T> MW_HD T hw_beta(const T (&c)[4])
{
    return T(0.5) * (T(Filt::g0) * (T(Filt::h0) * c[0] + T(Filt::h1) * c[2]) + T(Filt::g1) * (T(Filt::h0) * c[1] + T(Filt::h1) * c[3]));
}
template <typename T> MW_HD T hw_gamma(const T (&c)[4])
{
    return T(0.5) * (T(Filt::g0) * (T(Filt::g0) * c[0] + T(Filt::g1) * c[2]) + T(Filt::g1) * (T(Filt::g0) * c[1] + T(Filt::g1) * c[3]));
}
template <typename T> MW_HD void hw_decode(T u, T a, T b, T g, T (&c)[4])
{
    const T h0 = T(Filt::h0), h1 = T(Filt::h1), g0 = T(Filt::g0), g1 = T(Filt::g1);
    c[0] = (h0 * (h0 * u + g0 * a) + g0 * (h0 * b + g0 * g)) * T(2.0);
    c[1] = (h1 * (h0 * u + g0 * a) + g1 * (h0 * b + g0 * g)) * T(2.0);
    c[2] = (h0 * (h1 * u + g1 * a) + g0 * (h1 * b + g1 * g)) * T(2.0);
    c[3] = (h1 * (h1 * u + g1 * a) + g1 * (h1 * b + g1 * g)) * T(2.0);
}

// ---------------------------------------------------------------- flow algebra
template <typename T> struct V3 { T h, qx, qy; };            // classes/FlowVector.h
template <typename T> struct P3 { T _0, _1x, _1y; };          // classes/PlanarCoefficients.h

template <typename T> MW_HD V3<T> operator+(const V3<T>& a, const V3<T>& b) { return {a.h + b.h, a.qx + b.qx, a.qy + b.qy}; }
template <typename T> MW_HD V3<T> operator-(const V3<T>& a, const V3<T>& b) { return {a.h - b.h, a.qx - b.qx, a.qy - b.qy}; }
template <typename T> MW_HD V3<T> operator*(T s, const V3<T>& a) { return {s * a.h, s * a.qx, s * a.qy}; }
template <typename T> MW_HD V3<T> operator/(const V3<T>& a, T s) { return {a.h / s, a.qx / s, a.qy / s}; }

// operators/eval_loc_face_val_dg2.cuh:7-15
template <typename T> MW_HD T face(const P3<T>& s, const P3<T>& b) { return s._0 * b._0 + s._1x * b._1x + s._1y * b._1y; }

// classes/FlowVector.h:13-48 (get_speed, calc_h_star, get_star)
template <typename T> MW_HD V3<T> star(const V3<T>& U, T z, T z_inter, T tol_h)
{
    const T eta = U.h + z;
    const T h_star = fmax(T(0.0), eta - z_inter);
    const T qx_star = h_star * ((U.h < tol_h) ? T(0) : U.qx / U.h);
    const T qy_star = h_star * ((U.h < tol_h) ? T(0) : U.qy / U.h);
    return {h_star, qx_star, qy_star};
}

// classes/FlowVector.h:50-81
template <typename T> MW_HD V3<T> phys_flux_x(const V3<T>& U, T tol_h, T g)
{
    if (U.h < tol_h) return {T(0), T(0), T(0)};
    return {U.qx, U.qx * U.qx / U.h + g * U.h * U.h / T(2.0), U.qx * U.qy / U.h};
}
template <typename T> MW_HD V3<T> phys_flux_y(const V3<T>& U, T tol_h, T g)
{
    if (U.h < tol_h) return {T(0), T(0), T(0)};
    return {U.qy, U.qx * U.qy / U.h, U.qy * U.qy / U.h + g * U.h * U.h / T(2.0)};
}

// operators/flux_HLL.cuh:9-111
template <typename T> MW_HD V3<T> flux_hll_x(const V3<T>& Un, const V3<T>& Up, T tol_h, T g)
{
    if (Un.h < tol_h && Up.h < tol_h) return {T(0), T(0), T(0)};
    const T h_neg = (Un.h < tol_h) ? T(0.0) : Un.h;
    const T u_neg = (Un.h < tol_h) ? T(0.0) : Un.qx / Un.h;
    const T v_neg = (Un.h < tol_h) ? T(0.0) : Un.qy / Un.h;
    const T h_pos = (Up.h < tol_h) ? T(0.0) : Up.h;
    const T u_pos = (Up.h < tol_h) ? T(0.0) : Up.qx / Up.h;
    const T v_pos = (Up.h < tol_h) ? T(0.0) : Up.qy / Up.h;
    const T a_neg = sqrt(g * h_neg);
    const T a_pos = sqrt(g * h_pos);
    const T h_star = (T(0.5) * (a_neg + a_pos) + T(0.25) * (u_neg - u_pos)) *
                     (T(0.5) * (a_neg + a_pos) + T(0.25) * (u_neg - u_pos)) / g;
    const T u_star = T(0.5) * (u_neg + u_pos) + a_neg - a_pos;
    const T a_star = sqrt(g * h_star);
    const T s_neg = (h_neg < tol_h) ? u_pos - T(2.0) * a_pos : fmin(u_neg - a_neg, u_star - a_star);
    const T s_pos = (h_pos < tol_h) ? u_neg + T(2.0) * a_neg : fmax(u_pos + a_pos, u_star + a_star);
    const V3<T> F_neg = {Un.qx, u_neg * Un.qx + T(0.5) * g * h_neg * h_neg, Un.qy * u_neg};
    const V3<T> F_pos = {Up.qx, u_pos * Up.qx + T(0.5) * g * h_pos * h_pos, Up.qy * u_pos};
    if (s_neg >= T(0.0)) return F_neg;
    if (s_neg < T(0.0) && s_pos >= T(0.0))
    {
        V3<T> F;
        F.h = (s_pos * F_neg.h - s_neg * F_pos.h + s_neg * s_pos * (h_pos - h_neg)) / (s_pos - s_neg);
        F.qx = (s_pos * F_neg.qx - s_neg * F_pos.qx + s_neg * s_pos * (Up.qx - Un.qx)) / (s_pos - s_neg);
        const T s_mid = (s_neg * h_pos * (u_pos - s_pos) - s_pos * h_neg * (u_neg - s_neg)) /
                        (h_pos * (u_pos - s_pos) - h_neg * (u_neg - s_neg));
        F.qy = (s_neg < T(0.0) && s_mid >= T(0.0)) ? F.h * v_neg : F.h * v_pos;
        return F;
    }
    return F_pos;
}
template <typename T> MW_HD V3<T> flux_hll_y(const V3<T>& Un, const V3<T>& Up, T tol_h, T g)
{
    const V3<T> rn = {Un.h, Un.qy, -Un.qx};
    const V3<T> rp = {Up.h, Up.qy, -Up.qx};
    const V3<T> Fr = flux_hll_x(rn, rp, tol_h, g);
    return {Fr.h, -Fr.qy, Fr.qx};
}

// operators/apply_friction.cuh:7-53 (implicit Manning friction on one point value)
template <typename T> MW_HD void apply_friction(T h, T tol_h, T tol_s, T& qx, T& qy, T n, T g, T dt)
{
    if (h < tol_h) { qx = T(0.0); qy = T(0.0); return; }
    const T ux = qx / h;
    const T uy = qy / h;
    if (fabs(ux) < tol_s && fabs(uy) < tol_s) { qx = T(0.0); qy = T(0.0); return; }
    const T Cf = g * n * n / pow(h, T(1.0) / T(3.0));
    const T speed = sqrt(ux * ux + uy * uy);
    const T Sf_x = -Cf * ux * speed;
    const T Sf_y = -Cf * uy * speed;
    const T D_x = T(1.0) + dt * Cf / h * (T(2.0) * ux * ux + uy * uy) / speed;
    const T D_y = T(1.0) + dt * Cf / h * (T(2.0) * uy * uy + ux * ux) / speed;
    qx += dt * Sf_x / D_x;
    qy += dt * Sf_y / D_y;
}

// operators/minmod.cuh:7-24
template <typename T> MW_HD T minmod(T a, T b, T c)
{
    if ((a * b > T(0.0)) && (a * c > T(0.0)))
    {
        const T sign_a = (a > T(0.0)) - (a < T(0.0));
        return fmin(fabs(a), fmin(fabs(b), fabs(c))) * sign_a;
    }
    return T(0.0);
}

// zorder/get_x_coord.cuh, get_y_coord.cuh, get_spatial_coord.cuh (cell centre)
template <typename T> MW_HD T cell_centre(int i, T d_loc) { return i * d_loc + d_loc / T(2.0); }

// Direction codes of types/Directions.h
enum Dir : int { NORTH = 1, EAST = 2, SOUTH = 4, WEST = 8 };

// operators/get_leg_basis.cuh:12-40 with get_{x,y}_face_{coord,unit}.cuh.
// (x, y): centre of the local cell; (xn, yn, dn): centre and size of the neighbour
// (unused when nb_is_border).
template <typename T, int DIR>
MW_HD P3<T> leg_basis(bool nb_is_border, T x, T y, T dx_loc, T dy_loc, T xn, T yn, T dxn, T dyn)
{
    T x_face, y_face;
    if (DIR == NORTH) { x_face = x - dx_loc / T(2.0) + T(0.5) * dx_loc; y_face = y - dy_loc / T(2.0) + T(1.0) * dy_loc; }
    else if (DIR == SOUTH) { x_face = x - dx_loc / T(2.0) + T(0.5) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.0) * dy_loc; }
    else if (DIR == EAST) { x_face = x - dx_loc / T(2.0) + T(1.0) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.5) * dy_loc; }
    else { x_face = x - dx_loc / T(2.0) + T(0.0) * dx_loc; y_face = y - dy_loc / T(2.0) + T(0.5) * dy_loc; }
    T xu, yu;
    if (nb_is_border)
    {
        xu = (DIR == NORTH || DIR == SOUTH) ? T(0.5) : (DIR == EAST) ? T(0.0) : T(1.0);
        yu = (DIR == EAST || DIR == WEST) ? T(0.5) : (DIR == NORTH) ? T(0.0) : T(1.0);
    }
    else
    {
        xu = (x_face - (xn - dxn / T(2.0))) / dxn;
        yu = (y_face - (yn - dyn / T(2.0))) / dyn;
    }
    return {T(1.0), sqrt(T(3.0)) * (T(2.0) * xu - T(1.0)), sqrt(T(3.0)) * (T(2.0) * yu - T(1.0))};
}

} // namespace mw
