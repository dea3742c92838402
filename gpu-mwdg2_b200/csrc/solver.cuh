// Per-leaf solver kernels: one thread per leaf, grid-stride over the device-side leaf
// count. Each kernel gathers the leaf and its four neighbours straight from the
// hierarchy and keeps all per-neighbour work in registers, replacing the reference's
// sequence load_soln_and_nghbr_coeffs -> add_ghost_cells -> friction_implicit ->
// copy_to_buf_assem_sol -> limit_slopes -> dg2_update (or fv1_update) -> get_dt_CFL
// and its five materialised neighbour copies.
#pragma once

#include "kernels.cuh"

namespace mw {

template <typename T> struct Cell { T h[3], qx[3], qy[3], z[3]; };

// neighbours/load_soln_and_nghbr_coeffs.cu:3-104 (h = eta - z)
template <typename T, bool MW> __device__ __forceinline__ void load_cell(const Hier<T>& hr, int a, Cell<T>& c)
{
#pragma unroll
    for (int m = 0; m < (MW ? 3 : 1); ++m)
    {
        c.z[m] = hr.s[3][m][a];
        c.h[m] = hr.s[0][m][a] - c.z[m];
        c.qx[m] = hr.s[1][m][a];
        c.qy[m] = hr.s[2][m][a];
    }
    if (!MW)
    {
        c.h[1] = c.h[2] = c.qx[1] = c.qx[2] = c.qy[1] = c.qy[2] = c.z[1] = c.z[2] = T(0.0);
    }
}

// Non-reflecting wave maker of the Monai valley benchmark (operators/non_reflective_wave.cuh:
// 15-94): the characteristic reaching the boundary cell is traced back over one step by
// Newton's method (at most 101 iterations); the outgoing invariant there and the incoming
// one set by the target level h_inlet (still water 0.13535 m) give the boundary depth and
// velocity. The arithmetic follows the reference term by term, so both builds agree.
template <typename T>
__device__ __forceinline__ void monai_inflow(T h_inlet, T dt, T dxl, T hp, T up, T hb, T ub, T g, T& h_out, T& u_out)
{
    const T tol = T(1e-6), xa = -dxl / T(2.0);
    T p0 = dxl / T(2.0), p1 = p0 - dxl / T(2.0), dp = T(0.0), f1 = T(0.0);
    T f0 = (p0 - xa) + dt * ((ub - (p0 - xa) / dxl * (ub - up)) - sqrt(g * (hb - (p0 - xa) / dxl * (hb - hp))));
    int cond = 0;
    for (int k = 0; k <= 100 && cond == 0; ++k)
    {
        const T df = T(1.0) + dt * ((up - ub) / dxl - T(0.5) * pow((g * (hb - (p0 - xa) / dxl * (hb - hp))), T(-0.5)) *
                                                         (g * (hp - hb) / dxl));
        if (fabs(df) <= T(0.0))
        {
            cond = 1;   // zero slope: keep the current point
            dp = p1 - p0;
            p1 = p0;
        }
        else
        {
            dp = f0 / df;
            p1 = p0 - dp;
        }
        f1 = (p1 - xa) + dt * ((ub - (p1 - xa) / dxl * (ub - up)) - sqrt(g * (hb - (p1 - xa) / dxl * (hb - hp))));
        const T relerr = fabs(dp) / (fabs(p1) + T(0.0));
        if (relerr < tol) cond = 2;
        if (fabs(f1) < tol) cond = 3;
        if (relerr <= tol && fabs(f1) < tol) cond = 4;
        p0 = p1;
        f0 = f1;
    }
    const T hr = hb - (hb - hp) * (p1 - xa) / dxl;
    const T ur = ub - (ub - up) * (p1 - xa) / dxl;
    const T cr = sqrt(g * hr);
    const T beta_minus = ur - T(2.0) * cr;
    const T beta_plus = T(2.0) * sqrt(g * (h_inlet + T(0.13535))) + h_inlet * sqrt(g / T(0.13535));
    h_out = T(1.0) / T(16.0) / g * (beta_plus - beta_minus) * (beta_plus - beta_minus);
    u_out = T(0.5) * (beta_plus + beta_minus);
}

// Ghost cells of a leaf at the domain border, raster cases
// (neighbours/add_ghost_cells.cu:18-500): directions N, E, S, W in order; a fine
// boundary cell of an HFIX/HVAR/QFIX/QVAR segment also resets the leaf's own depth.
// gh/gq*: mode-0 values of the ghost in direction d (slopes are zero, bed = own bed).
template <typename T>
__device__ __forceinline__ void ghost_pass(T& own_h0, T own_qx0, T own_qy0, T own_z0, const int32_t (&nid)[4], int level,
                                           int act, const Params<T>& P, const Bnd<T>& B, T dt, T (&gh)[4], T (&gqx)[4],
                                           T (&gqy)[4])
{
    const int code = act - lvl_idx(level);
    const int x = compact(code), y = compact(code >> 1);
    const bool finest = (level == P.L);
#pragma unroll
    for (int d = 0; d < 4; ++d)
    {
        if (nid[d] != -1) continue;
        gh[d] = own_h0;
        gqx[d] = (d == 1 || d == 3) ? T(0.0) : own_qx0;
        gqy[d] = (d == 0 || d == 2) ? T(0.0) : own_qy0;
        const int c = (d == 0 || d == 2) ? x : y;
        const bool bound = (c >= B.start[d] && c <= B.end[d]);
        const bool border = (d == 0) ? (y == P.ysz - 1) : (d == 1) ? (x == P.xsz - 1) : (d == 2) ? (y == 0) : (x == 0);
        if (!(finest && bound && border)) continue;
        const int t = B.type[d];
        if (t == FREE)
        {
            const T q = (d == 0 || d == 2) ? own_qy0 : own_qx0;
            gh[d] = pow((q * q) / P.g, T(1.0) / T(3.0));
            gqx[d] = own_qx0;
            gqy[d] = own_qy0;
        }
        else if ((t == HFIX || t == HVAR) && d == 3 && B.west_special == 1)
        {
            // monai: the ghost carries the wave maker's state, the leaf keeps its own
            const T up = (own_h0 > P.tol_h) ? own_qx0 / own_h0 : T(0.0);
            T hb, ub;
            monai_inflow(B.inlet[d], dt, P.dx, own_h0, up, T(0.13535), T(0.0), P.g, hb, ub);
            gh[d] = hb - own_z0;
            gqx[d] = hb * ub;
        }
        else if ((t == HFIX || t == HVAR) && d == 3 && B.west_special == 2)
        {
            // oregon-seaside: wave-maker speed s(t), the ghost reflects the leaf's velocity about 2s
            gh[d] = own_h0;
            const T s = T(0.6) * exp(-T(0.25) * (B.time - T(14.75)) * (B.time - T(14.75)));
            const T v0 = (own_h0 > P.tol_h) ? own_qx0 / own_h0 : T(0.0);
            gqx[d] = ((T(2.0) * s - v0) * gh[d]);
        }
        else if (t == HFIX || t == HVAR)
        {
            own_h0 = B.inlet[d] - own_z0;
            gh[d] = own_h0;
        }
        else if (t == QFIX || t == QVAR)
        {
            own_h0 = B.inlet[d] * dt / P.dx;
            gh[d] = own_h0;
        }
    }
}

// operators/friction_implicit.cu:155-264 -- implicit friction on the mode-0 value and,
// for MWDG2, on the four Gauss-point values, whose differences rebuild the slopes.
// One out-of-line copy of the implicit Manning update of a point value (apply_friction);
// a stage kernel applies it at 25 points per leaf (5 points of the leaf and of each of its
// four neighbours) and would otherwise hold 25 inlined copies of its pow and divisions.
template <typename T> struct Q2 { T qx, qy; };
template <typename T> __device__ __noinline__ Q2<T> friction_point(T h, T qx, T qy, T tol_h, T tol_s, T n, T g, T dt)
{
    apply_friction(h, tol_h, tol_s, qx, qy, n, g, dt);
    return {qx, qy};
}

template <typename T, bool MW> __device__ __forceinline__ void friction_cell(Cell<T>& c, const Params<T>& P, T dt)
{
    if (!MW)
    {
        apply_friction(c.h[0], P.tol_h, P.tol_s, c.qx[0], c.qy[0], P.manning, P.g, dt);
        return;
    }
    const T hlx = c.h[0] - c.h[1], hux = c.h[0] + c.h[1];
    const T hly = c.h[0] - c.h[2], huy = c.h[0] + c.h[2];
    T qxlx = c.qx[0] - c.qx[1], qxux = c.qx[0] + c.qx[1];
    T qxly = c.qx[0] - c.qx[2], qxuy = c.qx[0] + c.qx[2];
    T qylx = c.qy[0] - c.qy[1], qyux = c.qy[0] + c.qy[1];
    T qyly = c.qy[0] - c.qy[2], qyuy = c.qy[0] + c.qy[2];
    Q2<T> r = friction_point(c.h[0], c.qx[0], c.qy[0], P.tol_h, P.tol_s, P.manning, P.g, dt);
    c.qx[0] = r.qx; c.qy[0] = r.qy;
    r = friction_point(hlx, qxlx, qylx, P.tol_h, P.tol_s, P.manning, P.g, dt);
    qxlx = r.qx; qylx = r.qy;
    r = friction_point(hux, qxux, qyux, P.tol_h, P.tol_s, P.manning, P.g, dt);
    qxux = r.qx; qyux = r.qy;
    r = friction_point(hly, qxly, qyly, P.tol_h, P.tol_s, P.manning, P.g, dt);
    qxly = r.qx; qyly = r.qy;
    r = friction_point(huy, qxuy, qyuy, P.tol_h, P.tol_s, P.manning, P.g, dt);
    qxuy = r.qx; qyuy = r.qy;
    c.qx[1] = T(0.5) * (qxux - qxlx);
    c.qx[2] = T(0.5) * (qxuy - qxly);
    c.qy[1] = T(0.5) * (qyux - qylx);
    c.qy[2] = T(0.5) * (qyuy - qyly);
}

// What the limiter and the flux of a face need from one neighbour.
template <typename T> struct NbFace
{
    T h0, eta0, qx0, qy0;   // mode-0 values
    T hf, qxf, qyf, zf;     // values at the shared face (neighbour's Legendre basis)
    T etaf;                 // face value of eta = z + h (limiter)
};

template <typename T> __device__ __forceinline__ NbFace<T> nb_face(const Cell<T>& c, const P3<T>& b)
{
    NbFace<T> r;
    r.h0 = c.h[0];
    r.qx0 = c.qx[0];
    r.qy0 = c.qy[0];
    r.eta0 = c.z[0] + c.h[0];
    r.hf = face(P3<T>{c.h[0], c.h[1], c.h[2]}, b);
    r.qxf = face(P3<T>{c.qx[0], c.qx[1], c.qx[2]}, b);
    r.qyf = face(P3<T>{c.qy[0], c.qy[1], c.qy[2]}, b);
    r.zf = face(P3<T>{c.z[0], c.z[1], c.z[2]}, b);
    r.etaf = face(P3<T>{c.z[0] + c.h[0], c.z[1] + c.h[1], c.z[2] + c.h[2]}, b);
    return r;
}

// operators/get_limited_slopes.cuh:10-78 for one field u (own planar coefficients),
// given the neighbours' face values and mode-0 values of that field.
template <typename T>
__device__ __forceinline__ void limited_slopes(const P3<T>& u, T un_pos, T ue_pos, T us_neg, T uw_neg, T un0, T ue0, T us0,
                                               T uw0, T dxf, T tolK, T& o1x, T& o1y)
{
    const T s3 = sqrt(T(3.0));
    const T u_n_neg = face(u, P3<T>{T(1.0), T(0.0), s3});
    const T u_e_neg = face(u, P3<T>{T(1.0), s3, T(0.0)});
    const T u_s_pos = face(u, P3<T>{T(1.0), T(0.0), -s3});
    const T u_w_pos = face(u, P3<T>{T(1.0), -s3, T(0.0)});
    const T jn = fabs(un_pos - u_n_neg);
    const T je = fabs(ue_pos - u_e_neg);
    const T js = fabs(u_s_pos - us_neg);
    const T jw = fabs(u_w_pos - uw_neg);
    const T norm_x = fmax(fabs(u._0 - u._1x), fabs(u._0 + u._1x));
    const T norm_y = fmax(fabs(u._0 - u._1y), fabs(u._0 + u._1y));
    const T DS_e = (norm_x > T(1e-12)) ? je / (T(0.5) * dxf * norm_x) : T(0.0);
    const T DS_w = (norm_x > T(1e-12)) ? jw / (T(0.5) * dxf * norm_x) : T(0.0);
    const T DS_n = (norm_y > T(1e-12)) ? jn / (T(0.5) * dxf * norm_y) : T(0.0);
    const T DS_s = (norm_y > T(1e-12)) ? js / (T(0.5) * dxf * norm_y) : T(0.0);
    o1x = (fmax(DS_e, DS_w) < tolK) ? u._1x : minmod(u._1x, (u._0 - uw0) / s3, (ue0 - u._0) / s3);
    o1y = (fmax(DS_n, DS_s) < tolK) ? u._1y : minmod(u._1y, (u._0 - us0), (un0 - u._0));
}

template <typename T> struct Geo { T x, y, dxl; bool in_extent; };

template <typename T> __device__ __forceinline__ Geo<T> leaf_geo(int act, int level, const Params<T>& P)
{
    Geo<T> g;
    g.dxl = P.dx * (1 << (P.L - level));
    const int code = act - lvl_idx(level);
    g.x = cell_centre(compact(code), g.dxl);
    g.y = cell_centre(compact(code >> 1), g.dxl);
    g.in_extent = !((g.x >= P.xsz * P.dx) || (g.y >= P.ysz * P.dx));
    return g;
}

// Legendre basis of the neighbour in direction D evaluated at the shared face.
template <typename T, int DIR>
__device__ __forceinline__ P3<T> nb_basis(const Geo<T>& g, int nid, int nlvl, const Params<T>& P)
{
    if (nid == -1) return leg_basis<T, DIR>(true, g.x, g.y, g.dxl, g.dxl, T(0), T(0), T(1), T(1));
    const T dn = P.dx * (1 << (P.L - nlvl));
    const int code = nid - lvl_idx(nlvl);
    const T xn = cell_centre(compact(code), dn);
    const T yn = cell_centre(compact(code >> 1), dn);
    return leg_basis<T, DIR>(false, g.x, g.y, g.dxl, g.dxl, xn, yn, dn, dn);
}

// operators/dg2_update.cu:160-334 -- the DG2 right-hand side applied to the own
// coefficients c (h, qx, qy planar; z planar) with the neighbours' face values.
template <typename T>
__device__ __forceinline__ void dg2_rhs_update(const P3<T>& ch, const P3<T>& cqx, const P3<T>& cqy, const P3<T>& zp,
                                               const NbFace<T> (&nf)[4], T dxl, const Params<T>& P, T dt, T (&out)[9])
{
    const T s3 = sqrt(T(3.0));
    const T g = P.g, tol_h = P.tol_h;
    const P3<T> bn = {T(1.0), T(0.0), s3}, be = {T(1.0), s3, T(0.0)};
    const P3<T> bs = {T(1.0), T(0.0), -s3}, bw = {T(1.0), -s3, T(0.0)};
    const T z_n_pos = nf[0].zf, z_e_pos = nf[1].zf, z_s_neg = nf[2].zf, z_w_neg = nf[3].zf;
    const T z_n_neg = face(zp, bn), z_e_neg = face(zp, be), z_s_pos = face(zp, bs), z_w_pos = face(zp, bw);
    const T zi_n = fmax(z_n_neg, z_n_pos), zi_e = fmax(z_e_neg, z_e_pos);
    const T zi_s = fmax(z_s_neg, z_s_pos), zi_w = fmax(z_w_neg, z_w_pos);
    const V3<T> Us_n_pos = star(V3<T>{nf[0].hf, nf[0].qxf, nf[0].qyf}, z_n_pos, zi_n, tol_h);
    const V3<T> Us_e_pos = star(V3<T>{nf[1].hf, nf[1].qxf, nf[1].qyf}, z_e_pos, zi_e, tol_h);
    const V3<T> Us_s_neg = star(V3<T>{nf[2].hf, nf[2].qxf, nf[2].qyf}, z_s_neg, zi_s, tol_h);
    const V3<T> Us_w_neg = star(V3<T>{nf[3].hf, nf[3].qxf, nf[3].qyf}, z_w_neg, zi_w, tol_h);
    const T hfn = face(ch, bn), hfe = face(ch, be), hfs = face(ch, bs), hfw = face(ch, bw);
    const V3<T> Us_n_neg = star(V3<T>{hfn, face(cqx, bn), face(cqy, bn)}, z_n_neg, zi_n, tol_h);
    const V3<T> Us_e_neg = star(V3<T>{hfe, face(cqx, be), face(cqy, be)}, z_e_neg, zi_e, tol_h);
    const V3<T> Us_s_pos = star(V3<T>{hfs, face(cqx, bs), face(cqy, bs)}, z_s_pos, zi_s, tol_h);
    const V3<T> Us_w_pos = star(V3<T>{hfw, face(cqx, bw), face(cqy, bw)}, z_w_pos, zi_w, tol_h);
    const V3<T> F_n = flux_hll_y(Us_n_neg, Us_n_pos, tol_h, g);
    const V3<T> F_e = flux_hll_x(Us_e_neg, Us_e_pos, tol_h, g);
    const V3<T> F_s = flux_hll_y(Us_s_neg, Us_s_pos, tol_h, g);
    const V3<T> F_w = flux_hll_x(Us_w_neg, Us_w_pos, tol_h, g);
    // x direction: modes 0 and 1x (operators/get_bed_src.cuh:46-72 for the bed slope)
    const V3<T> U0x = (Us_e_neg + Us_w_pos) / T(2.0);
    const V3<T> U1x = (Us_e_neg - Us_w_pos) / (T(2.0) * s3);
    V3<T> Lx0 = (-T(1.0) * (F_e - F_w)) / dxl;
    V3<T> Lx1 = (-s3 / dxl) * (F_e + F_w - phys_flux_x(U0x - U1x, tol_h, g) - phys_flux_x(U0x + U1x, tol_h, g));
    {
        const T eta_e_neg = hfe + z_e_neg, eta_w_pos = hfw + z_w_pos;
        const T zse = zi_e - fmax(T(0.0), -(eta_e_neg - zi_e));
        const T zsw = zi_w - fmax(T(0.0), -(eta_w_pos - zi_w));
        const T z1 = (zse - zsw) / (T(2.0) * s3);
        Lx0.qx = Lx0.qx + -T(2.0) * s3 * g * U0x.h * z1 / dxl;
        Lx1.qx = Lx1.qx + -T(2.0) * s3 * g * U1x.h * z1 / dxl;
        Lx0.h = Lx0.h + T(0.0); Lx0.qy = Lx0.qy + T(0.0);
        Lx1.h = Lx1.h + T(0.0); Lx1.qy = Lx1.qy + T(0.0);
    }
    // y direction: modes 0 and 1y
    const V3<T> U0y = (Us_n_neg + Us_s_pos) / T(2.0);
    const V3<T> U1y = (Us_n_neg - Us_s_pos) / (T(2.0) * s3);
    V3<T> Ly0 = (-T(1.0) * (F_n - F_s)) / dxl;
    V3<T> Ly1 = (-s3 / dxl) * (F_s + F_n - phys_flux_y(U0y - U1y, tol_h, g) - phys_flux_y(U0y + U1y, tol_h, g));
    {
        const T eta_n_neg = hfn + z_n_neg, eta_s_pos = hfs + z_s_pos;
        const T zsn = zi_n - fmax(T(0.0), -(eta_n_neg - zi_n));
        const T zss = zi_s - fmax(T(0.0), -(eta_s_pos - zi_s));
        const T z1 = (zsn - zss) / (T(2.0) * s3);
        Ly0.qy = Ly0.qy + -T(2.0) * s3 * g * U0y.h * z1 / dxl;
        Ly1.qy = Ly1.qy + -T(2.0) * s3 * g * U1y.h * z1 / dxl;
        Ly0.h = Ly0.h + T(0.0); Ly0.qx = Ly0.qx + T(0.0);
        Ly1.h = Ly1.h + T(0.0); Ly1.qx = Ly1.qx + T(0.0);
    }
    // coeffs += dt * (Lx + Ly): Lx has modes (0, 1x, 0), Ly has (0, 0, 1y)
    const T zero = T(0.0);
    out[0] = ch._0 + dt * (Lx0.h + Ly0.h);
    out[1] = ch._1x + dt * (Lx1.h + zero);
    out[2] = ch._1y + dt * (zero + Ly1.h);
    out[3] = cqx._0 + dt * (Lx0.qx + Ly0.qx);
    out[4] = cqx._1x + dt * (Lx1.qx + zero);
    out[5] = cqx._1y + dt * (zero + Ly1.qx);
    out[6] = cqy._0 + dt * (Lx0.qy + Ly0.qy);
    out[7] = cqy._1x + dt * (Lx1.qy + zero);
    out[8] = cqy._1y + dt * (zero + Ly1.qy);
}

// Depth after ghost cells of the own leaf and its four neighbours; a leaf is dry when all
// five are below tol_h: it is not updated (dg2_update.cu:36-50), not limited (the limiter
// needs a depth above 0.05 max_h) and, being below tol_h, gets no friction, so it needs
// none of its neighbours' other coefficients.
template <typename T>
__device__ __forceinline__ bool leaf_is_dry(const Hier<T>& hr, T own_h0, const int32_t (&nid)[4], const T (&gh)[4], T tol_h)
{
    if (!(own_h0 < tol_h)) return false;
#pragma unroll
    for (int d = 0; d < 4; ++d)
    {
        const T h = (nid[d] != -1) ? hr.s[0][0][nid[d]] - hr.s[3][0][nid[d]] : gh[d];
        if (!(h < tol_h)) return false;
    }
    return true;
}

// Leaf state u (h, qx, qy by mode, the layout of Leaves::un) into the hierarchy at `a`,
// depths as surface elevations eta = h + z (mra/reinsert_assem_sol.cu:3-32).
template <typename T>
__device__ __forceinline__ void put_leaf(const Hier<T>& hr, int a, const T (&u)[9], const T (&z)[3], uint32_t mark = 0)
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
    {
        hr.s[0][m][a] = u[m] + z[m];
        hr.s[1][m][a] = u[3 + m];
        hr.s[2][m][a] = u[6 + m];
    }
    if (hr.tag) hr.tag[a] = mark;   // the stage hierarchy of the keep-values decode
}

// Running maxima of the state at the end of a step, as the next step's
// mra/get_max_scale_coeffs.cu:3-27 reads them (|eta|, |h0|, |qx0|, |z0|; the reference
// also uses qx0 for the qy maximum).
template <typename T> struct StateMax
{
    T eta = T(0), h = T(0), qx = T(0), z = T(0);
    __device__ __forceinline__ void add(const T (&u)[9], T z0)
    {
        const T e = u[0] + z0;
        eta = fmax(eta, fabs(e));
        h = fmax(h, fabs(u[0]));
        qx = fmax(qx, fabs(u[3]));
        z = fmax(z, fabs(z0));
    }
    __device__ __forceinline__ void flush(Scalars<T>* sc)
    {
        T v[4] = {eta, h, qx, z};
        T* const dst[4] = {&sc->next_max[0], &sc->next_max[1], &sc->next_max[2], &sc->next_max[3]};
        block_max_atomic<T, 4>(v, dst);
    }
};

// The FV1 result of a leaf into the other of the two alternating hierarchy buffers at the
// leaf's own index (the re-insertion of mra/reinsert_assem_sol.cu:3-32, eta = h + z), and
// into the maxima the next step's thresholds use (mra/get_max_scale_coeffs.cu:3-27).
template <typename T>
__device__ __forceinline__ void put_leaf_fv1(const Hier<T>& hout, int a, T h, T qx, T qy, T z, StateMax<T>& mx)
{
    hout.s[0][0][a] = h + z;
    hout.s[1][0][a] = qx;
    hout.s[2][0][a] = qy;
    const T u[9] = {h, T(0), T(0), qx, T(0), T(0), qy, T(0), T(0)};
    mx.add(u, z);
}

// Wet test of one RK stage (the rule of leaf_is_dry, after ghost cells): wet leaves are
// appended to `wet` (warp-aggregated) for k_mwdg2_stage<.., LIST=true> (a NaN depth is not
// below tol_h, so a NaN leaf is listed and the stage kernel reports it), dry ones marked in
// `dry` for k_stage_dry, which then runs beside the wet-list kernel (the two touch disjoint
// leaves). Stage 1 also keeps a dry leaf's depth after ghost cells in U^n (un[0]); stage 2
// reports initial_tstep as the CFL step of dry leaves (dg2_update.cu:61).
template <typename T, int STAGE>
__device__ __forceinline__ void k_stage_wet_body(int bid, int nb, Leaves<T> lf, Hier<T> hin, Scalars<T>* sc, Params<T> P,
                                                   const StepArgs<T>* args, uint8_t* dry, int32_t* wet,
                                                   const uint8_t* dry1 = nullptr, uint32_t* clean_tag = nullptr)
{
    const T dt = args->dt;
    const Bnd<T>& B = args->B;
    const int n = sc->n_leaves;
    bool any_dry = false;
    for (int i0 = bid * blockDim.x; i0 < n; i0 += nb * blockDim.x)
    {
        const int i = i0 + threadIdx.x;
        bool is_wet = false;
        if (i < n)
        {
            const int a = lf.act[i];
            int32_t nid[4];
#pragma unroll
            for (int d = 0; d < 4; ++d) nid[d] = lf.nb[d][i];
            // own and neighbour loads issued together (almost every leaf is dry here); the
            // level and the discharges only enter the ghost cells of faces on the border
            // (ghost_pass)
            const bool border = (nid[0] == -1) | (nid[1] == -1) | (nid[2] == -1) | (nid[3] == -1);
            const int level = border ? lf.lvl[i] : 0;
            const T e0 = hin.s[0][0][a], z0 = hin.s[3][0][a];
            const T qx0 = border ? hin.s[1][0][a] : T(0.0), qy0 = border ? hin.s[2][0][a] : T(0.0);
            T nbh[4];
#pragma unroll
            for (int d = 0; d < 4; ++d)
                nbh[d] = (nid[d] != -1) ? hin.s[0][0][nid[d]] - hin.s[3][0][nid[d]] : T(0.0);
            T h0 = e0 - z0;
            T gh[4], gqx[4], gqy[4];
            ghost_pass(h0, qx0, qy0, z0, nid, level, a, P, B, dt, gh, gqx, gqy);
            bool is_dry = h0 < P.tol_h;
#pragma unroll
            for (int d = 0; d < 4; ++d) is_dry = is_dry && ((nid[d] != -1) ? nbh[d] : gh[d]) < P.tol_h;
            is_wet = !is_dry;
            any_dry |= is_dry;
            dry[i] = is_dry ? 1 : 0;
            if (STAGE == 1 && is_dry) lf.un[0][i] = h0;
            if (STAGE == 2 && clean_tag && is_dry && dry1[i]) clean_tag[a] = sc->step_tag;
        }
        // warp-aggregated append
        const unsigned mask = __ballot_sync(0xffffffffu, is_wet);
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == 0 && mask) base = atomicAdd(&sc->wet[STAGE - 1], __popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (is_wet) wet[base + __popc(mask & ((1u << lane) - 1u))] = i;
    }
    if (STAGE == 2 && __syncthreads_or(any_dry) && threadIdx.x == 0) atomic_min_nn(&sc->dt_min, P.initial_tstep);
}
template <typename T, int STAGE>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_stage_wet(Leaves<T> lf, Hier<T> hin, Scalars<T>* sc, Params<T> P,
                                                   const StepArgs<T>* args, uint8_t* dry, int32_t* wet,
                                                   const uint8_t* dry1 = nullptr, uint32_t* clean_tag = nullptr)
{
    k_stage_wet_body<T, STAGE>(blockIdx.x, gridDim.x, lf, hin, sc, P, args, dry, wet, dry1, clean_tag);
}

// The dry leaves of one RK stage, marked by k_stage_wet (bandwidth-bound; it runs beside
// the latency-bound wet-list kernel). Stage 1 (hin: hierarchy, hout: stage hierarchy): U^n
// is the leaf's state with the discharge cleared by friction (depth after ghost cells as
// k_stage_wet left it in un[0]) and U* equals it. Stage 2 (hout: hierarchy): the leaf keeps
// U^n, which is re-inserted into the hierarchy and enters the next step's maxima.
// pm (learned refinement proposal, applied steps with both stages over the wet list): a
// leaf inside a subtree the proposal left out (its subtree's encode and decode are skipped
// too) keeps its state as it stands in the hierarchy where nothing has changed it. With the
// keep-values decode, which rewrites no leaf that persists, pm leaves out every subtree but
// those holding point sources.
// Stage 1 leaves such a dry leaf's U* in the stage hierarchy as it stands when the leaf was
// a leaf dry in both stages of the last step (clean_tag[a], at its hierarchy index, is the
// last step's tag: written by that step's stage-2 wet test; null when that step did not
// record it): U* is then still the one written when the leaf last changed. Its U^n copy
// (un, by leaf position) is rewritten only where the position now holds another leaf than
// in the last step (lf.same). Stage 1 marks the leaves it freezes (dry[i] = 2); stage 2
// writes nothing for such a leaf that is dry in stage 2 as well (dry1: stage 1's marks) and
// only adds it to the maxima, so a leaf's state is re-inserted at least once after it last
// changed.
template <typename T, int STAGE>
__device__ __forceinline__ void k_stage_dry_body(int bid, int nb, Leaves<T> lf, Hier<T> hin, Hier<T> hout, Scalars<T>* sc, Params<T> P,
                                                   bool friction, uint8_t* dry, const uint8_t* dry1, PropMask pm,
                                                   const uint32_t* clean_tag = nullptr)
{
    const uint32_t last_tag = sc->step_tag - 1u;
    const uint32_t wmark = (sc->step_tag << 1) | 1u;   // a written stage-hierarchy slot (Hier::tag)
    const int n = sc->n_leaves;
    const int stride = nb * blockDim.x;
    StateMax<T> mx;
    unsigned frozen = 0;
    // software pipeline: the next leaf's mark and hierarchy index are loaded while this
    // leaf's gathers at its index are in flight (one dependent round trip per leaf, not two)
    int i = bid * blockDim.x + threadIdx.x;
    bool dry_next = i < n && dry[i];
    int a_next = i < n ? lf.act[i] : 0;
    for (; i < n; i += stride)
    {
        const bool is_dry = dry_next;
        const int a = a_next;
        if (i + stride < n)
        {
            dry_next = dry[i + stride];
            a_next = lf.act[i + stride];
        }
        if (!is_dry) continue;
        bool keep_ustar = false;
        if (pm.prop && (STAGE == 2 || clean_tag))
        {
            const int lv = lf.lvl[i];
            const bool left_out = lv >= pm.level && pm_out(pm, (a - lvl_idx(lv)) >> (2 * (lv - pm.level)));
            if (STAGE == 1 && left_out && clean_tag[a] == last_tag)
            {
                dry[i] = 2;
                ++frozen;
                if (hout.tag) hout.tag[a] = wmark & ~1u;   // U* stands
                if (lf.same[i]) continue;
                keep_ustar = true;   // un only
            }
            if (STAGE == 2 && left_out && dry1[i] == 2)
            {
                T u[9];
                u[0] = lf.un[0][i];
                u[3] = lf.un[3][i];
                mx.add(u, hin.s[3][0][a]);
                if (P.dt_leaf) P.dt_leaf[i] = P.initial_tstep;
                continue;
            }
        }
        const T z[3] = {hin.s[3][0][a], hin.s[3][1][a], hin.s[3][2][a]};
        T u[9];
        if (STAGE == 1)
        {
            u[0] = lf.un[0][i];
            u[3] = friction ? T(0.0) : hin.s[1][0][a];
            u[6] = friction ? T(0.0) : hin.s[2][0][a];
#pragma unroll
            for (int m = 1; m < 3; ++m)
            {
                u[m] = hin.s[0][m][a] - z[m];
                u[3 + m] = hin.s[1][m][a];
                u[6 + m] = hin.s[2][m][a];
            }
#pragma unroll
            for (int k = 1; k < 9; ++k) lf.un[k][i] = u[k];
            if (keep_ustar) continue;
        }
        else
        {
#pragma unroll
            for (int k = 0; k < 9; ++k) u[k] = lf.un[k][i];
            mx.add(u, z[0]);
            if (P.dt_leaf) P.dt_leaf[i] = P.initial_tstep;
        }
        put_leaf(hout, a, u, z, wmark);
    }
    if (STAGE == 2) mx.flush(sc);
    if (STAGE == 1 && pm.prop)
    {
        frozen = __reduce_add_sync(0xffffffffu, frozen);
        if ((threadIdx.x & 31) == 0 && frozen) atomicAdd(&sc->prop_frozen, frozen);
    }
}
template <typename T, int STAGE>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 5) k_stage_dry(Leaves<T> lf, Hier<T> hin, Hier<T> hout, Scalars<T>* sc, Params<T> P,
                                                   bool friction, uint8_t* dry, const uint8_t* dry1, PropMask pm,
                                                   const uint32_t* clean_tag = nullptr)
{
    k_stage_dry_body<T, STAGE>(blockIdx.x, gridDim.x, lf, hin, hout, sc, P, friction, dry, dry1, pm, clean_tag);
}

// One RK2 stage of MWDG2, reading the hierarchy `hin` and writing each leaf's result into
// the hierarchy `hout` at the leaf's own index (which no leaf reads in this stage).
// STAGE 1 (hin: hierarchy, hout: stage hierarchy): friction (once per step), limiter with
// the step's max depth, U* -> hout, U^n (after friction and limiter) -> un.
// STAGE 2 (hin: stage hierarchy, hout: hierarchy): limiter with the stage's max depth,
// U^{n+1} = (U** + U^n)/2 -> un and hout (the next step's re-insertion,
// mra/reinsert_assem_sol.cu), the next step's maxima, CFL dt. LIST: only the leaves in
// the wet list built by k_stage_wet; otherwise every leaf.
template <typename T, int STAGE, bool LIST>
__device__ __forceinline__ void k_mwdg2_stage_body(int bid, int nb, Leaves<T> lf, Hier<T> hin, Hier<T> hout, Scalars<T>* sc,
                                                                Params<T> P, const StepArgs<T>* args, bool friction,
                                                                const int32_t* wet)
{
    const T dt = args->dt;
    const Bnd<T>& B = args->B;
    const Hier<T>& hr = hin;
    StateMax<T> mx;
    const int n = LIST ? sc->wet[STAGE - 1] : sc->n_leaves;
    T dt_loc = (sizeof(T) == 8) ? T(1.0e308) : T(3.0e38);
    bool nan_seen = false;
    unsigned n_wet = 0;
    const T max_h = (STAGE == 1) ? fmax(T(1.0), sc->max_h) : sc->max_h2;
    const uint32_t wmark = (sc->step_tag << 1) | 1u;   // a written stage-hierarchy slot (Hier::tag)
    for (int k = bid * blockDim.x + threadIdx.x; k < n; k += nb * blockDim.x)
    {
        const int i = LIST ? wet[k] : k;
        const int a = lf.act[i];
        const int level = lf.lvl[i];
        int32_t nid[4];
        int nl[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) { nid[d] = lf.nb[d][i]; nl[d] = nid[d] == -1 ? level : level_of(nid[d]); }
        Cell<T> own;
        load_cell<T, true>(hr, a, own);
        // a NaN depth anywhere in the state (a dry-looking NaN leaf is never updated below)
        nan_seen |= (own.h[0] != own.h[0]);
        T gh[4], gqx[4], gqy[4];
        ghost_pass(own.h[0], own.qx[0], own.qy[0], own.z[0], nid, level, a, P, B, dt, gh, gqx, gqy);
        // Depths of the four neighbours (after ghost cells). A leaf whose own depth and
        // neighbour depths are all below tol_h is not updated (dg2_update.cu:36-50), is not
        // limited (the limiter needs a depth above 0.05 max_h) and, being below tol_h, gets
        // no friction: it needs none of the neighbours' other coefficients.
        const bool dry = !LIST && leaf_is_dry(hr, own.h[0], nid, gh, P.tol_h);
        n_wet += dry ? 0 : 1;
        // friction_implicit.cu:24-48: shallow or slow leaves lose their discharge and
        // skip friction (their neighbours' copies are then left untouched too)
        bool fric = false;
        if (STAGE == 1 && friction)
        {
            const T h = own.h[0];
            const bool below_depth = (h < P.tol_h);
            const T ux = below_depth ? T(0.0) : own.qx[0] / h;
            const T uy = below_depth ? T(0.0) : own.qy[0] / h;
            const bool below_speed = (fabs(ux) < P.tol_s && fabs(uy) < P.tol_s);
            if (below_depth || below_speed) { own.qx[0] = T(0.0); own.qy[0] = T(0.0); }
            fric = !(below_depth || below_speed);
            if (fric) friction_cell<T, true>(own, P, dt);
        }
        if (dry)
        {
            T u[9];
            if (STAGE == 1)
            {
#pragma unroll
                for (int m = 0; m < 3; ++m) { u[m] = own.h[m]; u[3 + m] = own.qx[m]; u[6 + m] = own.qy[m]; }
#pragma unroll
                for (int k = 0; k < 9; ++k) lf.un[k][i] = u[k];
            }
            else
            {
#pragma unroll
                for (int k = 0; k < 9; ++k) u[k] = lf.un[k][i];
                mx.add(u, own.z[0]);
            }
            put_leaf(hout, a, u, own.z, wmark);
            if (STAGE == 2 && P.dt_leaf) P.dt_leaf[i] = P.initial_tstep;
            dt_loc = fmin(dt_loc, P.initial_tstep);
            continue;
        }
        const Geo<T> geo = leaf_geo<T>(a, level, P);
        NbFace<T> nf[4];
#pragma unroll
        for (int d = 0; d < 4; ++d)
        {
            Cell<T> c;
            if (nid[d] != -1) load_cell<T, true>(hr, nid[d], c);
            else
            {
                c.h[0] = gh[d]; c.qx[0] = gqx[d]; c.qy[0] = gqy[d]; c.z[0] = own.z[0];
                c.h[1] = c.h[2] = c.qx[1] = c.qx[2] = c.qy[1] = c.qy[2] = c.z[1] = c.z[2] = T(0.0);
            }
            if (fric) friction_cell<T, true>(c, P, dt);
            P3<T> b;
            if (d == 0) b = nb_basis<T, NORTH>(geo, nid[d], nl[d], P);
            else if (d == 1) b = nb_basis<T, EAST>(geo, nid[d], nl[d], P);
            else if (d == 2) b = nb_basis<T, SOUTH>(geo, nid[d], nl[d], P);
            else b = nb_basis<T, WEST>(geo, nid[d], nl[d], P);
            nf[d] = nb_face(c, b);
        }
        // operators/copy_to_buf_assem_sol.cu: the stage-1 result of a leaf that is not
        // updated is its state before limiting
        T pre[9];
        if (STAGE == 1)
        {
#pragma unroll
            for (int m = 0; m < 3; ++m) { pre[m] = own.h[m]; pre[3 + m] = own.qx[m]; pre[6 + m] = own.qy[m]; }
        }
        // operators/limit_slopes.cu:3-238 (finest-level leaves inside the DEM only)
        if (P.limit && level == P.L && geo.in_extent)
        {
            const P3<T> eta = {own.z[0] + own.h[0], own.z[1] + own.h[1], own.z[2] + own.h[2]};
            const P3<T> qx = {own.qx[0], own.qx[1], own.qx[2]}, qy = {own.qy[0], own.qy[1], own.qy[2]};
            T e1x, e1y, q1x, q1y, r1x, r1y;
            limited_slopes(eta, nf[0].etaf, nf[1].etaf, nf[2].etaf, nf[3].etaf, nf[0].eta0, nf[1].eta0, nf[2].eta0,
                           nf[3].eta0, P.dx, P.tol_Krivo, e1x, e1y);
            limited_slopes(qx, nf[0].qxf, nf[1].qxf, nf[2].qxf, nf[3].qxf, nf[0].qx0, nf[1].qx0, nf[2].qx0, nf[3].qx0,
                           P.dx, P.tol_Krivo, q1x, q1y);
            limited_slopes(qy, nf[0].qyf, nf[1].qyf, nf[2].qyf, nf[3].qyf, nf[0].qy0, nf[1].qy0, nf[2].qy0, nf[3].qy0,
                           P.dx, P.tol_Krivo, r1x, r1y);
            const bool ax = (T(0.05) * max_h < fmin(own.h[0], fmin(nf[1].h0, nf[3].h0)));
            const bool ay = (T(0.05) * max_h < fmin(own.h[0], fmin(nf[0].h0, nf[2].h0)));
            if (ax) { own.h[1] = e1x - own.z[1]; own.qx[1] = q1x; own.qy[1] = r1x; }
            if (ay) { own.h[2] = e1y - own.z[2]; own.qx[2] = q1y; own.qy[2] = r1y; }
        }
        if (STAGE == 1)
        {
#pragma unroll
            for (int m = 0; m < 3; ++m) { lf.un[m][i] = own.h[m]; lf.un[3 + m][i] = own.qx[m]; lf.un[6 + m][i] = own.qy[m]; }
        }
        // operators/dg2_update.cu:31-79 (wet leaves, not high wall, inside the DEM)
        const bool highwall = (fabs(own.z[0] - P.wall_height) < T(1e-10));
        const bool wet = (own.h[0] >= P.tol_h || nf[0].h0 >= P.tol_h || nf[1].h0 >= P.tol_h || nf[2].h0 >= P.tol_h ||
                          nf[3].h0 >= P.tol_h) && !highwall;
        T leaf_dt = P.initial_tstep;
        if (wet && geo.in_extent)
        {
            // the leaf changes: the encode of the next step revisits its subtree
            if (P.act && level >= P.act_level) P.act[(a - lvl_idx(level)) >> (2 * (level - P.act_level))] = 1;
            T u[9];
            dg2_rhs_update(P3<T>{own.h[0], own.h[1], own.h[2]}, P3<T>{own.qx[0], own.qx[1], own.qx[2]},
                           P3<T>{own.qy[0], own.qy[1], own.qy[2]}, P3<T>{own.z[0], own.z[1], own.z[2]}, nf, geo.dxl, P, dt, u);
            if (STAGE == 2)
            {
#pragma unroll
                for (int k = 0; k < 9; ++k) u[k] = T(0.5) * (u[k] + lf.un[k][i]);
            }
            if (u[0] < P.tol_h)
            {
                u[3] = u[4] = u[5] = u[6] = u[7] = u[8] = T(0.0);
            }
            else if (STAGE == 2)
            {
                const T ux = u[3] / u[0], uy = u[6] / u[0];
                const T dtx = P.CFL * geo.dxl / (fabs(ux) + sqrt(P.g * u[0]));
                const T dty = P.CFL * geo.dxl / (fabs(uy) + sqrt(P.g * u[0]));
                leaf_dt = fmin(dtx, dty);
            }
            if (STAGE == 2)
            {
#pragma unroll
                for (int k = 0; k < 9; ++k) lf.un[k][i] = u[k];
                nan_seen |= (u[0] != u[0]);
                mx.add(u, own.z[0]);
            }
            put_leaf(hout, a, u, own.z, wmark);
        }
        else if (STAGE == 1) put_leaf(hout, a, pre, own.z, wmark);
        else
        {
            T u[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) u[k] = lf.un[k][i];
            mx.add(u, own.z[0]);
            put_leaf(hout, a, u, own.z, wmark);
        }
        if (STAGE == 2 && P.dt_leaf) P.dt_leaf[i] = leaf_dt;
        dt_loc = fmin(dt_loc, leaf_dt);
    }
    if (!LIST)
    {
        const unsigned tot = __reduce_add_sync(0xffffffffu, n_wet);
        if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&sc->wet[STAGE - 1], (int)tot);
    }
    if (STAGE == 2)
    {
        mx.flush(sc);
        dt_loc = warp_min(dt_loc);
        __shared__ T red[kSolverThreads / 32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) red[w] = dt_loc;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            T m = red[0];
            for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = fmin(m, red[k]);
            atomic_min_nn(&sc->dt_min, m);
        }
        if (__syncthreads_or(nan_seen) && threadIdx.x == 0) atomicOr(&sc->status, 1);
    }
}
template <typename T, int STAGE, bool LIST>
__global__ void __launch_bounds__(kSolverThreads, sizeof(T) == 4 ? 5 : 2) k_mwdg2_stage(Leaves<T> lf, Hier<T> hin, Hier<T> hout, Scalars<T>* sc,
                                                                Params<T> P, const StepArgs<T>* args, bool friction,
                                                                const int32_t* wet)
{
    k_mwdg2_stage_body<T, STAGE, LIST>(blockIdx.x, gridDim.x, lf, hin, hout, sc, P, args, friction, wet);
}

// max |h0| of the stage-2 leaf state after ghost cells (run_simulation.cu:613-620).
template <typename T>
__device__ __forceinline__ void k_stage2_maxh_body(int bid, int nb, Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, Params<T> P,
                                                     const StepArgs<T>* args)
{
    const T dt = args->dt;
    const Bnd<T>& B = args->B;
    const int n = sc->n_leaves;
    T mh = T(0);
    for (int i = bid * blockDim.x + threadIdx.x; i < n; i += nb * blockDim.x)
    {
        const int a = lf.act[i];
        const T z0 = hr.s[3][0][a];
        T h0 = hr.s[0][0][a] - z0;
        int32_t nid[4];
        bool border = false;
#pragma unroll
        for (int d = 0; d < 4; ++d) { nid[d] = lf.nb[d][i]; border |= (nid[d] == -1); }
        if (border)
        {
            T gh[4], gqx[4], gqy[4];
            ghost_pass(h0, hr.s[1][0][a], hr.s[2][0][a], z0, nid, (int)lf.lvl[i], a, P, B, dt, gh, gqx, gqy);
        }
        mh = fmax(mh, fabs(h0));
    }
    T v[1] = {mh};
    T* const dst[1] = {&sc->max_h2};
    block_max_atomic<T, 1>(v, dst);
}
template <typename T>
__global__ void __launch_bounds__(256) k_stage2_maxh(Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, Params<T> P,
                                                     const StepArgs<T>* args)
{
    k_stage2_maxh_body<T>(blockIdx.x, gridDim.x, lf, hr, sc, P, args);
}

// operators/fv1_update.cu:3-243 with friction and ghost cells fused. Reads the leaf and its
// neighbours from `hr` and writes the result into the leaf arrays and, at the leaf's own
// index, into `hout`, the other of two alternating hierarchy buffers (no leaf reads `hout`
// in this kernel), with the next step's maxima: the next step needs no re-insertion pass.
template <typename T>
__global__ void __launch_bounds__(kSolverThreads, sizeof(T) == 4 ? 6 : 3) k_hwfv1(Leaves<T> lf, Hier<T> hr, Hier<T> hout, Scalars<T>* sc,
                                                          Params<T> P, const StepArgs<T>* args, bool friction)
{
    const T dt = args->dt;
    const Bnd<T>& B = args->B;
    const int n = sc->n_leaves;
    T dt_loc = (sizeof(T) == 8) ? T(1.0e308) : T(3.0e38);
    bool nan_seen = false;
    StateMax<T> mx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int a = lf.act[i];
        const int level = lf.lvl[i];
        int32_t nid[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) nid[d] = lf.nb[d][i];
        Cell<T> own;
        load_cell<T, false>(hr, a, own);
        // a NaN depth anywhere in the state (a NaN leaf with NaN neighbours is never updated)
        nan_seen |= (own.h[0] != own.h[0]);
        T gh[4], gqx[4], gqy[4];
        ghost_pass(own.h[0], own.qx[0], own.qy[0], own.z[0], nid, level, a, P, B, dt, gh, gqx, gqy);
        bool fric = false;
        if (friction)
        {
            const T h = own.h[0];
            const bool below_depth = (h < P.tol_h);
            const T ux = below_depth ? T(0.0) : own.qx[0] / h;
            const T uy = below_depth ? T(0.0) : own.qy[0] / h;
            const bool below_speed = (fabs(ux) < P.tol_s && fabs(uy) < P.tol_s);
            if (below_depth || below_speed) { own.qx[0] = T(0.0); own.qy[0] = T(0.0); }
            fric = !(below_depth || below_speed);
            if (fric) friction_cell<T, false>(own, P, dt);
        }
        T nbh[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) nbh[d] = (nid[d] != -1) ? hr.s[0][0][nid[d]] - hr.s[3][0][nid[d]] : gh[d];
        if (own.h[0] < P.tol_h && nbh[0] < P.tol_h && nbh[1] < P.tol_h && nbh[2] < P.tol_h && nbh[3] < P.tol_h)
        {
            // dry leaf: not updated (fv1_update.cu:27-46), discharge zeroed by friction if enabled
            lf.un[0][i] = own.h[0];
            lf.un[3][i] = own.qx[0];
            lf.un[6][i] = own.qy[0];
            put_leaf_fv1(hout, a, own.h[0], own.qx[0], own.qy[0], own.z[0], mx);
            if (P.dt_leaf) P.dt_leaf[i] = P.initial_tstep;
            dt_loc = fmin(dt_loc, P.initial_tstep);
            continue;
        }
        V3<T> U[4];
        T zn[4];
#pragma unroll
        for (int d = 0; d < 4; ++d)
        {
            Cell<T> c;
            if (nid[d] != -1) load_cell<T, false>(hr, nid[d], c);
            else { c.h[0] = gh[d]; c.qx[0] = gqx[d]; c.qy[0] = gqy[d]; c.z[0] = own.z[0]; }
            if (fric) friction_cell<T, false>(c, P, dt);
            U[d] = V3<T>{c.h[0], c.qx[0], c.qy[0]};
            zn[d] = c.z[0];
        }
        T h = own.h[0], qx = own.qx[0], qy = own.qy[0];
        const bool wet = (h >= P.tol_h || U[0].h >= P.tol_h || U[1].h >= P.tol_h || U[2].h >= P.tol_h || U[3].h >= P.tol_h);
        T leaf_dt = P.initial_tstep;
        if (wet)
        {
            const T dxl = P.dx * (1 << (P.L - level));
            const T z = own.z[0];
            const T eta_loc = h + z;
            const T zin = fmax(z, zn[0]), zie = fmax(z, zn[1]), zis = fmax(z, zn[2]), ziw = fmax(z, zn[3]);
            const V3<T> Uc = {h, qx, qy};
            const V3<T> Usnn = star(Uc, z, zin, P.tol_h), Usnp = star(U[0], zn[0], zin, P.tol_h);
            const V3<T> F_n = flux_hll_y(Usnn, Usnp, P.tol_h, P.g);
            const V3<T> Usen = star(Uc, z, zie, P.tol_h), Usep = star(U[1], zn[1], zie, P.tol_h);
            const V3<T> F_e = flux_hll_x(Usen, Usep, P.tol_h, P.g);
            const V3<T> Ussn = star(U[2], zn[2], zis, P.tol_h), Ussp = star(Uc, z, zis, P.tol_h);
            const V3<T> F_s = flux_hll_y(Ussn, Ussp, P.tol_h, P.g);
            const V3<T> Uswn = star(U[3], zn[3], ziw, P.tol_h), Uswp = star(Uc, z, ziw, P.tol_h);
            const V3<T> F_w = flux_hll_x(Uswn, Uswp, P.tol_h, P.g);
            // operators/get_bed_src.cuh:7-44
            const T zsw = ziw - fmax(T(0.0), -(eta_loc - ziw));
            const T zse = zie - fmax(T(0.0), -(eta_loc - zie));
            const T bx = P.g * T(0.5) * (Uswp.h + Usen.h) * (zse - zsw) / dxl;
            const T zss = zis - fmax(T(0.0), -(eta_loc - zis));
            const T zsn = zin - fmax(T(0.0), -(eta_loc - zin));
            const T by = P.g * T(0.5) * (Ussp.h + Usnn.h) * (zsn - zss) / dxl;
            h = h - dt * (F_e.h - F_w.h) / dxl;
            qx = qx - dt * ((F_e.qx - F_w.qx) / dxl + bx);
            qy = qy - dt * (F_e.qy - F_w.qy) / dxl;
            h = h - dt * (F_n.h - F_s.h) / dxl;
            qx = qx - dt * (F_n.qx - F_s.qx) / dxl;
            qy = qy - dt * ((F_n.qy - F_s.qy) / dxl + by);
            const bool below_depth = (h < P.tol_h);
            const bool below_disch = (fabs(qx) < P.tol_q && fabs(qy) < P.tol_q);
            if (below_depth || below_disch) { qx = T(0.0); qy = T(0.0); }
            if (!below_depth)
            {
                const T ux = qx / h, uy = qy / h;
                const T dtx = P.CFL * dxl / (fabs(ux) + sqrt(P.g * h));
                const T dty = P.CFL * dxl / (fabs(uy) + sqrt(P.g * h));
                leaf_dt = fmin(dtx, dty);
            }
            nan_seen |= (h != h);
        }
        lf.un[0][i] = h;
        lf.un[3][i] = qx;
        lf.un[6][i] = qy;
        put_leaf_fv1(hout, a, h, qx, qy, own.z[0], mx);
        if (P.dt_leaf) P.dt_leaf[i] = leaf_dt;
        dt_loc = fmin(dt_loc, leaf_dt);
    }
    mx.flush(sc);
    dt_loc = warp_min(dt_loc);
    __shared__ T red[kSolverThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = dt_loc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        T m = red[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = fmin(m, red[k]);
        atomic_min_nn(&sc->dt_min, m);
    }
    if (__syncthreads_or(nan_seen) && threadIdx.x == 0) atomicOr(&sc->status, 1);
}

// Leaf containing each finest cell code (search over the leaves' Z-order starts) and its
// depth eta0 - z0, discharges and bed (output/project_assem_sol.cu:3-77). One warp per
// point: lane j probes position lo + (j + 1) * step of the range [lo, hi] that holds the
// answer (the last leaf whose start is <= c; starts increase along the leaf list), and the
// ballot of the probes narrows the range 32-fold per round (two rounds for a tile's leaves).
// tile_offsets (the scanned leaf counts of the 4^5-cell tiles, ntiles of them; null before
// the first step) narrow the start: leaves are in Z order, so the leaf holding finest cell
// c is among the leaves of tile c >> 10, or is the last leaf before them when a coarser leaf
// covers the whole tile.
template <typename T>
__device__ __forceinline__ void k_sample_points_body(Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, int L, const int32_t* codes, int np,
                                const int32_t* tile_offsets, int ntiles, T* out)
{
    const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (k >= np) return;   // the whole warp
    const int n = sc->n_leaves;
    const int c = codes[k];
    int lo = 0, hi = n - 1;
    if (tile_offsets)
    {
        const int t = c >> (2 * kTileDepth);
        lo = tile_offsets[t];
        hi = (t + 1 < ntiles ? tile_offsets[t + 1] : n) - 1;
        if (hi < lo) lo = hi = lo - 1;
    }
    while (lo < hi)
    {
        const int step = (hi - lo + 31) / 32;
        const int pos = min(hi, lo + (lane + 1) * step);
        const int l = lf.lvl[pos];
        const bool le = ((lf.act[pos] - lvl_idx(l)) << (2 * (L - l))) <= c;
        const int t = __popc(__ballot_sync(0xffffffffu, le));   // probes 0..t-1 start at or before c
        const int nlo = t == 0 ? lo : min(hi, lo + t * step);
        const int nhi = t == 32 ? hi : min(hi, lo + (t + 1) * step) - 1;
        lo = nlo;
        hi = nhi;
    }
    if (lane != 0) return;
    const int a = lf.act[lo];
    const T z0 = hr.s[3][0][a];
    const T eta = lf.un[0][lo] + z0;
    out[4 * k + 0] = eta - z0;
    out[4 * k + 1] = lf.un[3][lo];
    out[4 * k + 2] = lf.un[6][lo];
    out[4 * k + 3] = z0;
}
template <typename T>
__global__ void k_sample_points(Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, int L, const int32_t* codes, int np,
                                const int32_t* tile_offsets, int ntiles, T* out)
{
    k_sample_points_body<T>(lf, hr, sc, L, codes, np, tile_offsets, ntiles, out);
}

// Leaf state with the bed coefficients gathered from the hierarchy, 12 rows of n values.
// Water volume of the leaf state in cell units: sum over leaves of h0 x 4^(L - level), each
// term exact in FP64 (a power-of-two scaling of the leaf's depth) and summed in FP64 whatever
// the state's precision; times dx^2 it is the volume in m^3. One atomic per block.
template <typename T> __global__ void __launch_bounds__(256) k_volume(Leaves<T> lf, const Scalars<T>* sc, int L, double* out)
{
    const int n = sc->n_leaves;
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v += ldexp((double)lf.un[0][i], 2 * (L - (int)lf.lvl[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(out, t);
    }
}

template <typename T> __global__ void k_gather_state(Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, bool mw, double* out)
{
    const int n = sc->n_leaves;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int a = lf.act[i];
        const size_t N = (size_t)n;
        out[0 * N + i] = lf.un[0][i];
        out[1 * N + i] = lf.un[3][i];
        out[2 * N + i] = lf.un[6][i];
        out[3 * N + i] = hr.s[3][0][a];
        out[4 * N + i] = mw ? (double)lf.un[1][i] : 0.0;
        out[5 * N + i] = mw ? (double)lf.un[4][i] : 0.0;
        out[6 * N + i] = mw ? (double)lf.un[7][i] : 0.0;
        out[7 * N + i] = mw ? (double)hr.s[3][1][a] : 0.0;
        out[8 * N + i] = mw ? (double)lf.un[2][i] : 0.0;
        out[9 * N + i] = mw ? (double)lf.un[5][i] : 0.0;
        out[10 * N + i] = mw ? (double)lf.un[8][i] : 0.0;
        out[11 * N + i] = mw ? (double)hr.s[3][2][a] : 0.0;
    }
}

} // namespace mw
