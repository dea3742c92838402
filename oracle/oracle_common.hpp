// CPU oracle for the adaptive MWDG2/HWFV1 time step: shared definitions.
//
// TEST INFRASTRUCTURE ONLY. This file and everything under oracle/ restate the
// reference algorithm (al0vya/gpu-mwdg2, source/) on the CPU so that tests and the
// CPU-baseline leg of bench.py can check the CUDA product. Nothing in the product
// links, imports or calls it.
//
// Floating-point expressions keep the reference's operand order and parenthesisation;
// the oracle is compiled with -ffp-contract=off, so it evaluates them in plain IEEE
// arithmetic (the CUDA builds may fuse multiply-adds).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace oracle {

// types/SolverTypes.h:3-7, types/InletTypes.h:3-11, types/Directions.h:3-14
enum Solver { HWFV1 = 1, MWDG2 = 2 };
enum Inlet { CLOSED = 1, FREE = 2, HFIX = 4, HVAR = 8, QFIX = 16, QVAR = 32 };
enum Dir { NORTH = 1, EAST = 2, SOUTH = 4, WEST = 8 };

// utilities/get_lvl_idx.cuh:6,11-24 -- first slot of level n in a hierarchy array
inline int lvl_idx(int level) { return ((1 << (2 * level)) - 1) / 3 + 3; }

// zorder/dilate.cuh:25-41
inline int dilate(int c)
{
    c &= 0x0000ffff;
    c = (c ^ (c << 8)) & 0x00ff00ff;
    c = (c ^ (c << 4)) & 0x0f0f0f0f;
    c = (c ^ (c << 2)) & 0x33333333;
    c = (c ^ (c << 1)) & 0x55555555;
    return c;
}

// zorder/compact.cuh:9-21
inline int compact(int code)
{
    int c = code & 0x55555555;
    c = (c ^ (c >> 1)) & 0x33333333;
    c = (c ^ (c >> 2)) & 0x0f0f0f0f;
    c = (c ^ (c >> 4)) & 0x00ff00ff;
    c = (c ^ (c >> 8)) & 0x0000ffff;
    return c;
}

// zorder/generate_morton_code.cuh:7-16
inline int morton(int x, int y) { return dilate(x) | (dilate(y) << 1); }

// Multiwavelet filter table of mra/Filters.h:202-397.
// kH/kGA/kGB/kGC[f][r][k] = HHf_(r+1)(k+1), GAf_.., GBf_.., GCf_.. ; f is the filter
// index, which maps to the child in Morton order as child = {0, 2, 1, 3}[f].
// The values are those of the reference so that results agree to the last bit.
constexpr double kH[4][3][3] = {
    {{0.5, 0.0, 0.0}, {-0.4330127018922193, 0.25, 0.0}, {-0.4330127018922193, 0.0, 0.25}},
    {{0.5, 0.0, 0.0}, {-0.4330127018922193, 0.25, 0.0}, {0.4330127018922193, 0.0, 0.25}},
    {{0.5, 0.0, 0.0}, {0.4330127018922193, 0.25, 0.0}, {-0.4330127018922193, 0.0, 0.25}},
    {{0.5, 0.0, 0.0}, {0.4330127018922193, 0.25, 0.0}, {0.4330127018922193, 0.0, 0.25}}};
constexpr double kGA[4][3][3] = {
    {{-0.2672612419124244, -0.4629100498862757, -0.4629100498862757}, {0.0, 0.0, -0.7071067811865476}, {0.0, -0.7071067811865476, 0.0}},
    {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
    {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
    {{0.2672612419124244, -0.4629100498862757, -0.4629100498862757}, {0.0, 0.0, 0.7071067811865476}, {0.0, 0.7071067811865476, 0.0}}};
constexpr double kGB[4][3][3] = {
    {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}},
    {{-0.2672612419124244, -0.4629100498862757, 0.46291004988627577}, {0.0, 0.0, -0.7071067811865476}, {0.0, -0.7071067811865476, 0.0}},
    {{0.2672612419124244, -0.4629100498862757, 0.46291004988627577}, {0.0, 0.0, 0.7071067811865476}, {0.0, 0.7071067811865476, 0.0}},
    {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}}};
constexpr double kGC[4][3][3] = {
    {{0.5, 0.0, 0.0}, {-0.1636634176769942, -0.2834733547569204, 0.37796447300922725}, {-0.1636634176769942, 0.37796447300922725, -0.2834733547569204}},
    {{-0.5, 0.0, 0.0}, {-0.1636634176769942, -0.2834733547569204, -0.3779644730092272}, {0.16366341767699427, -0.3779644730092272, -0.2834733547569204}},
    {{-0.5, 0.0, 0.0}, {0.16366341767699427, -0.2834733547569204, -0.3779644730092272}, {-0.1636634176769942, -0.3779644730092272, -0.2834733547569204}},
    {{0.5, 0.0, 0.0}, {0.16366341767699427, -0.2834733547569204, 0.37796447300922725}, {0.16366341767699427, 0.37796447300922725, -0.2834733547569204}}};
// Haar filter pair (mra/Filters.h:202-205)
constexpr double kH0 = 0.7071067811865475, kH1 = 0.7071067811865475;
constexpr double kG0 = 0.7071067811865475, kG1 = -0.7071067811865475;

// Children of one parent: u[m][c] = mode m (0, 1x, 1y) of child c (Morton order 0..3).
template <typename T> struct Kids { T u[3][4]; };
// Nine details of one field: d[t][m], t = alpha, beta, gamma; m = mode 0, 1x, 1y.
template <typename T> struct Det9 { T d[3][3]; };

// Order in which the reference sums the 12 taps of one filter row
// (mra/encode_scale.cuh:13-38): filter 0 on child 0, filter 1 on child 2,
// filter 2 on child 1, filter 3 on child 3; modes 0, 1x, 1y within each.
template <typename T>
inline T mw_row(const double (&F)[4][3][3], int r, const Kids<T>& k)
{
    const int child_of[4] = {0, 2, 1, 3};
    T acc = T(F[0][r][0]) * k.u[0][child_of[0]];
    for (int f = 0; f < 4; ++f)
        for (int m = 0; m < 3; ++m)
        {
            if (f == 0 && m == 0) continue;
            acc = acc + T(F[f][r][m]) * k.u[m][child_of[f]];
        }
    return acc / T(2.0);
}

// mra/encode_scale.cuh:13-38 (scale modes 0, 1x, 1y of the parent)
template <typename T> inline T encode_scale_mw(int r, const Kids<T>& k) { return mw_row(kH, r, k); }

// mra/encode_details.cuh:65-188 -> (alpha, beta, gamma) x (0, 1x, 1y)
template <typename T> inline Det9<T> encode_details_mw(const Kids<T>& k)
{
    Det9<T> d;
    for (int m = 0; m < 3; ++m)
    {
        d.d[0][m] = mw_row(kGA, m, k);
        d.d[1][m] = mw_row(kGB, m, k);
        d.d[2][m] = mw_row(kGC, m, k);
    }
    return d;
}

// classes/SubDetail.h:12-46 -- max |detail| of the nine details of one field
template <typename T> inline T det9_max(const Det9<T>& d)
{
    T m[3];
    for (int i = 0; i < 3; ++i)
    {
        T a = std::fmax(std::fabs(d.d[0][i]), std::fabs(d.d[1][i]));
        m[i] = std::fmax(std::fabs(d.d[2][i]), a);
    }
    T mx = std::fmax(m[0], m[1]);
    return std::fmax(m[2], mx);
}

// mra/decode_scale_children.cuh:81-395 -- mode k of child c from the parent's
// scale modes s[3] and nine details; terms in the reference's order.
template <typename T>
inline T decode_mw(int c, int k, const T (&s)[3], const Det9<T>& d)
{
    const int filt_of[4] = {0, 2, 1, 3};
    const int f = filt_of[c];
    T acc = T(kH[f][0][k]) * s[0];
    acc = acc + T(kH[f][1][k]) * s[1];
    acc = acc + T(kH[f][2][k]) * s[2];
    acc = acc + T(kGA[f][0][k]) * d.d[0][0];
    acc = acc + T(kGA[f][1][k]) * d.d[0][1];
    acc = acc + T(kGA[f][2][k]) * d.d[0][2];
    acc = acc + T(kGB[f][0][k]) * d.d[1][0];
    acc = acc + T(kGB[f][1][k]) * d.d[1][1];
    acc = acc + T(kGB[f][2][k]) * d.d[1][2];
    acc = acc + T(kGC[f][0][k]) * d.d[2][0];
    acc = acc + T(kGC[f][1][k]) * d.d[2][1];
    acc = acc + T(kGC[f][2][k]) * d.d[2][2];
    return acc * T(2.0);
}

// Haar (FV1) filters: mra/encode_scale.cuh:7-11, mra/encode_details.cuh:7-23
template <typename T> inline T hw_scale(const T (&c)[4])
{
    return T(0.5) * (T(kH0) * (T(kH0) * c[0] + T(kH1) * c[2]) + T(kH1) * (T(kH0) * c[1] + T(kH1) * c[3]));
}
template <typename T> inline T hw_alpha(const T (&c)[4])
{
    return T(0.5) * (T(kH0) * (T(kG0) * c[0] + T(kG1) * c[2]) + T(kH1) * (T(kG0) * c[1] + T(kG1) * c[3]));
}
template <typename T> inline T hw_beta(const T (&c)[4])
{
    return T(0.5) * (T(kG0) * (T(kH0) * c[0] + T(kH1) * c[2]) + T(kG1) * (T(kH0) * c[1] + T(kH1) * c[3]));
}
template <typename T> inline T hw_gamma(const T (&c)[4])
{
    return T(0.5) * (T(kG0) * (T(kG0) * c[0] + T(kG1) * c[2]) + T(kG1) * (T(kG0) * c[1] + T(kG1) * c[3]));
}
// mra/decode_scale_children.cuh:38-76 (children 0..3 in Morton order)
template <typename T> inline void hw_decode(T u, T a, T b, T g, T (&out)[4])
{
    out[0] = (T(kH0) * (T(kH0) * u + T(kG0) * a) + T(kG0) * (T(kH0) * b + T(kG0) * g)) * T(2.0);
    out[2] = (T(kH0) * (T(kH1) * u + T(kG1) * a) + T(kG0) * (T(kH1) * b + T(kG1) * g)) * T(2.0);
    out[1] = (T(kH1) * (T(kH0) * u + T(kG0) * a) + T(kG1) * (T(kH0) * b + T(kG0) * g)) * T(2.0);
    out[3] = (T(kH1) * (T(kH1) * u + T(kG1) * a) + T(kG1) * (T(kH1) * b + T(kG1) * g)) * T(2.0);
}

} // namespace oracle
