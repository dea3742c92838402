// Host entry points over the library's filter functions (gpu-mwdg2_b200/csrc/mw_math.cuh,
// the same templates the CUDA kernels use), for tests/test_filter_kat.py, which compiles
// this file with nvcc into a temporary shared library. prec: 32 or 64 (the type T).
#include "../gpu-mwdg2_b200/csrc/mw_math.cuh"

namespace {

template <typename T> void mw_encode(const double* in, double* scale, double* details)
{
    T c[3][4];
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 4; ++k) c[m][k] = T(in[4 * m + k]);
    T s[3], d[3][3];
    mw::mw_encode_scale(c, s);
    mw::mw_encode_details(c, d);
    for (int r = 0; r < 3; ++r) scale[r] = s[r];
    for (int t = 0; t < 3; ++t)
        for (int r = 0; r < 3; ++r) details[3 * t + r] = d[t][r];
}

template <typename T> void mw_decode(const double* scale, const double* details, double* out)
{
    T s[3], d[3][3], c[3][4];
    for (int r = 0; r < 3; ++r) s[r] = T(scale[r]);
    for (int t = 0; t < 3; ++t)
        for (int r = 0; r < 3; ++r) d[t][r] = T(details[3 * t + r]);
    mw::mw_decode(s, d, c);
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 4; ++k) out[4 * m + k] = c[m][k];
}

template <typename T> void hw_encode(const double* in, double* out)
{
    const T c[4] = {T(in[0]), T(in[1]), T(in[2]), T(in[3])};
    out[0] = mw::hw_scale(c);
    out[1] = mw::hw_alpha(c);
    out[2] = mw::hw_beta(c);
    out[3] = mw::hw_gamma(c);
}

}  // namespace

extern "C" {
void kat_mw_encode(int prec, const double* children, double* scale, double* details)
{
    if (prec == 32) mw_encode<float>(children, scale, details);
    else mw_encode<double>(children, scale, details);
}
void kat_mw_decode(int prec, const double* scale, const double* details, double* children)
{
    if (prec == 32) mw_decode<float>(scale, details, children);
    else mw_decode<double>(scale, details, children);
}
void kat_hw_encode(int prec, const double* children, double* out)
{
    if (prec == 32) hw_encode<float>(children, out);
    else hw_encode<double>(children, out);
}
}
