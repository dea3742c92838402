// Host entry points over the CPU oracle's filter functions (oracle/oracle_common.hpp), for
// tests/test_filter_kat.py, which compiles this file with g++ into a temporary shared
// library; same signatures as tests/filter_kat_host.cu (FP64 only: the oracle's filters are
// checked in the type its golden fixtures pin).
#include "../oracle/oracle_common.hpp"

extern "C" {
void kat_oracle_mw_encode(const double* in, double* scale, double* details)
{
    oracle::Kids<double> k;
    for (int m = 0; m < 3; ++m)
        for (int c = 0; c < 4; ++c) k.u[m][c] = in[4 * m + c];
    for (int r = 0; r < 3; ++r) scale[r] = oracle::encode_scale_mw(r, k);
    const oracle::Det9<double> d = oracle::encode_details_mw(k);
    for (int t = 0; t < 3; ++t)
        for (int r = 0; r < 3; ++r) details[3 * t + r] = d.d[t][r];
}
void kat_oracle_mw_decode(const double* scale, const double* details, double* out)
{
    const double s[3] = {scale[0], scale[1], scale[2]};
    oracle::Det9<double> d;
    for (int t = 0; t < 3; ++t)
        for (int r = 0; r < 3; ++r) d.d[t][r] = details[3 * t + r];
    for (int c = 0; c < 4; ++c)
        for (int m = 0; m < 3; ++m) out[4 * m + c] = oracle::decode_mw(c, m, s, d);
}
void kat_oracle_hw_encode(const double* in, double* out)
{
    const double c[4] = {in[0], in[1], in[2], in[3]};
    out[0] = oracle::hw_scale(c);
    out[1] = oracle::hw_alpha(c);
    out[2] = oracle::hw_beta(c);
    out[3] = oracle::hw_gamma(c);
}
}
