// The learned refinement proposal inside a time step: the MLP's features from the hierarchy,
// and the step's activity labels. No counterpart in the reference.
//
// Coarse level C = L - 3 (a coarse cell spans 8 x 8 finest cells at every max_ref_lvl, so a
// model trained on one mesh size applies to another): the proposal decides per node of
// level C + 1. Only the per-level kernels (levels above kBandMaxLevel) take the mask; the
// banded small levels are always encoded and decoded in full, so the proposal acts on
// max_ref_lvl >= 11 (levels 10 and up) and only records at smaller ones.
#pragma once

#include "kernels.cuh"
#include "proposal.cuh"

namespace mw {

__host__ __device__ inline int proposal_level(int L) { return L - 3; }

// Feature scales: depths in units of 2 m, discharges of 4 m^2/s, bed differences of 8 m.
constexpr float kFeatH = 0.5f, kFeatQ = 0.25f, kFeatZ = 0.125f, kFeatClamp = 16.0f;

template <typename T>
__device__ __forceinline__ float feat(T v, float scale)
{
    const float f = (float)v * scale;
    return fminf(kFeatClamp, fmaxf(-kFeatClamp, f));
}

// One feature row per node c of level C (row-major BF16 [4^C][128]): for the node and its
// eight neighbours (dx, dy in -1..1, row-major from the south-west), the 12 values h, qx, qy
// and z - z_centre (modes 0, 1x, 1y each) of the node, or of the coarser leaf holding it
// (the first level on its root path whose node is not significant); zeros outside the
// mesh; then the four children's activity bits of the last step, a constant 1, zeros.
template <typename T>
__global__ void __launch_bounds__(128) k_prop_features(Hier<T> hr, int C, const uint8_t* __restrict__ lab_prev,
                                                       __nv_bfloat16* __restrict__ feats)
{
    const int64_t nC = (int64_t)1 << (2 * C);
    const int nside = 1 << C;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nC; c += (int64_t)gridDim.x * blockDim.x)
    {
        const int x = compact((int)c), y = compact((int)(c >> 1));
        uint4* row = reinterpret_cast<uint4*>(feats + c * mlp::kIn);
        float stage[8];
        int ns = 0, col = 0;
        auto flush = [&]() {
            __align__(16) __nv_bfloat162 b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) b[i] = __floats2bfloat162_rn(stage[2 * i], stage[2 * i + 1]);
            row[col++] = *reinterpret_cast<const uint4*>(b);
            ns = 0;
        };
        auto push = [&](float v) {
            stage[ns++] = v;
            if (ns == 8) flush();
        };
        T zc = T(0);
#pragma unroll 1
        for (int s = 0; s < 9; ++s)
        {
            // the centre first, so its bed is known for the others
            const int k = (s == 0) ? 4 : (s <= 4 ? s - 1 : s);
            const int xx = x + (k % 3) - 1, yy = y + (k / 3) - 1;
            float v[12];
            if (xx < 0 || yy < 0 || xx >= nside || yy >= nside)
            {
#pragma unroll
                for (int i = 0; i < 12; ++i) v[i] = 0.0f;
            }
            else
            {
                const int code = morton(xx, yy);
                int lev = C;
                for (int j = 0; j < C; ++j)
                    if (!(hr.flags[lvl_idx(j) + (code >> (2 * (C - j)))] & F_SIG)) { lev = j; break; }
                const int node = lvl_idx(lev) + (code >> (2 * (C - lev)));
                const T z0 = hr.s[3][0][node];
                if (s == 0) zc = z0;
#pragma unroll
                for (int m = 0; m < 3; ++m)
                {
                    const T z = hr.s[3][m][node];
                    v[m] = feat(hr.s[0][m][node] - z, kFeatH);
                    v[3 + m] = feat(hr.s[1][m][node], kFeatQ);
                    v[6 + m] = feat(hr.s[2][m][node], kFeatQ);
                    v[9 + m] = feat(m == 0 ? z - zc : z, kFeatZ);
                }
            }
#pragma unroll
            for (int i = 0; i < 12; ++i) push(v[i]);
        }
        const uint32_t bits = lab_prev[c];
#pragma unroll
        for (int j = 0; j < 4; ++j) push((float)((bits >> j) & 1u));
        push(1.0f);
        while (col < mlp::kIn / 8) push(0.0f);
    }
}

// End of a step: the activity of the four children of every node c of level C (act, one
// byte per node of level C + 1, set by the encode and the RK stages) becomes lab[c] (bit j:
// child j), the next step's input bits and, for training, the label of this step's features;
// act is cleared for the next step. With a proposal (prop: one byte per node of level C + 1)
// counts the active subtrees it left out.
static __global__ void __launch_bounds__(256) k_prop_labels(uint8_t* __restrict__ act, const uint8_t* __restrict__ prop,
                                                     uint8_t* __restrict__ lab, int64_t nC, uint32_t* __restrict__ counts)
{
    uint32_t active = 0, missed = 0, proposed = 0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nC; c += (int64_t)gridDim.x * blockDim.x)
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(act + 4 * c);
        const uint32_t a = *w;
        const uint32_t bits = (a & 1u) | ((a >> 7) & 2u) | ((a >> 14) & 4u) | ((a >> 21) & 8u);
        lab[c] = (uint8_t)bits;
        if (a) *w = 0u;
        active += __popc(bits);
        if (prop)
        {
            const uint32_t p = *reinterpret_cast<const uint32_t*>(prop + 4 * c);
            const uint32_t pb = (p & 1u) | ((p >> 7) & 2u) | ((p >> 14) & 4u) | ((p >> 21) & 8u);
            missed += __popc(bits & ~pb);
            proposed += __popc(pb);
        }
    }
    active = __reduce_add_sync(0xffffffffu, active);
    missed = __reduce_add_sync(0xffffffffu, missed);
    proposed = __reduce_add_sync(0xffffffffu, proposed);
    if ((threadIdx.x & 31) == 0)
    {
        if (active) atomicAdd(&counts[0], active);
        if (missed) atomicAdd(&counts[1], missed);
        if (proposed) atomicAdd(&counts[2], proposed);
    }
}

} // namespace mw
