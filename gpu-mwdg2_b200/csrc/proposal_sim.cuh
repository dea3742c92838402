// The learned refinement proposal inside a time step: the MLP's features from the hierarchy,
// the step's activity labels, and the fused proposal kernel. No counterpart in the reference.
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

// The node holding cell `code` of level C: the first level on its root path whose node is not
// significant (a coarser leaf), else the cell itself. The C flag loads are independent.
__device__ __forceinline__ int coarse_node(const uint8_t* flags, int C, int code)
{
    uint32_t nonsig = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (j < C && !(flags[lvl_idx(j) + (code >> (2 * (C - j)))] & F_SIG)) nonsig |= 1u << j;
    const int lev = nonsig ? __ffs(nonsig) - 1 : C;
    return lvl_idx(lev) + (code >> (2 * (C - lev)));
}

// One feature row per node c of level C (row-major BF16 [4^C][128]): for the node and its
// eight neighbours (the centre first, then dx, dy in -1..1 row-major from the south-west),
// the 12 values h, qx, qy and z - z_centre (modes 0, 1x, 1y each) of the node, or of the
// coarser leaf holding it; zeros outside the mesh; then the four children's activity bits of
// the last step, a constant 1, zeros.
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
        auto push = [&](float v) {
            stage[ns++] = v;
            if (ns == 8)
            {
                __align__(16) __nv_bfloat162 b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) b[i] = __floats2bfloat162_rn(stage[2 * i], stage[2 * i + 1]);
                row[col++] = *reinterpret_cast<const uint4*>(b);
                ns = 0;
            }
        };
        T zc = T(0);
#pragma unroll
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
                const int node = coarse_node(hr.flags, C, morton(xx, yy));
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
#pragma unroll
        for (int i = 0; i < 15; ++i) push(0.0f);
    }
}

// End of a step: the activity of the four children of every node c of level C, which
// becomes lab[c] (bit j: child j), the next step's input bits and, for training, the label
// of this step's features. A child subtree (node s of level C + 1) is active when the RK
// stages updated one of its leaves (act[s], set by the stage kernels; cleared here for the
// next step) or when its significance flags at the end of the step -- s and its four
// children, the last two parent levels -- differ from those at the end of the last step
// (sig[s], a 5-bit signature kept here). The final flags are compared, not the encode's
// decisions: a flag the encode clears and extra significance sets again in the same step
// is no change. With a proposal (prop: one byte per node of level C + 1) counts the active
// subtrees it left out.
// (static kernels here: the header is included by more than one translation unit)
static __global__ void __launch_bounds__(256) k_prop_labels(uint8_t* __restrict__ act, const uint8_t* __restrict__ prop,
                                                            const uint8_t* __restrict__ flags, int C,
                                                            uint8_t* __restrict__ sig, uint8_t* __restrict__ lab,
                                                            int64_t nC, uint32_t* __restrict__ counts)
{
    uint32_t active = 0, missed = 0, proposed = 0;
    const uint8_t* f1 = flags + lvl_idx(C + 1);
    const uint8_t* f2 = flags + lvl_idx(C + 2);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nC; c += (int64_t)gridDim.x * blockDim.x)
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(act + 4 * c);
        const uint32_t a = *w;
        uint32_t* sw = reinterpret_cast<uint32_t*>(sig + 4 * c);
        const uint32_t old = *sw;
        const uint32_t own = *reinterpret_cast<const uint32_t*>(f1 + 4 * c);
        uint32_t now = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const uint32_t kids = *reinterpret_cast<const uint32_t*>(f2 + 16 * c + 4 * j);
            const uint32_t s5 = ((own >> (8 * j)) & F_SIG) | ((kids & F_SIG) << 1) | (((kids >> 8) & F_SIG) << 2) |
                                (((kids >> 16) & F_SIG) << 3) | (((kids >> 24) & F_SIG) << 4);
            now |= s5 << (8 * j);
        }
        if (now != old) *sw = now;
        const uint32_t changed = now ^ old;
        uint32_t bits = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (((a >> (8 * j)) & 0xffu) || ((changed >> (8 * j)) & 0xffu)) bits |= 1u << j;
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
    __shared__ uint32_t red[3][8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
    {
        red[0][w] = active;
        red[1][w] = missed;
        red[2][w] = proposed;
    }
    __syncthreads();
    if (threadIdx.x < 3)
    {
        uint32_t t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[threadIdx.x][k];
        if (t) atomicAdd(&counts[threadIdx.x], t);
    }
}

// ---------------------------------------------------------------- fused proposal
// Shared memory of k_mlp_propose after the MLP's own regions: the coarse-level values of a
// tile's 16 x 8 cells and their one-cell ring (18 x 10), and the ring's activity bits.
template <typename T> struct ProposeSmem
{
    static constexpr int kHx = 18, kHy = 10, kHalo = kHx * kHy;
    static constexpr int Vals = (mlp::FwdSmem::Total + 15) / 16 * 16;   // [180][12] T
    static constexpr int Labs = Vals + kHalo * 12 * (int)sizeof(T);     // [180] bytes
    static constexpr int Total = Labs + (kHalo + 15) / 16 * 16;
};

// Proposal of one step in one kernel (learned mode; the parameters as k_mlp_pack's image):
// per 128-row tile of the coarse level (a 16 x 8 block of its nodes in Z order) the ring of
// last-step activity bits decides whether the tile can hold activity at all; a tile with
// none around it proposes nothing (no features, no MLP). Otherwise the 180 cells of the
// block and its ring are read once into shared memory (the same node search and values as
// k_prop_features), each thread assembles its row of features from them into the MLP's
// operand tile, and the tensor-core forward pass (mlp::forward_tile) gives the four
// children's proposal bits.
template <typename T>
__global__ void __launch_bounds__(mlp::kRows, 1) k_mlp_propose(const uint8_t* __restrict__ pack, Hier<T> hr, int C,
                                                               const uint8_t* __restrict__ lab_prev,
                                                               uint8_t* __restrict__ prop, float thr, int* err)
{
    using S = ProposeSmem<T>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + mlp::FwdSmem::Bar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + mlp::FwdSmem::Slot);
    T* vals = reinterpret_cast<T*>(sm + S::Vals);
    uint8_t* labs = sm + S::Labs;
    const int r = threadIdx.x;
    mlp::load_packed(pack, sm + mlp::FwdSmem::W1);
    if (r == 0) mlp::mbar_init(bar, 1);
    if (r < 32) mlp::tmem_alloc(slot, 256);
    mlp::tc_fence_before();
    __syncthreads();
    mlp::tc_fence_after();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    const int nside = 1 << C;
    const int64_t ntiles = ((int64_t)1 << (2 * C)) / mlp::kRows;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x)
    {
        const int code0 = (int)(t * mlp::kRows);
        const int x0 = compact(code0), y0 = compact(code0 >> 1);
        // activity bits of the block and its ring
        bool any = false;
        for (int i = r; i < S::kHalo; i += blockDim.x)
        {
            const int gx = x0 + i % S::kHx - 1, gy = y0 + i / S::kHx - 1;
            const bool in = gx >= 0 && gy >= 0 && gx < nside && gy < nside;
            const uint8_t b = in ? lab_prev[morton(gx, gy)] : (uint8_t)0;
            labs[i] = b;
            any |= (b != 0);
        }
        if (!__syncthreads_or(any ? 1 : 0))
        {
            *reinterpret_cast<uint32_t*>(prop + 4 * (int64_t)(code0 + r)) = 0u;
            continue;
        }
        // values of the block and its ring: the node, or the coarser leaf holding it
        for (int i = r; i < S::kHalo; i += blockDim.x)
        {
            const int gx = x0 + i % S::kHx - 1, gy = y0 + i / S::kHx - 1;
            T* v = vals + 12 * i;
            if (gx < 0 || gy < 0 || gx >= nside || gy >= nside) continue;   // never read
            const int node = coarse_node(hr.flags, C, morton(gx, gy));
#pragma unroll
            for (int m = 0; m < 3; ++m)
            {
                const T z = hr.s[3][m][node];
                v[m] = hr.s[0][m][node] - z;
                v[3 + m] = hr.s[1][m][node];
                v[6 + m] = hr.s[2][m][node];
                v[9 + m] = z;
            }
        }
        __syncthreads();
        // this thread's row, in the order of k_prop_features, into the MLP's operand tile
        {
            const int lx = compact(r) + 1, ly = compact(r >> 1) + 1;
            const int x = x0 + lx - 1, y = y0 + ly - 1;
            uint8_t* sX = sm + mlp::FwdSmem::X;
            float stage[8];
            int ns = 0, col = 0;
            auto push = [&](float f) {
                stage[ns++] = f;
                if (ns == 8)
                {
                    mlp::st_row8(sX, r, 8 * col, mlp::kIn, stage);
                    ++col;
                    ns = 0;
                }
            };
            const T zc = vals[12 * (ly * S::kHx + lx) + 9];
#pragma unroll
            for (int s = 0; s < 9; ++s)
            {
                const int k = (s == 0) ? 4 : (s <= 4 ? s - 1 : s);
                const int dx = (k % 3) - 1, dy = (k / 3) - 1;
                const bool in = x + dx >= 0 && y + dy >= 0 && x + dx < nside && y + dy < nside;
                const T* v = vals + 12 * ((ly + dy) * S::kHx + lx + dx);
#pragma unroll
                for (int m = 0; m < 3; ++m) push(in ? feat(v[m], kFeatH) : 0.0f);
#pragma unroll
                for (int m = 0; m < 3; ++m) push(in ? feat(v[3 + m], kFeatQ) : 0.0f);
#pragma unroll
                for (int m = 0; m < 3; ++m) push(in ? feat(v[6 + m], kFeatQ) : 0.0f);
#pragma unroll
                for (int m = 0; m < 3; ++m) push(in ? feat(m == 0 ? v[9] - zc : v[9 + m], kFeatZ) : 0.0f);
            }
            const uint32_t bits = labs[ly * S::kHx + lx];
#pragma unroll
            for (int j = 0; j < 4; ++j) push((float)((bits >> j) & 1u));
            push(1.0f);
#pragma unroll
            for (int i = 0; i < 15; ++i) push(0.0f);
        }
        float z[mlp::kOut];
        ok = mlp::forward_tile(sm, tmem, bar, phase, z, false, nullptr, nullptr, nullptr);
        if (!ok) break;
        uint32_t pbits = 0;
#pragma unroll
        for (int o = 0; o < mlp::kOut; ++o) pbits |= (z[o] > thr ? 1u : 0u) << (8 * o);
        *reinterpret_cast<uint32_t*>(prop + 4 * (int64_t)(code0 + r)) = pbits;
    }
    if (!ok && err) atomicExch(err, 1);
    mlp::tc_fence_before();
    __syncthreads();
    if (r < 32) mlp::tmem_dealloc(tmem, 256);
}

} // namespace mw
