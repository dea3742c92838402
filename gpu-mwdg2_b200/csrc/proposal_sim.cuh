// The learned refinement proposal inside a time step: the MLP's features from the hierarchy,
// the step's activity labels, and the fused proposal kernel. No counterpart in the reference.
//
// Coarse level C = L - 3 (a coarse cell spans 8 x 8 finest cells at every max_ref_lvl, so a
// model trained on one mesh size applies to another): the proposal decides per node of
// level C + 1. A subtree left out keeps its flags and values: the per-level kernels (levels
// above kBandMaxLevel) skip its parents, a band CTA whose whole subtree is left out returns
// at once (band_left_out), and the RK stages' dry-leaf writer leaves its dry leaves' state
// where it stands (k_stage_dry). Wet leaves are updated wherever they are.
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

// Proposal tiles: 128 consecutive Morton codes of level C, a block of 16 x 8 cells.
constexpr int kPropTile = 128;

// Where an active cell sits in its tile, for the tile summaries (Proposal ring bits): bit 0
// any; 1-4 on the north, south, east, west edge; 5-8 in the NE, NW, SE, SW corner.
__device__ __forceinline__ uint32_t ring_bits(int local)
{
    const int lx = compact(local), ly = compact(local >> 1);   // 0..15, 0..7
    const bool n = ly == 7, so = ly == 0, e = lx == 15, w = lx == 0;
    return 1u | (n ? 2u : 0u) | (so ? 4u : 0u) | (e ? 8u : 0u) | (w ? 16u : 0u) | (n && e ? 32u : 0u) |
           (n && w ? 64u : 0u) | (so && e ? 128u : 0u) | (so && w ? 256u : 0u);
}

// Whether tile t (south-west cell x0, y0) or the one-cell ring around it held activity in
// the last step: its own summary and the facing edge or corner of each of its 8 neighbours.
__device__ __forceinline__ bool tile_needed(const uint16_t* ring, int C, int x0, int y0)
{
    const int nside = 1 << C;
    bool need = false;
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        const int dx = k % 3 - 1, dy = k / 3 - 1;
        const int x = x0 + (dx < 0 ? -1 : dx * 16), y = y0 + (dy < 0 ? -1 : dy * 8);
        if (x < 0 || y < 0 || x >= nside || y >= nside) continue;
        // the neighbour's side that faces this tile
        const uint32_t want = (dx == 0 && dy == 0) ? 1u
                            : (dx == 0) ? (dy > 0 ? 4u : 2u)                      // north tile: its south edge
                            : (dy == 0) ? (dx > 0 ? 16u : 8u)                     // east tile: its west edge
                            : (dy > 0) ? (dx > 0 ? 256u : 128u)                   // NE: its SW corner; NW: its SE
                                       : (dx > 0 ? 64u : 32u);                    // SE: its NW corner; SW: its NE
        need |= (ring[morton(x, y) >> 7] & want) != 0;
    }
    return need;
}

// End of a step: the activity of the four children of every node c of level C, which
// becomes lab[c] (bit j: child j), the next step's input bits and, for training, the label
// of this step's features. A child subtree (node s of level C + 1) is active when the RK
// stages updated one of its leaves (act[s], set by the stage kernels; cleared here for the
// next step) or when its significance flags at the end of the step -- s and its four
// children, the last two parent levels -- differ from those at the end of the last step
// (sig[s], a 5-bit signature kept here). The final flags are compared, not the encode's
// decisions: a flag the encode clears and extra significance sets again in the same step
// is no change. With a proposal (prop: one byte per node of level C + 1) counts the subtrees
// it left out that needed the step (counts[1]): their leaves were updated or their flags
// gained significance (a subtree left out where significance is lost keeps detail that the
// step would have dropped, which costs nothing in accuracy), the subtrees proposed
// (counts[2]) and those that needed the step (counts[3]); counts[0]: the active subtrees
// (the labels). ring[t]: the summary of tile t's bits (ring_bits) for the next
// step's k_mlp_propose.
// (static kernels here: the header is included by more than one translation unit)
static __global__ void __launch_bounds__(256) k_prop_labels(uint8_t* __restrict__ act, const uint8_t* __restrict__ prop,
                                                            const uint8_t* __restrict__ flags, int C,
                                                            uint8_t* __restrict__ sig, uint8_t* __restrict__ lab,
                                                            uint16_t* __restrict__ ring, int64_t nC,
                                                            uint32_t* __restrict__ counts)
{
    uint32_t active = 0, missed = 0, proposed = 0, needed = 0;
    const uint8_t* f1 = flags + lvl_idx(C + 1);
    const uint8_t* f2 = flags + lvl_idx(C + 2);
    __shared__ uint32_t tile_or[8];
    // the loop is uniform over the block: each round takes 256 consecutive nodes (two tiles)
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nC; base += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t c = base + threadIdx.x;
        uint32_t edge = 0;
        if (c < nC)
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
            const uint32_t changed = now ^ old, gained = now & ~old;
            uint32_t bits = 0, need = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                if (((a >> (8 * j)) & 0xffu) || ((changed >> (8 * j)) & 0xffu)) bits |= 1u << j;
                if (((a >> (8 * j)) & 0xffu) || ((gained >> (8 * j)) & 0xffu)) need |= 1u << j;
            }
            lab[c] = (uint8_t)bits;
            if (a) *w = 0u;
            active += __popc(bits);
            if (prop)
            {
                const uint32_t p = *reinterpret_cast<const uint32_t*>(prop + 4 * c);
                const uint32_t pb = (p & 1u) | ((p >> 7) & 2u) | ((p >> 14) & 4u) | ((p >> 21) & 8u);
                missed += __popc(need & ~pb);
                proposed += __popc(pb);
                needed += __popc(need);
            }
            edge = bits ? ring_bits((int)(c & (kPropTile - 1))) : 0u;
        }
        // the tile summaries for the next step's k_mlp_propose (a warp's 32 nodes lie in one
        // tile of 128)
        edge = __reduce_or_sync(0xffffffffu, edge);
        if ((threadIdx.x & 31) == 0) tile_or[threadIdx.x >> 5] = edge;
        __syncthreads();
        if (threadIdx.x < 2 && base + kPropTile * threadIdx.x < nC)
        {
            const int w0 = 4 * threadIdx.x;
            ring[(base >> 7) + threadIdx.x] = (uint16_t)(tile_or[w0] | tile_or[w0 + 1] | tile_or[w0 + 2] | tile_or[w0 + 3]);
        }
        __syncthreads();
    }
    active = __reduce_add_sync(0xffffffffu, active);
    missed = __reduce_add_sync(0xffffffffu, missed);
    proposed = __reduce_add_sync(0xffffffffu, proposed);
    needed = __reduce_add_sync(0xffffffffu, needed);
    __shared__ uint32_t red[4][8];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
    {
        red[0][w] = active;
        red[1][w] = missed;
        red[2][w] = proposed;
        red[3][w] = needed;
    }
    __syncthreads();
    if (threadIdx.x < 4)
    {
        uint32_t t = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[threadIdx.x][k];
        if (t) atomicAdd(&counts[threadIdx.x], t);
    }
}

// What the proposal keeps whatever the MLP says: the subtrees that were active in the last
// step (lab_prev: their leaves or flags changed, so their parents must be encoded again
// before their values are read as neighbours) and the subtrees holding a point source (its
// inflow enters the finest level and reaches the leaves only through the encode).
static __global__ void __launch_bounds__(256) k_prop_force(uint8_t* __restrict__ prop, const uint8_t* __restrict__ lab_prev,
                                                           int64_t nC, const int32_t* __restrict__ src_nodes, int nsrc)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nC; c += (int64_t)gridDim.x * blockDim.x)
    {
        const uint32_t b = lab_prev[c];
        if (b)
            atomicOr(reinterpret_cast<unsigned int*>(prop + 4 * c),
                     (b & 1u) | ((b & 2u) << 7) | ((b & 4u) << 14) | ((b & 8u) << 21));
    }
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < nsrc; i += blockDim.x)
            atomicOr(reinterpret_cast<unsigned int*>(prop + (src_nodes[i] & ~3)), 1u << (8 * (src_nodes[i] & 3)));
}

// ---------------------------------------------------------------- fused proposal
// Shared memory of k_mlp_propose after the MLP's own regions: the coarse-level values of a
// tile's 16 x 8 cells and their one-cell ring (18 x 10), the CTA's list of tiles to run, and
// the mbarrier of the parameters' bulk copy.
template <typename T> struct ProposeSmem
{
    static constexpr int kHx = 18, kHy = 10, kHalo = kHx * kHy, kList = mlp::kRows;
    static constexpr int Vals = (mlp::FwdSmem::Total + 15) / 16 * 16;   // [180][12] T
    static constexpr int List = Vals + kHalo * 12 * (int)sizeof(T);     // [kList] int32 tile ids
    static constexpr int Count = List + kList * 4;                      // int32
    static constexpr int ParBar = Count + 8;                            // uint64 mbarrier
    static constexpr int Total = ParBar + 8;
};

// Bulk copy (TMA, this GPU's memory, no multicast) of `bytes` from global memory into this
// CTA's shared memory, completing on `bar`; one thread issues it. Both addresses are 16-byte
// aligned and bytes is a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mlp::smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     mlp::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(mlp::smem_u32(bar))
                 : "memory");
}

// Proposal of one step in one kernel (learned mode; the parameters as k_mlp_pack's image).
// Each CTA takes the tiles t = blockIdx.x + j * gridDim.x (128 rows each: a 16 x 8 block of
// level-C nodes in Z order). The tile summaries of the last step's labels (ring, from
// k_prop_labels) say which of them, or the one-cell ring around them, held activity; a tile
// with none proposes nothing (activity spreads within a step only from an active
// neighbour), so its 128 proposal words are cleared and nothing else is read. A CTA with
// tiles to run copies the parameter image into shared memory with one bulk copy, overlapped
// with its first tile's gather, and allocates its tensor memory; per tile the 180 cells of
// the block and its ring are read once into shared memory (the same node search and values
// as k_prop_features), each thread assembles its row of features from them into the MLP's
// operand tile, and the tensor-core forward pass (mlp::forward_tile) gives the four
// children's proposal bits. A tensor-core or copy wait that runs out sets bit 1 of *err (the
// step's Scalars::status, read back with the step's scalars).
template <typename T>
__global__ void __launch_bounds__(mlp::kRows, 1) k_mlp_propose(const uint8_t* __restrict__ pack, Hier<T> hr, int C,
                                                               const uint8_t* __restrict__ lab_prev,
                                                               const uint16_t* __restrict__ ring,
                                                               uint8_t* __restrict__ prop, float thr, int* err)
{
    using S = ProposeSmem<T>;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + mlp::FwdSmem::Bar);
    uint64_t* pbar = reinterpret_cast<uint64_t*>(sm + S::ParBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + mlp::FwdSmem::Slot);
    T* vals = reinterpret_cast<T*>(sm + S::Vals);
    int* list = reinterpret_cast<int*>(sm + S::List);
    int* count = reinterpret_cast<int*>(sm + S::Count);
    const int r = threadIdx.x;
    const int nside = 1 << C;
    const int64_t ntiles = ((int64_t)1 << (2 * C)) / mlp::kRows;
    bool started = false, have_params = false, ok = true;
    uint32_t tmem = 0, phase = 0;
    for (int64_t j0 = 0; blockIdx.x + j0 * gridDim.x < ntiles && ok; j0 += S::kList)
    {
        // which of the next kList tiles of this CTA need the MLP; the others are cleared here
        if (r == 0) *count = 0;
        __syncthreads();
        const int64_t t = blockIdx.x + (j0 + r) * gridDim.x;
        if (t < ntiles)
        {
            const int code0 = (int)(t * mlp::kRows);
            if (tile_needed(ring, C, compact(code0), compact(code0 >> 1))) list[atomicAdd(count, 1)] = (int)t;
            else
            {
                uint4* w = reinterpret_cast<uint4*>(prop + 4 * (int64_t)code0);
#pragma unroll 8
                for (int i = 0; i < mlp::kRows * 4 / 16; ++i) w[i] = make_uint4(0u, 0u, 0u, 0u);
            }
        }
        __syncthreads();
        const int n = *count;
        __syncthreads();   // every thread holds n before the next round resets the count
        if (n > 0 && !started)
        {
            started = true;
            if (r == 0)
            {
                mlp::mbar_init(bar, 1);
                mlp::mbar_init(pbar, 1);
                mlp::fence_async_smem();
                bulk_load(sm + mlp::FwdSmem::W1, pack, mlp::kPackBytes, pbar);
            }
            if (r < 32) mlp::tmem_alloc(slot, 256);
            mlp::tc_fence_before();
            __syncthreads();
            mlp::tc_fence_after();
            tmem = *slot;
        }
        for (int k = 0; k < n && ok; ++k)
        {
            const int code0 = list[k] * mlp::kRows;
            const int x0 = compact(code0), y0 = compact(code0 >> 1);
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
            const uint32_t bits = lab_prev[code0 + r];
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
                    const int kk = (s == 0) ? 4 : (s <= 4 ? s - 1 : s);
                    const int dx = (kk % 3) - 1, dy = (kk / 3) - 1;
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
#pragma unroll
                for (int jb = 0; jb < 4; ++jb) push((float)((bits >> jb) & 1u));
                push(1.0f);
#pragma unroll
                for (int i = 0; i < 15; ++i) push(0.0f);
            }
            // the parameters, before the CTA's first MMA (phase 0 of their barrier)
            if (!have_params)
            {
                have_params = true;
                if (!mlp::mbar_wait(pbar, 0)) { ok = false; break; }
            }
            float z[mlp::kOut];
            ok = mlp::forward_tile(sm, tmem, bar, phase, z, false, nullptr, nullptr, nullptr);
            if (!ok) break;
            uint32_t pbits = 0;
#pragma unroll
            for (int o = 0; o < mlp::kOut; ++o) pbits |= (z[o] > thr ? 1u : 0u) << (8 * o);
            *reinterpret_cast<uint32_t*>(prop + 4 * (int64_t)(code0 + r)) = pbits;
        }
    }
    if (started)
    {
        // the parameter copy has landed before the CTA ends (bounded: a copy that never
        // lands is reported through err)
        if (!mlp::mbar_wait(pbar, 0)) ok = false;
        if (!ok && err && r == 0) atomicOr(err, 2);
        mlp::tc_fence_before();
        __syncthreads();
        if (r < 32) mlp::tmem_dealloc(tmem, 256);
    }
}

} // namespace mw
