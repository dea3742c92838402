// Batched ensemble step: one launch per kernel over every member of a size class (same
// max_ref_lvl, MWDG2, same precision). Member m is blockIdx.y; its arrays, scalars and
// parameters come from a table in device memory (MemberArgs), and the kernel bodies are the
// single-simulation kernels' own (the *_body functions), so a member's step computes
// exactly what a standalone step of it computes. The per-level, band and tile bodies see
// blockIdx.x and gridDim.x of their member's row of the grid; the persistent per-leaf bodies
// take the block index and count within their member from a block map that shares the
// launch's blocks among the members by their last step's work. No counterpart in the
// reference, which runs one case per process (run_simulation.cu:9-222).
//
// The batched step takes one fixed sequence of kernels: both RK stages over the wet list
// (the wet test, the dry-leaf writer beside the wet-list kernel) and the per-level kernel for
// every level above the bands. A standalone step picks between these and a one-sweep stage
// or a sparse-level kernel from the last step's counts; every choice gives the same bits.
#pragma once

#include "kernels.cuh"
#include "solver.cuh"

namespace mw {

template <typename T> struct MemberArgs
{
    Scalars<T>* sc;              // device scalars (and the stage-point values after them)
    void* sc_host;               // the member's pinned host copy of that block (mapped)
    int scal_bytes;
    const StepArgs<T>* m_args;   // this step's dt and boundary values (mapped pinned)
    StepArgs<T>* d_args;
    const Src<T>* m_src;         // point sources (mapped pinned)
    int nsrc;
    Hier<T> hr, hs;
    Leaves<T> lf;
    Params<T> P;
    T dx, eps;
    int M, xsz, ysz;
    int32_t* tile_counts;
    uint8_t* dry1;
    uint8_t* dry2;
    int32_t* wet;
    int fric, limit;
    const int32_t* stage_codes;
    int np;
    T* stage_out;
};

// The members' table, passed by value as the kernels' parameter (a __grid_constant__
// parameter lives in the constant bank, so a block reads its member's pointers where it uses
// them instead of holding the whole entry in registers); a class has at most kMax members.
template <typename T> struct MemberTable
{
    static constexpr int kMax = 30000 / (int)sizeof(MemberArgs<T>);
    MemberArgs<T> m[kMax];
};

// Per-leaf launches split their blocks among the members in proportion to each member's
// work in the last step (leaves, or wet leaves for the wet-list kernels), so that a large or
// wet member does not finish long after the others with a fixed share: first[m] is the
// first block of member m and first[n] the blocks in use (kBlockMaps maps of n + 1 entries:
// leaves, stage-1 wet list, stage-2 wet list).
constexpr int kBlockMaps = 3;

// The member of block b: the last m with first[m] <= b (members with no blocks share their
// start with the next one).
__device__ __forceinline__ int member_of(const int32_t* first, int n, int b)
{
    int lo = 0, hi = n;
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The step's first kernel: member m steps when active[m] (mapped pinned, written by the
// host before the launch); the flag goes to on[m] in device memory for the later kernels,
// and so do the block maps (map_host -> map, kBlockMaps x (n + 1)).
template <typename T>
__global__ void k_members_open(const __grid_constant__ MemberTable<T> tab, const uint8_t* active, uint8_t* on, int L,
                               const int32_t* map_host, int32_t* map, int n)
{
    const int m = blockIdx.y;
    __shared__ int go;
    if (threadIdx.x == 0)
    {
        go = active[m];
        on[m] = (uint8_t)go;
    }
    if (threadIdx.x < kBlockMaps)
    {
        const int k = threadIdx.x * (n + 1) + m;
        map[k] = map_host[k];
        if (m == n - 1) map[k + 1] = map_host[k + 1];
    }
    __syncthreads();
    if (!go) return;
    const MemberArgs<T>& a = tab.m[m];
    k_step_open_body<T>(a.sc, true, a.m_args, a.d_args, a.m_src, a.nsrc, a.hr, a.dx, L);
}

// FULL: the encode of the hierarchy, else the scale-only re-encode of the stage hierarchy.
template <typename T, bool FULL>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_members_encode_level(const __grid_constant__ MemberTable<T> tab,
                                                                                     const uint8_t* on, int L, int level)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_encode_level_body<T, true, FULL>(FULL ? a.hr : a.hs, a.sc, L, level, a.eps);
}

template <typename T, bool FULL>
__global__ void __launch_bounds__(256) k_members_encode_band(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int L, int lo,
                                                            int depth)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_encode_band_body<T, true, FULL>(FULL ? a.hr : a.hs, a.sc, L, lo, depth, a.eps, PropMask{});
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_members_decode_band(const __grid_constant__ MemberTable<T> tab,
                                                                                    const uint8_t* on, int L, int lo,
                                                                                    int depth)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_decode_band_body<T, true>(a.hr, a.sc, L, lo, depth, a.eps, PropMask{});
}

template <typename T>
__global__ void __launch_bounds__(256) k_members_extra_sig(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int L, int level)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_extra_sig_level_body<T>(a.hr.flags, a.sc, L, level, a.eps);
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_members_decode_level(const __grid_constant__ MemberTable<T> tab,
                                                                                     const uint8_t* on, int L, int level)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_decode_level_body<T, true>(a.hr, a.sc, L, level, a.eps, PropMask{});
}

template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_members_tile_count(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int L)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_tile_count_body(a.hr.flags, L, a.tile_counts);
}

template <typename T>
__global__ void __launch_bounds__(1024) k_members_tile_scan(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int ntiles)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_tile_scan_body<T>(a.tile_counts, ntiles, a.sc);
}

template <typename T>
__global__ void __launch_bounds__(kTileThreads, 8) k_members_tile_emit(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int L)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    k_tile_emit_body<T, false>(a.lf, a.hr.flags, a.tile_counts, L, a.M, a.xsz, a.ysz, &a.sc->min_leaf, &a.sc->n_prev);
}

// The member of this block of a per-leaf launch (one-dimensional grid) and the block's
// index and count within the member; false: no member's block.
// The RK stage kernels: stage 1 reads the hierarchy and writes the stage hierarchy, stage 2
// the reverse (friction in stage 1 only).
__device__ __forceinline__ bool member_block(const int32_t* first, int n, const uint8_t* on, int& m, int& bid, int& nb)
{
    const int b = blockIdx.x;
    if (b >= first[n]) return false;
    m = member_of(first, n, b);
    bid = b - first[m];
    nb = first[m + 1] - first[m];
    return on[m] != 0;
}

template <typename T, int STAGE>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_members_stage_wet(const __grid_constant__ MemberTable<T> tab,
                                                                                  const uint8_t* on,
                                                                                  const int32_t* first, int n)
{
    int m, bid, nb;
    if (!member_block(first, n, on, m, bid, nb)) return;
    const MemberArgs<T>& a = tab.m[m];
    k_stage_wet_body<T, STAGE>(bid, nb, a.lf, STAGE == 1 ? a.hr : a.hs, a.sc, a.P, a.d_args,
                               STAGE == 1 ? a.dry1 : a.dry2, a.wet);
}

template <typename T, int STAGE>
__global__ void __launch_bounds__(kSolverThreads, sizeof(T) == 4 ? 5 : 2) k_members_stage_list(const __grid_constant__ MemberTable<T> tab,
                                                                                              const uint8_t* on,
                                                                                              const int32_t* first,
                                                                                              int n)
{
    int m, bid, nb;
    if (!member_block(first, n, on, m, bid, nb)) return;
    const MemberArgs<T>& a = tab.m[m];
    k_mwdg2_stage_body<T, STAGE, true>(bid, nb, a.lf, STAGE == 1 ? a.hr : a.hs, STAGE == 1 ? a.hs : a.hr, a.sc, a.P,
                                       a.d_args, STAGE == 1 && a.fric, a.wet);
}

template <typename T, int STAGE>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 5) k_members_stage_dry(const __grid_constant__ MemberTable<T> tab, const uint8_t* on,
                                                          const int32_t* first, int n)
{
    int m, bid, nb;
    if (!member_block(first, n, on, m, bid, nb)) return;
    const MemberArgs<T>& a = tab.m[m];
    k_stage_dry_body<T, STAGE>(bid, nb, a.lf, STAGE == 1 ? a.hr : a.hs, STAGE == 1 ? a.hs : a.hr, a.sc, a.P,
                               STAGE == 1 && a.fric, STAGE == 1 ? a.dry1 : a.dry2, a.dry1, PropMask{});
}

template <typename T>
__global__ void __launch_bounds__(256) k_members_stage2_maxh(const __grid_constant__ MemberTable<T> tab, const uint8_t* on,
                                                            const int32_t* first, int n)
{
    int m, bid, nb;
    if (!member_block(first, n, on, m, bid, nb)) return;
    const MemberArgs<T>& a = tab.m[m];
    if (!a.limit) return;
    k_stage2_maxh_body<T>(bid, nb, a.lf, a.hs, a.sc, a.P, a.d_args);
}

// The step's end: the stage points of members that have them, then every stepping member's
// scalars (and stage-point values) straight into its pinned host block.
template <typename T>
__global__ void k_members_sample(const __grid_constant__ MemberTable<T> tab, const uint8_t* on, int L, int ntiles)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    if ((int)(blockIdx.x * blockDim.x) >= 32 * a.np) return;
    k_sample_points_body<T>(a.lf, a.hr, a.sc, L, a.stage_codes, a.np, a.tile_counts, ntiles, a.stage_out);
}

template <typename T> __global__ void k_members_scalars_out(const __grid_constant__ MemberTable<T> tab, const uint8_t* on)
{
    if (!on[blockIdx.y]) return;
    const MemberArgs<T>& a = tab.m[blockIdx.y];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.sc);
    uint32_t* dst = reinterpret_cast<uint32_t*>(a.sc_host);
    for (int i = threadIdx.x; i < a.scal_bytes / 4; i += blockDim.x) dst[i] = src[i];
}

} // namespace mw
