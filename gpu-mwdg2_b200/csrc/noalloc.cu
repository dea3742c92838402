// Leaf-topology construction that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs under a memory manager which owns
// all of the device's memory (a host framework that reserves the device heap up front),
// and real-time loops that must not enter the CUDA allocator (cudaMalloc and cudaFree may
// synchronise the device and take driver locks). mwdg2_leaf_topology_static serves them:
// the caller passes the significance flags and the output arrays, and the only scratch
// the kernels need -- one leaf count per tile and the total -- lives in the file-scope
// device array g_topology_scratch below. Every GPU that loads this library holds that
// array (about 256 KiB) until the process exits.
#include "../../include/mwdg2.h"
#include "kernels.cuh"

#include <string>

// Records the text returned by mwdg2_last_error (defined with the other entry points).
void mwdg2_detail_set_last_error(const char* msg);

namespace {

// 4^(max_ref_lvl - 5) tiles of 4^5 finest cells: 65536 tiles covers max_ref_lvl <= 13.
constexpr int kStaticMaxLevel = 13;
constexpr int kStaticMaxTiles = 1 << (2 * (kStaticMaxLevel - mw::kTileDepth));

struct TopologyScratch
{
    int32_t tile_counts[kStaticMaxTiles];  // per-tile leaf counts, then their exclusive scan
    mw::Scalars<float> scalars;            // n_leaves: total written by the scan
};

// Shared by every call on this device; see the synchronisation note in include/mwdg2.h.
static __device__ __align__(256) TopologyScratch g_topology_scratch;

mwdg2_status fail(mwdg2_status st, const std::string& msg)
{
    mwdg2_detail_set_last_error(msg.c_str());
    return st;
}

// Device address of g_topology_scratch on the current device. In host code the symbol
// itself is only a host-side stand-in and must never be passed to a kernel. The address is
// looked up on every call rather than cached: the lookup is cheap, and a cached address
// would go stale if the caller reset the device (the module, and the array with it, is
// loaded again afterwards and may land elsewhere).
mwdg2_status scratch_on_current_device(TopologyScratch** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_topology_scratch);
    if (e != cudaSuccess || p == nullptr)
        return fail(MWDG2_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = static_cast<TopologyScratch*>(p);
    return MWDG2_OK;
}

} // namespace

extern "C" mwdg2_status mwdg2_leaf_topology_static(const uint8_t* d_sig, int max_ref_lvl, int xsz, int ysz,
                                                   int32_t* d_act, uint8_t* d_levels, int32_t* d_nb_ids,
                                                   uint8_t* d_nb_levels, int64_t cap, int64_t* n_leaves_out,
                                                   void* stream)
{
    if (!d_sig || !d_act || !d_levels || !d_nb_ids || !d_nb_levels || !n_leaves_out)
        return fail(MWDG2_ERR_ARG, "mwdg2_leaf_topology_static: null pointer argument");
    if (max_ref_lvl < mw::kTileDepth || max_ref_lvl > kStaticMaxLevel)
        return fail(MWDG2_ERR_ARG, "mwdg2_leaf_topology_static: max_ref_lvl must be between 5 and 13 "
                                   "(the static scratch holds 65536 tile counts)");
    // the kernels read the flags four at a time
    if (reinterpret_cast<uintptr_t>(d_sig) % 4 != 0)
        return fail(MWDG2_ERR_ARG, "mwdg2_leaf_topology_static: d_sig must be 4-byte aligned");
    const int M = 1 << max_ref_lvl;
    if (xsz < 1 || ysz < 1 || xsz > M || ysz > M)
        return fail(MWDG2_ERR_ARG, "mwdg2_leaf_topology_static: xsz and ysz must be within 1..2^max_ref_lvl");
    const int64_t F = (int64_t)M * M;
    if (cap < F)
        return fail(MWDG2_ERR_ARG, "mwdg2_leaf_topology_static: cap must be at least 4^max_ref_lvl");
    TopologyScratch* scratch = nullptr;
    if (mwdg2_status s = scratch_on_current_device(&scratch)) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int D = mw::kTileDepth;
    const int ntiles = 1 << (2 * (max_ref_lvl - D));
    // Every tile count and the total are written before they are read, so nothing in the
    // scratch has to start at zero.
    mw::k_tile_count<<<ntiles, mw::kTileThreads, 0, st>>>(d_sig, max_ref_lvl, scratch->tile_counts);
    mw::k_tile_scan<float><<<1, 1024, 0, st>>>(scratch->tile_counts, ntiles, &scratch->scalars);
    mw::Leaves<float> lf{};
    lf.act = d_act;
    lf.lvl = d_levels;
    for (int d = 0; d < 4; ++d)
    {
        lf.nb[d] = d_nb_ids + (size_t)d * cap;
        lf.nbl[d] = d_nb_levels + (size_t)d * cap;
    }
    mw::k_tile_emit<float, true><<<ntiles, mw::kTileThreads, 0, st>>>(lf, d_sig, scratch->tile_counts, max_ref_lvl, M, xsz,
                                                                ysz, nullptr, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MWDG2_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    int32_t n = 0;
    e = cudaMemcpyAsync(&n, &scratch->scalars.n_leaves, sizeof(n), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(MWDG2_ERR_CUDA, std::string("leaf topology: ") + cudaGetErrorString(e));
    *n_leaves_out = n;
    return MWDG2_OK;
}
