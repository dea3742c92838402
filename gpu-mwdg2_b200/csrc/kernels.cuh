// CUDA kernels of the adaptive MWDG2/HWFV1 time step for sm_100a.
//
// Data layout in HBM (one simulation):
//   hierarchy  s[field][mode][h]   field eta,qx,qy,z; mode 0,1x,1y; h = get_lvl_idx(level)+Morton
//   flags[p]                       parents only (levels 0..L-1); flag bits F_SIG/F_ENC/F_PRE
//   stage      s[field<3][mode][h] of the RK stage-1 result (leaves and significant parents;
//              the bed is shared with the hierarchy)
//   leaves     act, lvl, nb[4], nbl[4], un[9] (state), in Z order
//
// Work per step touches the significant part of the tree and the leaves only. Details are
// never stored: the decode recomputes them from the children (F_ENC marks the parents
// whose details are non-zero this step), so no detail or norm array is written or cleared.
#pragma once

#include "mw_math.cuh"

namespace mw {

constexpr int kTileDepth = 5;        // a leaf-enumeration tile covers 4^5 finest cells
constexpr int kTileThreads = 256;
constexpr int kSolverThreads = 128;

template <typename T> struct Hier
{
    T* s[4][3];
    uint8_t* flags;
    // Keep-values decode, stage hierarchy only (null otherwise): per hierarchy index,
    // (step tag << 1) | changed for the step in which the slot's value was last made
    // current; changed = 1 where that step wrote a value (RK stage 1 at a leaf, the scale
    // re-encode at a parent), 0 where it confirmed the one standing (a frozen dry leaf, a
    // parent whose children all stood). See encode_parent.
    uint32_t* tag = nullptr;
};

template <typename T> struct Leaves
{
    int32_t* act;
    uint8_t* lvl;
    int32_t* nb[4];
    uint8_t* nbl[4];
    T* un[9];   // [field*3 + mode], field h, qx, qy
    // learned refinement proposal (null otherwise): same[i] = 1 where position i holds the
    // leaf it held in the last step (k_tile_emit), so un[i] already holds that leaf's state
    uint8_t* same;
};

template <typename T> struct Scalars
{
    T max_eta, max_h, max_qx, max_z;  // raw maxima of |.| over leaves (floored at 1 by users)
    T max_h2;                         // max |h0| for the stage-2 limiter (not floored)
    T dt_min;
    int32_t n_leaves;
    int32_t status;                   // bit 0: NaN seen in the state; bit 1: a proposal wait ran out
    unsigned long long enc, enc2, dec;
    uint32_t sig_level[16];           // significant parents decoded per level (levels above the bands)
    int32_t wet[2];                   // leaves not dry in RK stage 1 / stage 2 (wet-list lengths)
    T next_max[4];                    // maxima of the state at the end of the step (eta, h, qx, z)
    T xs_factor;                      // 2^(M_BAR+1) of the extra-significance threshold (extra_eps)
    int32_t min_leaf;                 // lowest leaf level of this step's tree (k_tile_emit)
    int32_t n_prev;                   // the last step's leaf count (k_tile_scan, before it writes n_leaves)
    // learned refinement proposal (csrc/proposal.cuh): subtrees of the proposal level that
    // were active in the step, left out though they needed the step, proposed, and needed
    uint32_t prop_active, prop_missed, prop_proposed, prop_needed;
    uint32_t prop_frozen;             // dry leaves of left-out subtrees the RK stages left as they stood
    uint32_t step_tag;                // 1, 2, ...: the step's number for the frozen-leaf tags
};

// The subtrees below the nodes of level `level` (the proposal level) that a step's encode and
// decode visit: prop[node] != 0 (null: all), or act[node] != 0 where act is given (the
// subtrees whose leaves this step's RK stages have updated so far).
struct PropMask
{
    const uint8_t* prop;
    int level;
    const uint8_t* act = nullptr;
};

// Whether the subtree below node `node` of the mask's level is left out.
__device__ __forceinline__ bool pm_out(const PropMask& pm, int64_t node)
{
    return pm.prop && !pm.prop[node] && !(pm.act && pm.act[node]);
}


// A band CTA (node blockIdx.x of level lo and its subtree) holding no node of the mask's
// level that the proposal kept: like the parents of a subtree the level kernels leave out,
// its parents keep their flags and values (PM semantics extended to the levels above the
// mask). Checked for masks at most 7 levels below lo (4^7 bytes per CTA); called by every
// thread of the CTA.
__device__ __forceinline__ bool band_left_out(const PropMask& pm, int lo)
{
    if (!pm.prop || pm.level < lo || pm.level - lo > 7) return false;
    const int sh = 2 * (pm.level - lo), n = 1 << sh;
    const int64_t first = (int64_t)blockIdx.x << sh;
    bool any = false;
    if (n >= 4)
    {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(pm.prop + first);
        const uint32_t* wa = pm.act ? reinterpret_cast<const uint32_t*>(pm.act + first) : nullptr;
        for (int i = threadIdx.x; i < n / 4; i += blockDim.x) any |= (w[i] != 0u) || (wa && wa[i] != 0u);
    }
    else
        for (int i = threadIdx.x; i < n; i += blockDim.x) any |= !pm_out(pm, first + i);
    return __syncthreads_or(any ? 1 : 0) == 0;
}

template <typename T> struct Params
{
    int L, M, xsz, ysz, limit;
    T dx, tol_h, tol_q, tol_s, g, manning, CFL, initial_tstep, wall_height, tol_Krivo, eps;
    T* dt_leaf;   // per-leaf CFL step of the final stage (VTK output), or null
    // learned refinement proposal: the RK stages mark the node of level act_level above every
    // leaf they update (act[node] = 1); null: no marks
    uint8_t* act;
    int act_level;
};

template <typename T> struct Bnd
{
    int start[4], end[4], type[4];   // N, E, S, W
    T inlet[4];
    int west_special;                // 1 monai, 2 oregon-seaside wave makers on the west side
    T time;                          // simulated time of the step (oregon-seaside wave maker)
};

template <typename T> struct Src { int code, type; T value; };

// Values that change from step to step, in device memory: the step's first operation copies
// them from pinned host memory, so a captured step replays with new values.
template <typename T> struct StepArgs
{
    T dt;        // the step's time step
    Bnd<T> B;    // boundary segments, inlet values and time at this step
};

// ---------------------------------------------------------------- atomics on non-negative reals
__device__ __forceinline__ void atomic_max_nn(double* a, double v)
{
    atomicMax(reinterpret_cast<unsigned long long*>(a), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_nn(float* a, float v)
{
    atomicMax(reinterpret_cast<unsigned int*>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_min_nn(double* a, double v)
{
    atomicMin(reinterpret_cast<unsigned long long*>(a), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_nn(float* a, float v)
{
    atomicMin(reinterpret_cast<unsigned int*>(a), __float_as_uint(v));
}

template <typename T> __device__ __forceinline__ T warp_max(T v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <typename T> __device__ __forceinline__ T warp_min(T v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide max of several values then one atomic per value per block.
template <typename T, int N>
__device__ __forceinline__ void block_max_atomic(T (&v)[N], T* const (&dst)[N])
{
    __shared__ T red[N][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = warp_max(v[k]);
    if (lane == 0)
    {
#pragma unroll
        for (int k = 0; k < N; ++k) red[k][w] = v[k];
    }
    __syncthreads();
    if (w == 0)
    {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
            T x = (lane < nw) ? red[k][lane] : T(0);
            x = warp_max(x);
            if (lane == 0) atomic_max_nn(dst[k], x);
        }
    }
}

// ---------------------------------------------------------------- step bookkeeping
// carry: the maxima come from the previous step's last solver kernel (every step after the
// first); otherwise k_leaf_maxima computes them.
template <typename T> __device__ __forceinline__ void step_begin(Scalars<T>* sc, bool carry)
{
    sc->max_eta = carry ? sc->next_max[0] : T(0);
    sc->max_h = carry ? sc->next_max[1] : T(0);
    sc->max_qx = carry ? sc->next_max[2] : T(0);
    sc->max_z = carry ? sc->next_max[3] : T(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) sc->next_max[k] = T(0);
    sc->max_h2 = T(0);
    sc->dt_min = (sizeof(T) == 8) ? T(1.0e308) : T(3.0e38);
    sc->enc = 0; sc->enc2 = 0; sc->dec = 0;
    sc->wet[0] = 0; sc->wet[1] = 0;
    sc->min_leaf = 1 << 30;
    // the expression of mra/extra_significance_kernel.cu, evaluated once per step instead of
    // once per parent (the same expression on the device gives the same bits everywhere)
    sc->xs_factor = pow(T(2.0), T(1.5) + 1);
#pragma unroll
    for (int l = 0; l < 16; ++l) sc->sig_level[l] = 0;
    sc->prop_active = 0;
    sc->prop_missed = 0;
    sc->prop_proposed = 0;
    sc->prop_needed = 0;
    sc->prop_frozen = 0;
    sc->step_tag += 1u;
}
template <typename T> __global__ void k_step_begin(Scalars<T>* sc, bool carry) { step_begin(sc, carry); }

// Point source i into the finest level (mra/reinsert_point_srcs.cu:3-29).
template <typename T> __device__ __forceinline__ void point_source(const Hier<T>& hr, const Src<T>& src, T dt, T dx, int L)
{
    const int h = lvl_idx(L) + src.code;
    const int t = src.type;
    if (t == HFIX || t == HVAR) hr.s[0][0][h] = src.value;
    else if (t == QFIX || t == QVAR) hr.s[0][0][h] += src.value * dt / dx;
}

// A step's first kernel (one block): resets the step's scalars, copies the step's
// arguments (dt, boundary values), which it reads straight from pinned host memory, to
// device memory for the later kernels, and applies the point sources, whose values it also
// reads from pinned host memory. One launch in place of two copies and two kernels.
template <typename T>
__device__ __forceinline__ void k_step_open_body(Scalars<T>* sc, bool carry, const StepArgs<T>* h_args, StepArgs<T>* d_args, const Src<T>* h_src,
                            int nsrc, Hier<T> hr, T dx, int L)
{
    __shared__ T s_dt;
    // the first source of each thread is read before the barrier, beside the arguments
    Src<T> first{};
    if ((int)threadIdx.x < nsrc) first = h_src[threadIdx.x];
    if (threadIdx.x == 0)
    {
        const StepArgs<T> a = *h_args;
        *d_args = a;
        s_dt = a.dt;
        step_begin(sc, carry);
    }
    __syncthreads();
    if ((int)threadIdx.x < nsrc) point_source(hr, first, s_dt, dx, L);
    for (int i = threadIdx.x + blockDim.x; i < nsrc; i += blockDim.x) point_source(hr, h_src[i], s_dt, dx, L);
}
template <typename T>
__global__ void k_step_open(Scalars<T>* sc, bool carry, const StepArgs<T>* h_args, StepArgs<T>* d_args, const Src<T>* h_src,
                            int nsrc, Hier<T> hr, T dx, int L)
{
    k_step_open_body<T>(sc, carry, h_args, d_args, h_src, nsrc, hr, dx, L);
}

// Maxima of the leaf state (mra/get_max_scale_coeffs.cu:3-27, with the reference's
// use of qx0 for the qy maximum), for the first step; later steps take them from the
// previous step's last solver kernel, which also re-inserts the state into the hierarchy
// (mra/reinsert_assem_sol.cu:3-32).
template <typename T>
__global__ void __launch_bounds__(256) k_leaf_maxima(Leaves<T> lf, Hier<T> hr, Scalars<T>* sc, int n_fixed)
{
    const int n = n_fixed >= 0 ? n_fixed : sc->n_leaves;
    T me = T(0), mh = T(0), mq = T(0), mz = T(0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int a = lf.act[i];
        const T h0 = lf.un[0][i], qx0 = lf.un[3][i];
        const T z0 = hr.s[3][0][a];
        const T eta = h0 + z0;
        me = fmax(me, fabs(eta));
        mh = fmax(mh, fabs(h0));
        mq = fmax(mq, fabs(qx0));
        mz = fmax(mz, fabs(z0));
    }
    T v[4] = {me, mh, mq, mz};
    T* const dst[4] = {&sc->max_eta, &sc->max_h, &sc->max_qx, &sc->max_z};
    block_max_atomic<T, 4>(v, dst);
}

// Point sources into the finest level, from device copies of the step's arguments.
template <typename T>
__global__ void k_point_sources(Hier<T> hr, const Src<T>* src, int n, const StepArgs<T>* args, T dx, int L)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) point_source(hr, src[i], args->dt, dx, L);
}

// ---------------------------------------------------------------- multiresolution analysis

template <typename T> __device__ __forceinline__ void load4(const T* p, T (&out)[4])
{
    if constexpr (sizeof(T) == 4)
    {
        const float4 v = *reinterpret_cast<const float4*>(p);
        out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
    }
    else
    {
        const double2 a = reinterpret_cast<const double2*>(p)[0];
        const double2 b = reinterpret_cast<const double2*>(p)[1];
        out[0] = a.x; out[1] = a.y; out[2] = b.x; out[3] = b.y;
    }
}
template <typename T> __device__ __forceinline__ void store4(T* p, const T (&v)[4])
{
    if constexpr (sizeof(T) == 4)
    {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
    else
    {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
}

// Epsilon of the threshold for a parent at `level` (mra/encode_flow_kernel_mw.cu:45);
// levels below 4 use level 3's value, as the reference's single-block encode does
// (mra/encode_flow_kernel_single_block_mw.cu:48).
template <typename T> __device__ __forceinline__ T encode_eps(T eps, int L, int level)
{
    const int lv = (level >= 4) ? level : 3;
    return eps / (1 << (L - lv));
}

// Extra-significance threshold of a parent at `level` (mra/extra_significance_kernel.cu):
// eps_l * 2^(M_BAR+1) with M_BAR = 1.5 (the factor from k_step_begin).
template <typename T> __device__ __forceinline__ T extra_eps(T eps, int L, int level, const Scalars<T>* sc)
{
    const T eps_local = eps / (1 << (L - level));
    return eps_local * sc->xs_factor;
}

// scale_only_needed: the scale-only re-encode of the stage hierarchy (U*) produces the
// values RK stage 2 reads where a leaf's neighbour id is a significant parent (the leaf's
// neighbours across that face are finer). A neighbour id sits at level min(own leaf level,
// adjacent leaf's level), so never at a level coarser than the step's coarsest leaf
// (Scalars::min_leaf, set by k_tile_emit), and nothing else reads the stage hierarchy's
// parents. The scale-only kernels therefore skip parent levels below min_leaf, whose
// values nothing would read; every output is the same bits.

// Encode one parent (mra/encode_flow_kernel_{mw,hw}.cu), threshold it and OR in the
// children's significance (mra/regularisation_kernel.cu). FULL = false re-encodes scale
// coefficients of significant parents only (run_simulation.cu:573-588).
template <typename T, bool MW, bool FULL, bool PM = false>
__device__ __forceinline__ void encode_parent(const Hier<T>& hr, const Scalars<T>* sc, int L, int level, int idx, T eps,
                                              unsigned& n_done, const PropMask& pm = PropMask{})
{
    const int p = lvl_idx(level) + idx;
    // PM: a parent in a subtree the proposal leaves out keeps its flags and values
    const int anc = (PM && level >= pm.level) ? (idx >> (2 * (level - pm.level))) : -1;
    if (PM && anc >= 0 && pm_out(pm, anc)) return;
    const uint8_t f = hr.flags[p];
    const bool was_sig = (f & F_SIG) != 0;
    const int c = lvl_idx(level + 1) + 4 * idx;
    if (!FULL)
    {
        if (!was_sig) return;
        uint32_t mark = 0;
        if (hr.tag)
        {
            // keep-values decode: a parent made current in the last step whose four children
            // all stand unchanged in this one (frozen leaves, parents confirmed below) keeps
            // its scale coefficients, which this encode would compute again from the same
            // values; children are 4 consecutive slots, 16-byte aligned (lvl_idx(l) is a
            // multiple of 4 for l >= 1)
            const uint32_t now = sc->step_tag << 1;
            const uint4 ct = *reinterpret_cast<const uint4*>(hr.tag + c);
            if (ct.x == now && ct.y == now && ct.z == now && ct.w == now && (hr.tag[p] >> 1) == sc->step_tag - 1u)
            {
                hr.tag[p] = now;
                return;
            }
            mark = now | 1u;
        }
#pragma unroll
        for (int fld = 0; fld < 3; ++fld)
        {
            if (MW)
            {
                T k[3][4];
                load4(hr.s[fld][0] + c, k[0]); load4(hr.s[fld][1] + c, k[1]); load4(hr.s[fld][2] + c, k[2]);
                T s[3];
                mw_encode_scale(k, s);
                hr.s[fld][0][p] = s[0]; hr.s[fld][1][p] = s[1]; hr.s[fld][2][p] = s[2];
            }
            else
            {
                T k[4];
                load4(hr.s[fld][0] + c, k);
                hr.s[fld][0][p] = hw_scale(k);
            }
        }
        if (mark) hr.tag[p] = mark;
        ++n_done;
        return;
    }
    uint8_t nf = f & F_PRE;
    if (was_sig)
    {
        nf |= F_ENC;
        const T mx[3] = {fmax(T(1.0), sc->max_eta), fmax(T(1.0), sc->max_qx), fmax(T(1.0), sc->max_qx)};
        T nd = T(0.0);
#pragma unroll
        for (int fld = 0; fld < 3; ++fld)
        {
            if (MW)
            {
                T k[3][4];
                load4(hr.s[fld][0] + c, k[0]); load4(hr.s[fld][1] + c, k[1]); load4(hr.s[fld][2] + c, k[2]);
                T s[3];
                mw_encode_scale(k, s);
                hr.s[fld][0][p] = s[0]; hr.s[fld][1][p] = s[1]; hr.s[fld][2][p] = s[2];
                T d[3][3];
                mw_encode_details(k, d);
                nd = fmax(nd, mw_detail_max(d) / mx[fld]);
            }
            else
            {
                T k[4];
                load4(hr.s[fld][0] + c, k);
                hr.s[fld][0][p] = hw_scale(k);
                const T a = hw_alpha(k), b = hw_beta(k), g = hw_gamma(k);
                T m1 = fmax(fabs(a), fabs(b));
                m1 = fmax(fabs(g), m1);
                nd = fmax(nd, m1 / mx[fld]);
            }
        }
        if (nd >= encode_eps(eps, L, level) || (f & F_PRE)) nf |= F_SIG;
        if (level <= L - 2 && nd >= extra_eps(eps, L, level, sc)) nf |= F_XS;
        if (!(nf & F_SIG) && level <= L - 2)
        {
            const uint32_t ch = *reinterpret_cast<const uint32_t*>(hr.flags + c);
            if (ch & 0x01010101u) nf |= F_SIG;
        }
        ++n_done;
    }
    if (nf != f) hr.flags[p] = nf;   // most large-level parents keep their flags
}

// Small levels are processed in bands of up to kBandDepth levels, one CTA per node of the
// band's top level `lo`; the CTA's nodes at level l are (blockIdx.x << 2(l - lo)) + k for
// k < 4^(l - lo), and __syncthreads orders one level's global writes before the next
// level reads them. A band replaces up to five launches whose small grids are pure launch
// latency; it pays for that with serial per-level latency inside each CTA, so only levels
// up to kBandMaxLevel (at most 4^5 CTAs: one wave) are banded and larger levels get one
// launch each (k_encode_level / k_decode_level).
constexpr int kBandDepth = 5;
constexpr int kBandMaxLevel = 9;

// One level of parents (levels above kBandMaxLevel). FOLD: the level below it (level + 1)
// is sparse, and each thread first encodes its own parent's children there that need it
// (significant ones; FULL also clears the stale flag bits of the others, as k_level_sparse
// does) before the parent itself: a child's data is touched by its parent's thread only,
// and the sparse level needs no launch (and no scan of its flags) of its own.
template <typename T, bool MW, bool FULL, bool FOLD = false, bool PM = false>
__device__ __forceinline__ void k_encode_level_body(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps,
                                                                         PropMask pm = PropMask{})
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = idx < (1 << (2 * level));
    unsigned done = 0;
    // FOLD: up to four children (level + 1) first, then the parent, through one call site of
    // encode_parent (one inlined copy keeps the plain kernel's register count and occupancy)
    const bool fold = FOLD && in && (FULL || sc->min_leaf <= level + 1);   // see scale_only_needed
    const int cb = 4 * idx, cfirst = lvl_idx(level + 1);
    const uint32_t cw = fold ? *reinterpret_cast<const uint32_t*>(hr.flags + cfirst + cb) : 0u;
#pragma unroll 1
    for (int j = (FOLD && cw) ? 0 : 4; j < 5; ++j)
    {
        bool go;
        int lv, id;
        if (j < 4)
        {
            const uint32_t f = (cw >> (8 * j)) & 0xffu;
            go = (f & F_SIG) != 0;
            const bool kept = PM && level + 1 >= pm.level && pm_out(pm, (cb + j) >> (2 * (level + 1 - pm.level)));
            if (FULL && !go && !kept && (f & ~(uint32_t)F_PRE)) hr.flags[cfirst + cb + j] = (uint8_t)(f & F_PRE);
            lv = level + 1;
            id = cb + j;
        }
        else
        {
            go = in && (FULL || sc->min_leaf <= level);
            lv = level;
            id = idx;
        }
        if (go) encode_parent<T, MW, FULL, PM>(hr, sc, L, lv, id, eps, done, pm);
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, done);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(FULL ? &sc->enc : &sc->enc2, (unsigned long long)tot);
}
template <typename T, bool MW, bool FULL, bool FOLD = false, bool PM = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_encode_level(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps,
                                                                         PropMask pm = PropMask{})
{
    k_encode_level_body<T, MW, FULL, FOLD, PM>(hr, sc, L, level, eps, pm);
}

// One field of one significant parent's encode: its scale coefficients (stored) and, for
// FULL, the normalised maximum |detail| of that field (returned; 0 otherwise). The same
// helper calls in the same order as one field of encode_parent.
template <typename T, bool MW, bool FULL>
__device__ __forceinline__ T encode_field(const Hier<T>& hr, const Scalars<T>* sc, int level, int idx, int fld)
{
    const int p = lvl_idx(level) + idx;
    const int c = lvl_idx(level + 1) + 4 * idx;
    // the field's arrays, chosen without indexing the parameter block by a runtime value
    T* const a0 = fld == 0 ? hr.s[0][0] : fld == 1 ? hr.s[1][0] : hr.s[2][0];
    T* const a1 = fld == 0 ? hr.s[0][1] : fld == 1 ? hr.s[1][1] : hr.s[2][1];
    T* const a2 = fld == 0 ? hr.s[0][2] : fld == 1 ? hr.s[1][2] : hr.s[2][2];
    T nd = T(0.0);
    if (MW)
    {
        T k[3][4];
        load4(a0 + c, k[0]); load4(a1 + c, k[1]); load4(a2 + c, k[2]);
        T s[3];
        mw_encode_scale(k, s);
        a0[p] = s[0]; a1[p] = s[1]; a2[p] = s[2];
        if (FULL)
        {
            const T mx = fld == 0 ? fmax(T(1.0), sc->max_eta) : fmax(T(1.0), sc->max_qx);
            T d[3][3];
            mw_encode_details(k, d);
            nd = mw_detail_max(d) / mx;
        }
    }
    else
    {
        T k[4];
        load4(a0 + c, k);
        a0[p] = hw_scale(k);
        if (FULL)
        {
            const T mx = fld == 0 ? fmax(T(1.0), sc->max_eta) : fmax(T(1.0), sc->max_qx);
            const T a = hw_alpha(k), b = hw_beta(k), g = hw_gamma(k);
            T m1 = fmax(fabs(a), fabs(b));
            m1 = fmax(fabs(g), m1);
            nd = m1 / mx;
        }
    }
    return nd;
}

// Encode (FULL: + threshold + regularise; else scale-only re-encode) levels
// lo + depth - 1 .. lo bottom-up (mra/encode_flow.cu, mra/regularisation.cu). One thread per
// parent and field (the fields of a parent are independent; one thread doing them in turn
// waits on three dependent round trips, as a field's stores may alias the next one's
// loads); the fields' detail norms meet in shared memory and are combined in field order,
// as encode_parent combines them, before the flags.
template <typename T, bool MW, bool FULL>
__device__ __forceinline__ void k_encode_band_body(Hier<T> hr, Scalars<T>* sc, int L, int lo, int depth, T eps,
                                                     PropMask pm = PropMask{})
{
    if (!FULL && sc->min_leaf > lo + depth - 1) return;   // see scale_only_needed
    if (band_left_out(pm, lo)) return;
    static_assert(kBandDepth <= 5, "a band level has at most 4^(kBandDepth - 1) <= 256 parents");
    __shared__ T s_nd[3][256];
    unsigned done = 0;
    for (int l = lo + depth - 1; l >= lo; --l)
    {
        const int sh = 2 * (l - lo), n = 1 << sh, base = (int)blockIdx.x << sh, first = lvl_idx(l) + base;
        for (int t = threadIdx.x; t < 3 * n; t += blockDim.x)
        {
            const int fld = t >> sh, j = t & (n - 1);
            if (!(hr.flags[first + j] & F_SIG)) continue;
            s_nd[fld][j] = encode_field<T, MW, FULL>(hr, sc, l, base + j, fld);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x)
        {
            const uint8_t f = hr.flags[first + j];
            const bool was_sig = (f & F_SIG) != 0;
            if (was_sig) ++done;
            if (!FULL) continue;
            uint8_t nf = f & F_PRE;
            if (was_sig)
            {
                nf |= F_ENC;
                T nd = T(0.0);
                nd = fmax(nd, s_nd[0][j]);
                nd = fmax(nd, s_nd[1][j]);
                nd = fmax(nd, s_nd[2][j]);
                if (nd >= encode_eps(eps, L, l) || (f & F_PRE)) nf |= F_SIG;
                if (l <= L - 2 && nd >= extra_eps(eps, L, l, sc)) nf |= F_XS;
                if (!(nf & F_SIG) && l <= L - 2)
                {
                    const uint32_t ch = *reinterpret_cast<const uint32_t*>(hr.flags + lvl_idx(l + 1) + 4 * (base + j));
                    if (ch & 0x01010101u) nf |= F_SIG;
                }
            }
            if (nf != f) hr.flags[first + j] = nf;
        }
        __syncthreads();
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, done);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(FULL ? &sc->enc : &sc->enc2, (unsigned long long)tot);
}
template <typename T, bool MW, bool FULL>
__global__ void __launch_bounds__(256) k_encode_band(Hier<T> hr, Scalars<T>* sc, int L, int lo, int depth, T eps,
                                                     PropMask pm = PropMask{})
{
    k_encode_band_body<T, MW, FULL>(hr, sc, L, lo, depth, eps, pm);
}

// Decode one significant parent into its four children (mra/decoding_kernel_{mw,hw}.cu)
// and apply extra significance (mra/extra_significance_kernel.cu: parents whose norm
// reaches eps_l * 2^(M_BAR+1) make all four children significant).
// The details of a parent encoded this step are recomputed here from its children,
// which no kernel has changed since the encode read them (encode runs bottom-up and
// decode top-down, so a level's children are overwritten only by this very decode);
// the result is bit-identical to the encode's and no detail arrays are stored. Parents
// made significant without being encoded have zero details and zero norm, as in the
// reference (mra/zero_details.cu).
// FLAGS = false: values only; the flags of the children are then set by k_extra_sig_level
// from F_XS, which the encode derived from the same details.
// keep (the keep-values decode, not in the reference): an encoded parent's children keep
// the values its encode read, which its decode would return up to rounding; only parents
// made significant without an encode (refined this step) are decoded, and an encoded
// parent's extra significance comes from F_XS.
template <typename T, bool MW, bool FLAGS = true, bool PM = false>
__device__ __forceinline__ void decode_parent(const Hier<T>& hr, const Scalars<T>* sc, int L, int level, int idx, T eps,
                                              unsigned& n_done, const PropMask& pm = PropMask{}, bool keep = false)
{
    const int p = lvl_idx(level) + idx;
    // PM: the children of a parent in a subtree the proposal leaves out keep their values
    if (PM && level >= pm.level && pm_out(pm, idx >> (2 * (level - pm.level)))) return;
    const uint8_t f = hr.flags[p];
    if (!(f & F_SIG)) return;
    const bool enc = (f & F_ENC) != 0;
    const int c = lvl_idx(level + 1) + 4 * idx;
    if (keep && enc)
    {
        ++n_done;
        if (FLAGS && level <= L - 2 && (f & F_XS)) *reinterpret_cast<uint32_t*>(hr.flags + c) |= 0x01010101u;
        return;
    }
    const T mx[3] = {fmax(T(1.0), sc->max_eta), fmax(T(1.0), sc->max_qx), fmax(T(1.0), sc->max_qx)};
    T nd = T(0.0);
#pragma unroll
    for (int fld = 0; fld < 3; ++fld)
    {
        if (MW)
        {
            const T s[3] = {hr.s[fld][0][p], hr.s[fld][1][p], hr.s[fld][2][p]};
            T d[3][3];
            if (enc)
            {
                T k[3][4];
                load4(hr.s[fld][0] + c, k[0]); load4(hr.s[fld][1] + c, k[1]); load4(hr.s[fld][2] + c, k[2]);
                mw_encode_details(k, d);
                nd = fmax(nd, mw_detail_max(d) / mx[fld]);
            }
            else
            {
#pragma unroll
                for (int t = 0; t < 3; ++t)
#pragma unroll
                    for (int m = 0; m < 3; ++m) d[t][m] = T(0.0);
            }
            T k[3][4];
            mw_decode(s, d, k);
            store4(hr.s[fld][0] + c, k[0]); store4(hr.s[fld][1] + c, k[1]); store4(hr.s[fld][2] + c, k[2]);
        }
        else
        {
            const T u = hr.s[fld][0][p];
            T a = T(0.0), b = T(0.0), g = T(0.0);
            if (enc)
            {
                T k[4];
                load4(hr.s[fld][0] + c, k);
                a = hw_alpha(k); b = hw_beta(k); g = hw_gamma(k);
                T m1 = fmax(fabs(a), fabs(b));
                m1 = fmax(fabs(g), m1);
                nd = fmax(nd, m1 / mx[fld]);
            }
            T k[4];
            hw_decode(u, a, b, g, k);
            store4(hr.s[fld][0] + c, k);
        }
    }
    ++n_done;
    if (FLAGS && level <= L - 2)
    {
        if (nd >= extra_eps(eps, L, level, sc)) *reinterpret_cast<uint32_t*>(hr.flags + c) |= 0x01010101u;
    }
}

// First level on the root -> node path whose node is not significant (levels 0..Tl, the
// last being node `tcode` of level Tl); Tl + 1 if all are. Called by a whole warp: lane j
// loads level j's flag, so the loads are independent. Needs Tl + 1 <= 32.
__device__ __forceinline__ int path_leaf_level_warp(const uint8_t* flags, int Tl, int tcode)
{
    const int lane = threadIdx.x & 31;
    const bool nonsig = lane <= Tl && !(flags[lvl_idx(lane) + (tcode >> (2 * (Tl - lane)))] & F_SIG);
    const unsigned m = __ballot_sync(0xffffffffu, nonsig);
    return m ? __ffs(m) - 1 : Tl + 1;
}

// One field of one significant parent's decode: its four children (stored) from its scale
// coefficients and details (recomputed from the children for an encoded parent, zero
// otherwise); returns the normalised maximum |detail| of that field (0 when not encoded).
// The same helper calls in the same order as one field of decode_parent.
template <typename T, bool MW>
__device__ __forceinline__ T decode_field(const Hier<T>& hr, const Scalars<T>* sc, int level, int idx, int fld, bool enc)
{
    const int p = lvl_idx(level) + idx;
    const int c = lvl_idx(level + 1) + 4 * idx;
    // the field's arrays, chosen without indexing the parameter block by a runtime value
    T* const a0 = fld == 0 ? hr.s[0][0] : fld == 1 ? hr.s[1][0] : hr.s[2][0];
    T* const a1 = fld == 0 ? hr.s[0][1] : fld == 1 ? hr.s[1][1] : hr.s[2][1];
    T* const a2 = fld == 0 ? hr.s[0][2] : fld == 1 ? hr.s[1][2] : hr.s[2][2];
    T nd = T(0.0);
    if (MW)
    {
        const T s[3] = {a0[p], a1[p], a2[p]};
        T d[3][3];
        if (enc)
        {
            const T mx = fld == 0 ? fmax(T(1.0), sc->max_eta) : fmax(T(1.0), sc->max_qx);
            T k[3][4];
            load4(a0 + c, k[0]); load4(a1 + c, k[1]); load4(a2 + c, k[2]);
            mw_encode_details(k, d);
            nd = mw_detail_max(d) / mx;
        }
        else
        {
#pragma unroll
            for (int t = 0; t < 3; ++t)
#pragma unroll
                for (int m = 0; m < 3; ++m) d[t][m] = T(0.0);
        }
        T k[3][4];
        mw_decode(s, d, k);
        store4(a0 + c, k[0]); store4(a1 + c, k[1]); store4(a2 + c, k[2]);
    }
    else
    {
        const T u = a0[p];
        T a = T(0.0), b = T(0.0), g = T(0.0);
        if (enc)
        {
            const T mx = fld == 0 ? fmax(T(1.0), sc->max_eta) : fmax(T(1.0), sc->max_qx);
            T k[4];
            load4(a0 + c, k);
            a = hw_alpha(k); b = hw_beta(k); g = hw_gamma(k);
            T m1 = fmax(fabs(a), fabs(b));
            m1 = fmax(fabs(g), m1);
            nd = m1 / mx;
        }
        T k[4];
        hw_decode(u, a, b, g, k);
        store4(a0 + c, k);
    }
    return nd;
}

// Decode levels lo .. lo + depth - 1 top-down (mra/decoding.cu, mra/extra_significance.cu),
// one thread per parent and field (see k_encode_band); the fields' detail norms are combined
// in field order, as decode_parent combines them, for extra significance.
// keep: the keep-values decode (decode_parent): encoded parents are not decoded, and their
// extra significance comes from F_XS.
template <typename T, bool MW>
__device__ __forceinline__ void k_decode_band_body(Hier<T> hr, Scalars<T>* sc, int L, int lo, int depth, T eps,
                                                                                 PropMask pm = PropMask{}, bool keep = false)
{
    if (band_left_out(pm, lo)) return;
    static_assert(kBandDepth <= 5, "a band level has at most 4^(kBandDepth - 1) <= 256 parents");
    __shared__ T s_nd[3][256];
    unsigned done = 0;
    for (int l = lo; l < lo + depth; ++l)
    {
        const int sh = 2 * (l - lo), n = 1 << sh, base = (int)blockIdx.x << sh, first = lvl_idx(l) + base;
        for (int t = threadIdx.x; t < 3 * n; t += blockDim.x)
        {
            const int fld = t >> sh, j = t & (n - 1);
            const uint8_t f = hr.flags[first + j];
            if (!(f & F_SIG) || (keep && (f & F_ENC))) continue;
            s_nd[fld][j] = decode_field<T, MW>(hr, sc, l, base + j, fld, (f & F_ENC) != 0);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x)
        {
            const uint8_t f = hr.flags[first + j];
            if (!(f & F_SIG)) continue;
            ++done;
            if (l <= L - 2)
            {
                bool xs;
                if (keep && (f & F_ENC)) xs = (f & F_XS) != 0;
                else
                {
                    T nd = T(0.0);
                    nd = fmax(nd, s_nd[0][j]);
                    nd = fmax(nd, s_nd[1][j]);
                    nd = fmax(nd, s_nd[2][j]);
                    xs = nd >= extra_eps(eps, L, l, sc);
                }
                if (xs) *reinterpret_cast<uint32_t*>(hr.flags + lvl_idx(l + 1) + 4 * (base + j)) |= 0x01010101u;
            }
        }
        __syncthreads();
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, done);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&sc->dec, (unsigned long long)tot);
}
template <typename T, bool MW>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_decode_band(Hier<T> hr, Scalars<T>* sc, int L, int lo, int depth, T eps,
                                                                                 PropMask pm = PropMask{}, bool keep = false)
{
    k_decode_band_body<T, MW>(hr, sc, L, lo, depth, eps, pm, keep);
}

// Extra significance of one level of parents from their flags (levels above kBandMaxLevel,
// level <= L - 2): a significant parent makes its children significant when its encode set
// F_XS, or, not encoded (zero details, zero norm), when the threshold is not above zero.
// Four parents per thread (one aligned flag word). The flags are final after this, so the
// leaf topology can run beside the value decode of the level (k_decode_level).
template <typename T>
__device__ __forceinline__ void k_extra_sig_level_body(uint8_t* flags, const Scalars<T>* sc, int L, int level, T eps)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= (1 << (2 * level - 2))) return;
    const uint32_t word = *reinterpret_cast<const uint32_t*>(flags + lvl_idx(level) + 4 * w);
    if (!(word & (0x01010101u * F_SIG))) return;
    const bool zero_norm_extra = T(0.0) >= extra_eps(eps, L, level, sc);
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const uint32_t f = (word >> (8 * j)) & 0xffu;
        if (!(f & F_SIG)) continue;
        const bool xs = (f & F_ENC) ? (f & F_XS) != 0 : zero_norm_extra;
        if (xs) *reinterpret_cast<uint32_t*>(flags + lvl_idx(level + 1) + 4 * (4 * w + j)) |= 0x01010101u;
    }
}
template <typename T>
__global__ void __launch_bounds__(256) k_extra_sig_level(uint8_t* flags, const Scalars<T>* sc, int L, int level, T eps)
{
    k_extra_sig_level_body<T>(flags, sc, L, level, eps);
}

// One level of parents (levels above kBandMaxLevel), values only (k_extra_sig_level set the
// children's flags).
template <typename T, bool MW, bool PM = false>
__device__ __forceinline__ void k_decode_level_body(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps,
                                                                         PropMask pm = PropMask{})
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned done = 0;
    if (idx < (1 << (2 * level))) decode_parent<T, MW, false, PM>(hr, sc, L, level, idx, eps, done, pm);
    const unsigned tot = __reduce_add_sync(0xffffffffu, done);
    if ((threadIdx.x & 31) == 0 && tot)
    {
        atomicAdd(&sc->dec, (unsigned long long)tot);
        atomicAdd(&sc->sig_level[level], tot);
    }
}
template <typename T, bool MW, bool PM = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) k_decode_level(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps,
                                                                         PropMask pm = PropMask{})
{
    k_decode_level_body<T, MW, PM>(hr, sc, L, level, eps, pm);
}

// Sparse form of one level (a level whose significant parents were few last step): a
// thread reads the flags of eight consecutive parents as one aligned 8-byte word
// (lvl_idx(level) is a multiple of 8 for level >= 2), finishes the parents that are not
// significant itself (FULL encode: clear their flag bits) and lists the significant ones
// in shared memory; the warp's lanes then take the listed parents in turn. A level of 4M
// parents with a handful significant costs 512K threads that read 8 bytes each instead of
// 4M threads. Op 0: FULL encode, 1: scale-only re-encode, 2: decode (values only, as
// k_decode_level; keep: the keep-values decode of decode_parent, where only the parents
// refined this step are listed and the encoded ones are just counted).
template <typename T, bool MW, int OP, bool PM = false>
__global__ void __launch_bounds__(256) k_level_sparse(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps,
                                                      PropMask pm = PropMask{}, bool keep = false)
{
    if (OP == 1 && sc->min_leaf > level) return;   // see scale_only_needed
    __shared__ int list[8][256];   // per warp: up to 32 lanes x 8 parents
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t first = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
    const int64_t np = (int64_t)1 << (2 * level);
    unsigned done = 0;
    uint32_t sig = 0;
    if (first < np)
    {
        const uint2 w = *reinterpret_cast<const uint2*>(hr.flags + lvl_idx(level) + first);
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            const uint32_t f = ((j < 4 ? w.x : w.y) >> (8 * (j & 3))) & 0xffu;
            const bool kept = PM && level >= pm.level && pm_out(pm, (int)((first + j) >> (2 * (level - pm.level))));
            if (f & F_SIG)
            {
                if (OP == 2 && keep && (f & F_ENC)) done += kept ? 0u : 1u;
                else sig |= kept ? 0u : 1u << j;
            }
            // FULL encode of a parent that was not significant: only its flag changes (its
            // encode / extra-significance bits from the last step clear, the preflag stays)
            else if (OP == 0 && !kept && (f & ~(uint32_t)F_PRE)) hr.flags[lvl_idx(level) + first + j] = (uint8_t)(f & F_PRE);
        }
    }
    const int c = __popc(sig);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int k = incl - c;
    for (int j = 0; j < 8; ++j)
        if (sig & (1u << j)) list[warp][k++] = (int)(first + j);
    __syncwarp();
    for (int e = lane; e < total; e += 32)
    {
        const int idx = list[warp][e];
        if (OP == 0) encode_parent<T, MW, true, PM>(hr, sc, L, level, idx, eps, done, pm);
        else if (OP == 1) encode_parent<T, MW, false, PM>(hr, sc, L, level, idx, eps, done, pm);
        else decode_parent<T, MW, false, PM>(hr, sc, L, level, idx, eps, done, pm);
    }
    const unsigned tot = __reduce_add_sync(0xffffffffu, done);
    if (lane == 0 && tot)
    {
        if (OP == 0) atomicAdd(&sc->enc, (unsigned long long)tot);
        else if (OP == 1) atomicAdd(&sc->enc2, (unsigned long long)tot);
        else
        {
            atomicAdd(&sc->dec, (unsigned long long)tot);
            atomicAdd(&sc->sig_level[level], tot);
        }
    }
}

// Bed encoding of one level and preflagging (mra/encode_topography_kernel_{mw,hw}.cu).
template <typename T, bool MW>
__global__ void __launch_bounds__(256) k_topo_level(Hier<T> hr, Scalars<T>* sc, int L, int level, T eps)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (1 << (2 * level))) return;
    const int p = lvl_idx(level) + idx, c = lvl_idx(level + 1) + 4 * idx;
    const T eps_local = eps / (1 << (L - level));
    const T mz = fmax(T(1.0), sc->max_z);
    T mx;
    if (MW)
    {
        T k[3][4];
        load4(hr.s[3][0] + c, k[0]); load4(hr.s[3][1] + c, k[1]); load4(hr.s[3][2] + c, k[2]);
        T s[3];
        mw_encode_scale(k, s);
        hr.s[3][0][p] = s[0]; hr.s[3][1][p] = s[1]; hr.s[3][2][p] = s[2];
        T d[3][3];
        mw_encode_details(k, d);
        mx = mw_detail_max(d);
    }
    else
    {
        T k[4];
        load4(hr.s[3][0] + c, k);
        const T a = hw_alpha(k), b = hw_beta(k), g = hw_gamma(k);
        hr.s[3][0][p] = hw_scale(k);
        T m1 = fmax(fabs(a), fabs(b));
        mx = fmax(fabs(g), m1);
    }
    if ((mx / mz) >= eps_local) hr.flags[p] |= F_PRE;
}

// ---------------------------------------------------------------- leaf topology
//
// The significance flags are closed upwards (a significant node's parent is significant),
// so the leaves of the subtree below a significant node r are 1 + 3 x (number of
// significant nodes in that subtree). Tiles are the nodes of level T = L - D; each tile
// counts its leaves, an exclusive scan gives output offsets, and each tile then writes
// its leaves in Z order (depth-first order of the quadtree, as the reference's
// traversal + compaction produce: mra/traverse_tree_of_sig_details.cu,
// neighbours/compaction.cu).

// First level j in [j0, lim) whose node on the path to finest cell `tc` is not
// significant; lim if none. The (at most 16) flag loads are issued independently.
__device__ __forceinline__ int first_nonsig_level(const uint8_t* flags, int L, int tc, int j0, int lim)
{
    unsigned nonsig = 0;
#pragma unroll
    for (int t = 0; t < 16; ++t)
    {
        const int j = j0 + t;
        if (j < lim && !(flags[lvl_idx(j) + (tc >> (2 * (L - j)))] & F_SIG)) nonsig |= 1u << t;
    }
    return nonsig ? j0 + __ffs(nonsig) - 1 : lim;
}

// Morton codes hold x in the even bits and y in the odd bits. Arithmetic on one
// coordinate of a code ("dilated integers") needs no de-interleaving: with m the mask of
// that coordinate's bits, (a | ~m) + b carries through the other coordinate's bits.
constexpr unsigned kXBits = 0x55555555u, kYBits = 0xAAAAAAAAu;
__device__ __forceinline__ unsigned dil_add(unsigned a, unsigned b, unsigned m) { return ((a | ~m) + b) & m; }
__device__ __forceinline__ unsigned dil_sub(unsigned a, unsigned b, unsigned m) { return (a - b) & m; }

// Word w (0..84) of the flags of levels Tl+1 .. Tl+4 below tile root `tcode` (levels
// Tl+1..Tl+4 hold 1, 4, 16, 64 words): its level offset j (1..4) and global byte index.
// lvl_idx(l) is a multiple of 4 for l >= 1, so every word is aligned.
__device__ __forceinline__ int tile_flag_word(int Tl, int tcode, int w, int& j)
{
    j = 1 + (w >= 1) + (w >= 5) + (w >= 21);
    const int wbase = (j == 1) ? 0 : (j == 2) ? 1 : (j == 3) ? 5 : 21;
    return lvl_idx(Tl + j) + (tcode << (2 * j)) + 4 * (w - wbase);
}

// Leaves of tile `tcode` (node of level Tl = L - 5): 1 + 3 x (significant nodes of its
// subtree) when every node on its root path is significant; otherwise 1 for the first
// tile of the coarser leaf covering it (or its own non-significant root) and 0 for the
// others. Called by the whole block (256 threads); returns the count in every thread.
__device__ __forceinline__ int tile_leaf_count(const uint8_t* flags, int Tl, int tcode)
{
    static_assert(kTileDepth == 5, "the word layout of tile_flag_word assumes 4^5-cell tiles");
    const int k = path_leaf_level_warp(flags, Tl, tcode);  // every warp finds it
    if (k <= Tl) return (k == Tl || (tcode & ((1 << (2 * (Tl - k))) - 1)) == 0) ? 1 : 0;
    // significant nodes of the subtree: the root plus levels Tl+1 .. L-1 (85 flag words)
    int cnt = 0;
    if (threadIdx.x < 85)
    {
        int j;
        const uint32_t w = *reinterpret_cast<const uint32_t*>(flags + tile_flag_word(Tl, tcode, threadIdx.x, j));
        cnt = __popc(w & (0x01010101u * F_SIG));
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    __shared__ int s_cnt[3];
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 96) s_cnt[threadIdx.x >> 5] = cnt;
    __syncthreads();
    const int total = 1 + 3 * (1 + s_cnt[0] + s_cnt[1] + s_cnt[2]);
    __syncthreads();  // s_cnt may be reused by a later call
    return total;
}

// Tile leaf counts from final flags.
// static: the header is included by more than one translation unit of the library
static __device__ __forceinline__ void k_tile_count_body(const uint8_t* flags, int L, int32_t* counts)
{
    const int c = tile_leaf_count(flags, L - kTileDepth, (int)blockIdx.x);
    if (threadIdx.x == 0) counts[blockIdx.x] = c;
}
static __global__ void __launch_bounds__(kTileThreads) k_tile_count(const uint8_t* flags, int L, int32_t* counts)
{
    k_tile_count_body(flags, L, counts);
}

// Exclusive scan of n tile counts in one block of 1024 threads; total -> sc->n_leaves.
// Thread t owns a contiguous chunk (read as int4 when chunks are multiples of four; tile
// counts come in powers of four), warps scan their chunk sums with shuffles, and the 32 warp
// totals are scanned by one warp.
template <typename T>
__device__ __forceinline__ void k_tile_scan_body(int32_t* counts, int n, Scalars<T>* sc)
{
    __shared__ int32_t warp_sum[32];
    const int per = (n + 1023) / 1024;
    const int lo = min(n, (int)threadIdx.x * per), hi = min(n, lo + per);
    const bool vec = (per % 4) == 0;
    int32_t s = 0;
    if (vec)
        for (int i = lo; i < hi; i += 4)
        {
            const int4 v = *reinterpret_cast<const int4*>(counts + i);
            s += v.x + v.y + v.z + v.w;
        }
    else
        for (int i = lo; i < hi; ++i) s += counts[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sum[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        int32_t t = warp_sum[lane], ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int32_t v = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += v;
        }
        warp_sum[lane] = ti - t;   // exclusive prefix of the warp totals
        if (lane == 31)
        {
            sc->n_prev = sc->n_leaves;
            sc->n_leaves = ti;
        }
    }
    __syncthreads();
    int32_t run = warp_sum[w] + incl - s;   // exclusive prefix of this thread's chunk
    if (vec)
        for (int i = lo; i < hi; i += 4)
        {
            int4 v = *reinterpret_cast<const int4*>(counts + i);
            const int4 c = v;
            v.x = run; run += c.x;
            v.y = run; run += c.y;
            v.z = run; run += c.z;
            v.w = run; run += c.w;
            *reinterpret_cast<int4*>(counts + i) = v;
        }
    else
        for (int i = lo; i < hi; ++i)
        {
            const int32_t c = counts[i];
            counts[i] = run;
            run += c;
        }
}
template <typename T>
__global__ void __launch_bounds__(1024) k_tile_scan(int32_t* counts, int n, Scalars<T>* sc)
{
    k_tile_scan_body<T>(counts, n, sc);
}

// Neighbour of a leaf (level l, finest reference cell code `ref`) across the finest cell
// (tx, ty), direction d (N, E, S, W): the ancestor of the leaf containing that cell at
// min(l, its level) (neighbours/find_neighbours.cu:100-108); -1 and level l across the
// DEM or mesh border (north/east from the leaf's north-east finest cell, south/west from
// its south-west one: neighbours/find_neighbours.cu:51-428, neighbours/compaction.cu:109-151).
// All shared ancestors of the leaf and that cell are significant, so the search starts
// at the first level where their paths differ.
__device__ __forceinline__ void leaf_neighbour(const uint8_t* flags, int L, int M, int xsz, int ysz, int act, int l,
                                               int d, int32_t& id, uint8_t& lv)
{
    const int code = act - lvl_idx(l);
    const int x = compact(code), y = compact(code >> 1);
    const int s = 1 << (L - l);
    const int x0 = x * s, y0 = y * s, xe = x0 + s - 1, ye = y0 + s - 1;
    const bool border = (d == 0) ? ((ye == M - 1 || ye == ysz - 1) && ye != 0)
                      : (d == 1) ? ((xe == M - 1 || xe == xsz - 1) && xe != 0)
                      : (d == 2) ? (y0 == 0) : (x0 == 0);
    if (border) { id = -1; lv = (uint8_t)l; return; }
    const int tx = (d == 0) ? xe : (d == 1) ? xe + 1 : (d == 2) ? x0 : x0 - 1;
    const int ty = (d == 0) ? ye + 1 : (d == 1) ? ye : (d == 2) ? y0 - 1 : y0;
    const int tc = morton(tx, ty);
    const int b = 31 - __clz(tc ^ morton(x0, y0));
    const int j0 = max(0, L - (b >> 1));
    const int m = first_nonsig_level(flags, L, tc, j0, l);
    id = lvl_idx(m) + (tc >> (2 * (L - m)));
    lv = (uint8_t)m;
}

// A tile holding one leaf (the tile's root or the first tile of a coarser leaf): threads
// 0..3 of the block find one neighbour each.
// Position pos of the leaf list gets leaf `act`; with lf.same, whether it held that leaf in
// the last step (n_prev leaves).
template <typename T>
__device__ __forceinline__ void put_act(const Leaves<T>& lf, int pos, int act, const int32_t* n_prev)
{
    if (lf.same) lf.same[pos] = (pos < *n_prev && lf.act[pos] == act) ? 1 : 0;
    lf.act[pos] = act;
}

template <typename T, bool NBL>
__device__ __forceinline__ void emit_single_leaf(const Leaves<T>& lf, const uint8_t* flags, int L, int M, int xsz,
                                                 int ysz, int pos, int act, int l, const int32_t* n_prev)
{
    const int d = threadIdx.x;
    if (d >= 4) return;
    if (d == 0) { put_act(lf, pos, act, n_prev); lf.lvl[pos] = (uint8_t)l; }
    int32_t id;
    uint8_t lv;
    leaf_neighbour(flags, L, M, xsz, ysz, act, l, d, id, lv);
    lf.nb[d][pos] = id;
    if (NBL) lf.nbl[d][pos] = lv;
}

// Leaves of one tile in Z order with their neighbours. The tile's subtree flags are
// copied to shared memory; every finest cell of the tile gets the level of the leaf that
// contains it, and so does the ring of cells just outside the tile (searches in the
// global flags); leaf starts are ranked with popcounts; then thread r writes the leaf of
// rank r (coalesced): the neighbour across a face is the ancestor of the neighbouring
// finest cell at min(own level, that cell's leaf level) (neighbours/find_neighbours.cu:
// 100-108), -1 across the DEM or mesh border (neighbours/find_neighbours.cu:51-428).
// Neighbouring cells are found by dilated-integer steps on the leaf's Morton code.
// NBL: also write the neighbours' levels (lf.nbl), which level_of(id) gives wherever the id
// is not -1 (-1: the leaf's own level).
template <typename T, bool NBL>
__device__ __forceinline__ void k_tile_emit_body(Leaves<T> lf, const uint8_t* flags, const int32_t* offsets,
                                                            int L, int M, int xsz, int ysz, int32_t* min_leaf,
                                                            const int32_t* n_prev)
{
    constexpr int D = kTileDepth, kCells = 1 << (2 * D);
    const int Tl = L - D;
    const int tcode = blockIdx.x;
    const int off = offsets[tcode];
    // subtree flags at lvl_idx(j) + local index (j = 1..4); lvl_idx(D) bytes
    __shared__ __align__(4) uint8_t sflag[((1 << (2 * D)) - 1) / 3 + 3];
    // leaf level of each node of level L - 1 (four finest cells), tile-local Morton order;
    // L when the node is significant (its four cells are leaves of level L)
    __shared__ uint8_t node_lvl[kCells / 4];
    __shared__ uint16_t start_of[kCells];             // tile-local start cell of the leaf of each rank
    __shared__ int32_t warp_starts[kTileThreads / 32];
    __shared__ int32_t warp_min[kTileThreads / 32];
    // leaf levels of the cells just outside the tile (N, E, S, W), indexed by the dilated
    // tile-local coordinate along the side (x bits for N/S, y bits shifted down for E/W)
    __shared__ uint8_t halo[4][(kXBits & (kCells - 1)) + 1];
    const int k = path_leaf_level_warp(flags, Tl, tcode);  // levels 0..Tl, every warp
    if (k < Tl)
    {
        if ((tcode & ((1 << (2 * (Tl - k))) - 1)) == 0)
        {
            if (min_leaf && threadIdx.x == 0) atomicMin(min_leaf, k);
            emit_single_leaf<T, NBL>(lf, flags, L, M, xsz, ysz, off, lvl_idx(k) + (tcode >> (2 * (Tl - k))), k, n_prev);
        }
        return;
    }
    if (k == Tl)
    {
        if (min_leaf && threadIdx.x == 0) atomicMin(min_leaf, Tl);
        emit_single_leaf<T, NBL>(lf, flags, L, M, xsz, ysz, off, lvl_idx(Tl) + tcode, Tl, n_prev);
        return;
    }
    if (threadIdx.x < 85)
    {
        int j;
        const int g = tile_flag_word(Tl, tcode, threadIdx.x, j);
        const int local = g - lvl_idx(Tl + j) - (tcode << (2 * j));
        *reinterpret_cast<uint32_t*>(sflag + lvl_idx(j) + local) =
            *reinterpret_cast<const uint32_t*>(flags + g) & (0x01010101u * F_SIG);
    }
    const unsigned tbase = (unsigned)tcode << (2 * D);   // finest Morton code of the tile's first cell
    static_assert((1 << D) == 32, "one warp per side of the tile");
    if (threadIdx.x < 4 * 32)
    {
        // warp `side` (N, E, S, W) takes the adjacent tile; lane i its i-th cell along the
        // shared edge. The neighbouring tile's root path decides for all lanes at once unless
        // that root is significant; then each lane reads its cell's four in-tile levels.
        const int side = threadIdx.x >> 5, i = threadIdx.x & 31;
        const int tx = compact(tcode), ty = compact(tcode >> 1), nt = 1 << Tl;
        const int nx = tx + (side == 1) - (side == 3), ny = ty + (side == 0) - (side == 2);
        uint8_t lev = 0;                               // cells outside the mesh are never looked up
        if (nx >= 0 && ny >= 0 && nx < nt && ny < nt)  // uniform in the warp
        {
            const int ncode = morton(nx, ny);
            const int kn = path_leaf_level_warp(flags, Tl, ncode);
            if (kn <= Tl) lev = (uint8_t)kn;
            else
            {
                const int lx = (side == 0 || side == 2) ? i : (side == 1 ? 0 : 31);
                const int ly = (side == 1 || side == 3) ? i : (side == 0 ? 0 : 31);
                const int lc = morton(lx, ly);
                int l = L;
#pragma unroll
                for (int j = D - 1; j >= 1; --j)
                    if (!(flags[lvl_idx(Tl + j) + (ncode << (2 * j)) + (lc >> (2 * (D - j)))] & F_SIG)) l = Tl + j;
                lev = (uint8_t)l;
            }
        }
        halo[side][dilate(i)] = lev;
    }
    __syncthreads();
    // one node q of level L - 1 per thread: its leaf level is the first level below the
    // (significant) root whose node on q's path is not significant, or L when q itself is
    // significant; its cells hold 4 leaf starts (level L), 1 (a leaf of level lev <= L - 1
    // starting at q's first cell) or none. A block scan of those counts ranks the leaves.
    static_assert(kTileThreads == kCells / 4, "one thread per node of level L - 1");
    const int q = threadIdx.x;
    int qlev = L;
#pragma unroll
    for (int j = D - 1; j >= 1; --j)
        if (!sflag[lvl_idx(j) + (q >> (2 * (D - 1 - j)))]) qlev = Tl + j;
    node_lvl[q] = (uint8_t)qlev;
    const int nstart = (qlev == L) ? 4 : (((4 * q) & ((1 << (2 * (L - qlev))) - 1)) == 0 ? 1 : 0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = nstart;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int wmin = __reduce_min_sync(0xffffffffu, qlev);
    if (lane == 31) warp_starts[warp] = incl;
    if (lane == 0) warp_min[warp] = wmin;
    __syncthreads();
    int rank = incl - nstart, total = 0;
#pragma unroll
    for (int w = 0; w < kTileThreads / 32; ++w)
    {
        const int c = warp_starts[w];
        rank += (w < warp) ? c : 0;
        total += c;
    }
    // the tree's coarsest leaf level (Scalars::min_leaf), one atomic per tile that lowers it
    if (min_leaf && threadIdx.x == 0)
    {
        int bmin = warp_min[0];
#pragma unroll
        for (int w = 1; w < kTileThreads / 32; ++w) bmin = min(bmin, warp_min[w]);
        if (bmin < *min_leaf) atomicMin(min_leaf, bmin);
    }
    if (nstart == 4)
    {
#pragma unroll
        for (int i = 0; i < 4; ++i) start_of[rank + i] = (uint16_t)(4 * q + i);
    }
    else if (nstart) start_of[rank] = (uint16_t)(4 * q);
    __syncthreads();
    const unsigned lmask = kCells - 1;
    // dilated coordinates of the mesh's last row/column and of the DEM's
    const unsigned mesh_x = kXBits & ((1u << (2 * L)) - 1u), mesh_y = mesh_x << 1;
    const unsigned dem_x = (unsigned)dilate(xsz - 1), dem_y = (unsigned)dilate(ysz - 1) << 1;
    for (int r = threadIdx.x; r < total; r += blockDim.x)
    {
        const int c = start_of[r];
        const int lev = node_lvl[c >> 2];
        const int sh = 2 * (L - lev);
        const unsigned gc = tbase + (unsigned)c;       // finest code of the leaf's south-west cell
        const int pos = off + r;
        put_act(lf, pos, lvl_idx(lev) + (int)(gc >> sh), n_prev);
        lf.lvl[pos] = (uint8_t)lev;
        const unsigned X0 = gc & kXBits, Y0 = gc & kYBits;            // dilated x0, y0
        const unsigned span = (1u << sh) - 1u;                         // dilated (size - 1) in both
        const unsigned Xe = X0 | (span & kXBits), Ye = Y0 | (span & kYBits);
        // target finest cell per direction: N (xe, ye+1), E (xe+1, ye), S (x0, y0-1), W (x0-1, y0)
        const bool border[4] = {(Ye == mesh_y || Ye == dem_y) && Ye != 0, (Xe == mesh_x || Xe == dem_x) && Xe != 0,
                                Y0 == 0, X0 == 0};
        const unsigned tc[4] = {Xe | dil_add(Ye, 2u, kYBits), dil_add(Xe, 1u, kXBits) | Ye, X0 | dil_sub(Y0, 2u, kYBits),
                                dil_sub(X0, 1u, kXBits) | Y0};
#pragma unroll
        for (int d = 0; d < 4; ++d)
        {
            int32_t id = -1;
            int lv = lev;
            if (!border[d])
            {
                const unsigned t = tc[d];
                int lt;
                if ((t >> (2 * D)) == (unsigned)tcode) lt = node_lvl[(t & lmask) >> 2];
                else if (d == 0 || d == 2) lt = halo[d][t & lmask & kXBits];
                else lt = halo[d][(t & lmask & kYBits) >> 1];
                lv = lev < lt ? lev : lt;
                id = lvl_idx(lv) + (int)(t >> (2 * (L - lv)));
            }
            lf.nb[d][pos] = id;
            if (NBL) lf.nbl[d][pos] = (uint8_t)lv;
        }
    }
}
template <typename T, bool NBL>
__global__ void __launch_bounds__(kTileThreads, 8) k_tile_emit(Leaves<T> lf, const uint8_t* flags, const int32_t* offsets,
                                                            int L, int M, int xsz, int ysz, int32_t* min_leaf,
                                                            const int32_t* n_prev)
{
    k_tile_emit_body<T, NBL>(lf, flags, offsets, L, M, xsz, ysz, min_leaf, n_prev);
}

// Initial leaf list: every finest cell, in Z order.
template <typename T> __global__ void k_init_leaves(Leaves<T> lf, int L, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        lf.act[i] = lvl_idx(L) + i;
        lf.lvl[i] = (uint8_t)L;
    }
}

} // namespace mw
