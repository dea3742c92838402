// Learned refinement proposal: a small per-coarse-cell MLP on the 5th-generation tensor cores.
//
// No counterpart in the reference (al0vya/gpu-mwdg2 encodes every previously significant
// parent each step, mra/encode_flow.cu:14-92, and decodes every significant one,
// mra/decoding.cu:3-67). Here a coarse level C (= L - 3) is chosen; the subtree under
// each node of level C + 1 is proposed for encoding and decoding, or not, by an MLP that
// looks at the 3 x 3 neighbourhood of its parent (a node of level C):
//
//   input   128 features per coarse cell: for the cell and its eight neighbours (level C,
//           or the coarser leaf holding them), h, qx, qy and the bed z relative to the
//           centre's, each with its x and y slope modes (9 x 12 = 108), the four
//           children's activity bits of the last step (112), a constant 1 (113), zeros
//   layers  128 -> 64 -> 64 -> 64 -> 4, ReLU between, BF16 weights and activations,
//           FP32 accumulation in tensor memory
//   output  4 logits: the children whose subtrees need their encode and decode this step
//
// A child subtree is "active" in a step when one of its leaves was updated by the RK stages
// (not dry) or its significance flags at the end of the step differ from the last step's;
// the step after, the encode must revisit it. The label of a training sample is the
// activity of the step the features precede.
//
// Kernels (one CTA of 128 threads = one warpgroup per 128-row tile; thread r owns row r,
// which is TMEM lane r of every accumulator):
//   k_mlp_forward   persistent inference: per tile, features -> shared memory (canonical
//                   no-swizzle K-major layout), 4 chained tcgen05.mma (kind::f16, BF16 x BF16
//                   -> FP32 in TMEM, M = 128), tcgen05.ld epilogues (bias, ReLU, BF16) back
//                   into shared memory for the next layer; output logits or proposal bits
//   k_mlp_train     forward + backward per tile, weight gradients accumulated in TMEM across
//                   the CTA's tiles (dW = dZ^T H: the activation tiles are read a second time
//                   as MN-major operands, so no transposed copies are written), then added to
//                   global FP32 gradients; bias gradients and the 4 x 64 last layer by warp
//                   reductions
//   k_mlp_adam      Adam step on the FP32 parameters
// Every wait on an mbarrier is bounded; a wait that runs out sets an error flag, and the
// kernel stops issuing work, waits (bounded) for what it issued and frees its TMEM.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace mlp {

constexpr int kIn = 128, kH = 64, kOut = 4, kOutPad = 16, kRows = 128;
constexpr int kStencilFeat = 108, kFeat = 113;
// parameter block (floats): W1[64][128] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[4][64] b4[4]
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kOut * kH, kParams = oB4 + kOut;
static_assert(kParams == 16836, "parameter block layout");

constexpr uint32_t kSpinLimit = 1u << 26;   // bounded mbarrier waits (~ a second or more)

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase of `parity` to complete; false if it did not within the limit.
__device__ __forceinline__ bool mbar_wait_thread(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kSpinLimit; ++it)
    {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

// The same for every thread of the CTA, with one outcome for all (a thread that gave up
// must not leave the others at a barrier).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const bool ok = mbar_wait_thread(bar, parity);
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory -> visible to the tensor cores' (async proxy) reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05, no swizzle): start address, leading-dimension
// byte offset (between the two 8 x 16-byte core matrices along K of one MMA for K-major
// operands; between 8-element groups along K for MN-major ones), stride-dimension byte
// offset (between 8-row groups along M/N), descriptor version 1 in bits 46-47.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// D[tmem] (+)= A * B, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 :
                 : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
                 : "memory");
}

// The MMAs this thread issued so far arrive on `bar` when they complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31),
// waited for before return (the wait names the registers, so no use moves above it).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 64 consecutive FP32 columns of this thread's TMEM lane in one load and one wait.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64])
{
    uint32_t r[64];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {"
                 "%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
                 "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
                 "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
                   "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
                   "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
                   "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
                   "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]),
                   "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                   "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31]),
                   "+r"(r[32]), "+r"(r[33]), "+r"(r[34]), "+r"(r[35]), "+r"(r[36]), "+r"(r[37]), "+r"(r[38]), "+r"(r[39]),
                   "+r"(r[40]), "+r"(r[41]), "+r"(r[42]), "+r"(r[43]), "+r"(r[44]), "+r"(r[45]), "+r"(r[46]), "+r"(r[47]),
                   "+r"(r[48]), "+r"(r[49]), "+r"(r[50]), "+r"(r[51]), "+r"(r[52]), "+r"(r[53]), "+r"(r[54]), "+r"(r[55]),
                   "+r"(r[56]), "+r"(r[57]), "+r"(r[58]), "+r"(r[59]), "+r"(r[60]), "+r"(r[61]), "+r"(r[62]), "+r"(r[63])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- shared-memory operand layout
// Canonical no-swizzle K-major tile of `K` columns: element (row r, column k) at
//   (r / 8) * (16 K) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2 bytes,
// i.e. 8 x 8 core matrices of 128 contiguous bytes, K-adjacent ones 128 B apart (LBO) and
// row-adjacent ones 16 K B apart (SBO). Read as an MN-major operand whose MN dimension is
// the column index k and whose K dimension is the row index r, the same bytes have
// 8-element groups along MN 128 B apart (SBO) and 8-row groups along K 16 K B apart (LBO).
__device__ __forceinline__ uint32_t kmaj_off(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// A[M = 128 rows][16 columns starting at 16 j] of a K-major tile, as an MMA operand.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, int K, int j)
{
    return sdesc(base + (uint32_t)j * 256u, 128u, (uint32_t)K * 16u);
}
// The K-major tile of K columns read transposed: operand [MN = its columns][K = rows
// 16 j .. 16 j + 15].
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, int K, int j)
{
    return sdesc(base + (uint32_t)j * 2u * (uint32_t)K * 16u, (uint32_t)K * 16u, 128u);
}

// Eight consecutive values of row r (columns k0 .. k0 + 7, k0 % 8 == 0) as one 16-byte store.
__device__ __forceinline__ void st_row8(uint8_t* tile, int r, int k0, int K, const float* v)
{
    __align__(16) __nv_bfloat162 b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) b[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(tile + kmaj_off(r, k0, K)) = *reinterpret_cast<const uint4*>(b);
}
__device__ __forceinline__ void ld_row8(const uint8_t* tile, int r, int k0, int K, float* v)
{
    const uint4 q = *reinterpret_cast<const uint4*>(tile + kmaj_off(r, k0, K));
    const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const float2 f = __bfloat1622float2(b[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

// Weights from the FP32 parameter block into K-major BF16 tiles ([out rows][in columns]);
// W4 is padded to 16 rows of zeros. Called by the whole CTA.
__device__ __forceinline__ void load_weights(const float* prm, uint8_t* sW1, uint8_t* sW2, uint8_t* sW3, uint8_t* sW4)
{
    for (int e = threadIdx.x; e < kH * kIn / 8; e += blockDim.x)
    {
        const int o = e / (kIn / 8), k0 = (e % (kIn / 8)) * 8;
        st_row8(sW1, o, k0, kIn, prm + oW1 + o * kIn + k0);
    }
    for (int e = threadIdx.x; e < kH * kH / 8; e += blockDim.x)
    {
        const int o = e / (kH / 8), k0 = (e % (kH / 8)) * 8;
        st_row8(sW2, o, k0, kH, prm + oW2 + o * kH + k0);
        st_row8(sW3, o, k0, kH, prm + oW3 + o * kH + k0);
    }
    for (int e = threadIdx.x; e < kOutPad * kH / 8; e += blockDim.x)
    {
        const int o = e / (kH / 8), k0 = (e % (kH / 8)) * 8;
        float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        st_row8(sW4, o, k0, kH, o < kOut ? prm + oW4 + o * kH + k0 : z);
    }
}

// The weights and biases as the forward kernels hold them in shared memory (the bytes from
// FwdSmem::W1 to FwdSmem::Bar), built once per parameter set by k_mlp_pack, so that a CTA
// starts with one vectorised copy instead of converting the FP32 block.
constexpr int kPackBytes = 35648;   // FwdSmem::Bar - FwdSmem::W1

// Shared-memory image of the parameters (one CTA).
__device__ __forceinline__ void load_packed(const uint8_t* __restrict__ pack, uint8_t* dst)
{
    const uint4* src = reinterpret_cast<const uint4*>(pack);
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll 6
    for (int i = threadIdx.x; i < kPackBytes / 16; i += blockDim.x) d[i] = src[i];
}

// Row r of the features: 128 BF16 values from a row-major global array (zeros past n).
__device__ __forceinline__ void load_feature_row(const __nv_bfloat16* feats, int64_t row, int64_t n, uint8_t* sX, int r)
{
    const uint4* src = reinterpret_cast<const uint4*>(feats + row * kIn);
#pragma unroll 4
    for (int c = 0; c < kIn / 8; ++c)
    {
        const uint4 q = row < n ? src[c] : make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4*>(sX + kmaj_off(r, 8 * c, kIn)) = q;
    }
}

// Epilogue of a hidden layer: this thread's 64 accumulators (TMEM lane = row) + bias, ReLU,
// BF16 into row r of the next layer's K-major tile.
__device__ __forceinline__ void hidden_epilogue(uint32_t tcol, const float* bias, uint8_t* sH, int r)
{
    const int warp = threadIdx.x >> 5;
    float v[kH];
    tmem_ld64(tcol + ((uint32_t)(warp * 32) << 16), v);
#pragma unroll
    for (int i = 0; i < kH; ++i) v[i] = fmaxf(v[i] + bias[i], 0.0f);
#pragma unroll
    for (int c = 0; c < kH; c += 8) st_row8(sH, r, c, kH, v + c);
}

// Dynamic shared memory of the forward kernel (bytes, 1024-aligned base).
struct FwdSmem
{
    static constexpr int X = 0, H = X + kRows * kIn * 2, W1 = H + kRows * kH * 2, W2 = W1 + kH * kIn * 2,
                         W3 = W2 + kH * kH * 2, W4 = W3 + kH * kH * 2, Bias = W4 + kOutPad * kH * 2,
                         Bar = Bias + (3 * kH + kOutPad) * 4, Slot = Bar + 8, Total = Slot + 16;
};

// The forward pass of one tile (128 rows in sX): four MMA groups and their epilogues. The
// logits of row r come back in z[0..3]. Returns false if an MMA wait ran out (the kernel
// must then stop).
__device__ __forceinline__ bool forward_tile(uint8_t* sm, uint32_t tmem, uint64_t* bar, uint32_t& phase, float* z,
                                             bool keep_hidden, uint8_t* sH1, uint8_t* sH2, uint8_t* sH3)
{
    const int r = threadIdx.x;
    uint8_t* sX = sm + FwdSmem::X;
    const float* bias = reinterpret_cast<const float*>(sm + FwdSmem::Bias);
    const uint32_t aX = smem_u32(sX), aW1 = smem_u32(sm + FwdSmem::W1), aW2 = smem_u32(sm + FwdSmem::W2),
                   aW3 = smem_u32(sm + FwdSmem::W3), aW4 = smem_u32(sm + FwdSmem::W4);
    uint8_t* hbuf[3] = {keep_hidden ? sH1 : sm + FwdSmem::H, keep_hidden ? sH2 : sm + FwdSmem::H,
                        keep_hidden ? sH3 : sm + FwdSmem::H};
    const uint32_t wdesc_base[3] = {aW2, aW3, aW4};
    // layer 1: X [128 x 128] * W1^T -> TMEM columns 0..63
    fence_async_smem();
    __syncthreads();
    if (r == 0)
    {
        tc_fence_after();
#pragma unroll
        for (int j = 0; j < kIn / 16; ++j)
            mma_bf16(tmem + 0, desc_kmajor(aX, kIn, j), desc_kmajor(aW1, kIn, j), idesc_bf16(kH, false, false), j > 0);
        mma_commit(bar);
    }
    bool ok = mbar_wait(bar, phase);
    phase ^= 1u;
    if (!ok) return false;
    tc_fence_after();
    hidden_epilogue(tmem + 0, bias, hbuf[0], r);
    // layers 2, 3 (N = 64) and 4 (N = 16, logits)
#pragma unroll 1
    for (int l = 0; l < 3; ++l)
    {
        const int n = (l < 2) ? kH : kOutPad;
        const uint32_t dcol = 64u * (uint32_t)(l + 1);
        tc_fence_before();
        fence_async_smem();
        __syncthreads();
        if (r == 0)
        {
            tc_fence_after();
            const uint32_t aH = smem_u32(hbuf[l]);
#pragma unroll
            for (int j = 0; j < kH / 16; ++j)
                mma_bf16(tmem + dcol, desc_kmajor(aH, kH, j), desc_kmajor(wdesc_base[l], kH, j),
                         idesc_bf16(n, false, false), j > 0);
            mma_commit(bar);
        }
        ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!ok) return false;
        tc_fence_after();
        if (l < 2) hidden_epilogue(tmem + dcol, bias + kH * (l + 1), hbuf[l + 1], r);
        else
        {
            float v[16];
            tmem_ld16(tmem + dcol + ((uint32_t)((threadIdx.x >> 5) * 32) << 16), v);
#pragma unroll
            for (int o = 0; o < kOut; ++o) z[o] = v[o] + bias[3 * kH + o];
        }
    }
    tc_fence_before();
    return true;
}

// Biases into shared memory (b1, b2, b3, b4 padded).
__device__ __forceinline__ void load_biases(const float* prm, float* bias)
{
    for (int i = threadIdx.x; i < 3 * kH + kOutPad; i += blockDim.x)
    {
        float v = 0.0f;
        if (i < kH) v = prm[oB1 + i];
        else if (i < 2 * kH) v = prm[oB2 + i - kH];
        else if (i < 3 * kH) v = prm[oB3 + i - 2 * kH];
        else if (i < 3 * kH + kOut) v = prm[oB4 + i - 3 * kH];
        bias[i] = v;
    }
}

static_assert(FwdSmem::Bar - FwdSmem::W1 == kPackBytes && FwdSmem::W1 % 16 == 0, "packed parameter image");

// (static kernels here: the header is included by more than one translation unit)
// The packed image of a parameter block (one CTA of 128 threads).
static __global__ void __launch_bounds__(kRows) k_mlp_pack(const float* __restrict__ prm, uint8_t* __restrict__ pack)
{
    uint8_t* base = pack - FwdSmem::W1;   // the image's offsets are those of the shared memory
    load_weights(prm, base + FwdSmem::W1, base + FwdSmem::W2, base + FwdSmem::W3, base + FwdSmem::W4);
    load_biases(prm, reinterpret_cast<float*>(base + FwdSmem::Bias));
}

// Inference over n rows of features (row-major BF16 [n][128]). Outputs (either may be null):
// logits[n][4]; prop[4 n] bytes, 1 where the logit exceeds `thr`. err: set to 1 if a wait
// ran out. One CTA of 128 threads per tile, persistent over the tiles.
static __global__ void __launch_bounds__(kRows, 1) k_mlp_forward(const float* __restrict__ prm, const __nv_bfloat16* __restrict__ feats,
                                                          int64_t n, float* logits, uint8_t* prop, float thr, int* err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + FwdSmem::Bar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + FwdSmem::Slot);
    const int r = threadIdx.x;
    load_weights(prm, sm + FwdSmem::W1, sm + FwdSmem::W2, sm + FwdSmem::W3, sm + FwdSmem::W4);
    load_biases(prm, reinterpret_cast<float*>(sm + FwdSmem::Bias));
    if (r == 0) mbar_init(bar, 1);
    if (r < 32) tmem_alloc(slot, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntiles = (n + kRows - 1) / kRows;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x)
    {
        const int64_t row = t * kRows + r;
        load_feature_row(feats, row, n, sm + FwdSmem::X, r);
        float z[kOut];
        ok = forward_tile(sm, tmem, bar, phase, z, false, nullptr, nullptr, nullptr);
        if (!ok) break;
        if (row < n)
        {
            if (logits)
            {
#pragma unroll
                for (int o = 0; o < kOut; ++o) logits[row * kOut + o] = z[o];
            }
            if (prop)
            {
                uint32_t bits = 0;
#pragma unroll
                for (int o = 0; o < kOut; ++o) bits |= (z[o] > thr ? 1u : 0u) << (8 * o);
                *reinterpret_cast<uint32_t*>(prop + 4 * row) = bits;
            }
        }
        // every thread's TMEM reads of this tile precede the next tile's MMAs (next barrier)
    }
    if (!ok && err) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (r < 32) tmem_dealloc(tmem, 256);
}

// ---------------------------------------------------------------- training

struct TrainSmem
{
    // the forward kernel's regions first (X, an unused H, weights, biases, barrier), then the
    // kept activations and the gradient tile, 1024-byte aligned
    static constexpr int H1 = (FwdSmem::Total + 1023) / 1024 * 1024, H2 = H1 + kRows * kH * 2, H3 = H2 + kRows * kH * 2,
                         DZ = H3 + kRows * kH * 2,                 // [128 rows][128] K-major, columns 64..127 zero
                         Red = DZ + kRows * kIn * 2,               // per-CTA gradient sums: db1..3, db4, dW4
                         Total = Red + (3 * kH + kOutPad + kOut * kH) * 4;
};
static_assert(FwdSmem::Bar % 8 == 0 && TrainSmem::H1 % 1024 == 0 && TrainSmem::Red % 16 == 0, "shared-memory layout");

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// dZ = dH (TMEM, 64 columns at tcol) * [H > 0] (H: this thread's row of the layer's BF16
// activations) -> row r of sDZ (columns 0..63, BF16); the bias gradient of the layer
// (sum over rows) is added into red[0..63].
__device__ __forceinline__ void relu_backward(uint32_t tcol, const uint8_t* sHl, uint8_t* sDZ, float* red, int r, bool valid)
{
    const int warp = threadIdx.x >> 5;
#pragma unroll 1
    for (int c = 0; c < kH; c += 16)
    {
        float g[16], h[16];
        tmem_ld16(tcol + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, g);
        ld_row8(sHl, r, c, kH, h);
        ld_row8(sHl, r, c + 8, kH, h + 8);
#pragma unroll
        for (int i = 0; i < 16; ++i) g[i] = (valid && h[i] > 0.0f) ? g[i] : 0.0f;
        // the operand of the weight-gradient and input-gradient MMAs is the BF16 value
#pragma unroll
        for (int i = 0; i < 16; ++i) g[i] = __bfloat162float(__float2bfloat16_rn(g[i]));
        st_row8(sDZ, r, c, kIn, g);
        st_row8(sDZ, r, c + 8, kIn, g + 8);
#pragma unroll
        for (int i = 0; i < 16; ++i)
        {
            const float s = warp_sum(g[i]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&red[c + i], s);
        }
    }
}

// Forward + backward over n rows of features with labels (bits 0..3 of labels[row]) and
// per-class positive weight pos_w: loss = sum over rows and outputs of
// w * (softplus(z) - y z) / n with w = pos_w for y = 1, else 1. Adds the gradient of the
// loss with respect to every parameter into grad[kParams] and the loss into *loss.
static __global__ void __launch_bounds__(kRows, 1) k_mlp_train(const float* __restrict__ prm, const __nv_bfloat16* __restrict__ feats,
                                                        const uint8_t* __restrict__ labels, int64_t n, float pos_w,
                                                        float* grad, float* loss, int* err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + FwdSmem::Bar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + FwdSmem::Slot);
    uint8_t *sX = sm + FwdSmem::X, *sH1 = sm + TrainSmem::H1, *sH2 = sm + TrainSmem::H2, *sH3 = sm + TrainSmem::H3,
            *sDZ = sm + TrainSmem::DZ;
    float* red = reinterpret_cast<float*>(sm + TrainSmem::Red);   // db1 db2 db3 (64 each) db4 (16) dW4 (4 x 64)
    const int r = threadIdx.x, warp = r >> 5, lane = r & 31;
    load_weights(prm, sm + FwdSmem::W1, sm + FwdSmem::W2, sm + FwdSmem::W3, sm + FwdSmem::W4);
    load_biases(prm, reinterpret_cast<float*>(sm + FwdSmem::Bias));
    for (int i = r; i < 3 * kH + kOutPad + kOut * kH; i += blockDim.x) red[i] = 0.0f;
    for (int c = 0; c < kIn; c += 8)
    {
        const float z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        st_row8(sDZ, r, c, kIn, z8);   // columns 64..127 stay zero: the padding rows of dZ^T
    }
    if (r == 0) mbar_init(bar, 1);
    if (r < 32) tmem_alloc(slot, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    // TMEM columns: forward D1 0..63, D2 64..127, D3 128..191, D4 192..207 (dH3, dH2, dH1 reuse
    // 0..63, 64..127, 128..191); accumulators dW1 256..383, dW2 384..447, dW3 448..511
    const uint32_t cW1 = 256, cW2 = 384, cW3 = 448;
    uint32_t phase = 0;
    bool ok = true, first = true;
    float loss_acc = 0.0f;
    const float inv_n = 1.0f / (float)(n > 0 ? n : 1);
    const uint32_t aX = smem_u32(sX), aH1 = smem_u32(sH1), aH2 = smem_u32(sH2), aDZ = smem_u32(sDZ),
                   aW2 = smem_u32(sm + FwdSmem::W2), aW3 = smem_u32(sm + FwdSmem::W3), aW4 = smem_u32(sm + FwdSmem::W4);
    const int64_t ntiles = (n + kRows - 1) / kRows;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x)
    {
        const int64_t row = t * kRows + r;
        const bool valid = row < n;
        load_feature_row(feats, row, n, sX, r);
        float z[kOut];
        ok = forward_tile(sm, tmem, bar, phase, z, true, sH1, sH2, sH3);
        if (!ok) break;
        // output layer: dZ4 = w (sigmoid(z) - y) / n
        const uint32_t lab = valid ? labels[row] : 0u;
        float dz4[kOutPad];
#pragma unroll
        for (int o = 0; o < kOutPad; ++o) dz4[o] = 0.0f;
#pragma unroll
        for (int o = 0; o < kOut; ++o)
        {
            const float y = (float)((lab >> o) & 1u);
            const float w = y > 0.5f ? pos_w : 1.0f;
            const float sp = fmaxf(z[o], 0.0f) + log1pf(expf(-fabsf(z[o])));   // softplus
            const float s = 1.0f / (1.0f + expf(-z[o]));
            if (valid)
            {
                loss_acc += w * (sp - y * z[o]) * inv_n;
                dz4[o] = __bfloat162float(__float2bfloat16_rn(w * (s - y) * inv_n));
            }
        }
        // dZ4 as columns 0..15 of the dZ tile (the rest of 0..63 zero) for dH3 = dZ4 W4
        st_row8(sDZ, r, 0, kIn, dz4);
        st_row8(sDZ, r, 8, kIn, dz4 + 8);
        {
            const float z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int c = 16; c < kH; c += 8) st_row8(sDZ, r, c, kIn, z8);
        }
        // db4, dW4 = sum over rows of dz4 (x) h3 (warp sums, then shared-memory atomics)
        {
            float h3[kH];
#pragma unroll
            for (int c = 0; c < kH; c += 8) ld_row8(sH3, r, c, kH, h3 + c);
#pragma unroll
            for (int o = 0; o < kOut; ++o)
            {
                const float s = warp_sum(dz4[o]);
                if (lane == 0) atomicAdd(&red[3 * kH + o], s);
#pragma unroll 8
                for (int f = 0; f < kH; ++f)
                {
                    const float p = warp_sum(dz4[o] * h3[f]);
                    if (lane == 0) atomicAdd(&red[3 * kH + kOutPad + o * kH + f], p);
                }
            }
        }
        // dH3 = dZ4 [128 x 16] * W4 [16 x 64] -> TMEM 0..63 (W4's tile read MN-major)
        tc_fence_before();
        fence_async_smem();
        __syncthreads();
        if (r == 0)
        {
            tc_fence_after();
            mma_bf16(tmem + 0, desc_kmajor(aDZ, kIn, 0), desc_mnmajor(aW4, kH, 0), idesc_bf16(kH, false, true), 0);
            mma_commit(bar);
        }
        ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        // layers 3, 2, 1: dZ_l = dH_l * relu'(H_l); dW_l += dZ_l^T H_(l-1); dH_(l-1) = dZ_l W_l
        const uint32_t dcol[3] = {0u, 64u, 128u};        // dH3, dH2, dH1
        const uint32_t accc[3] = {cW3, cW2, cW1};
        uint8_t* const hl[3] = {sH3, sH2, sH1};          // activations of the layer
        const uint32_t hprev[3] = {aH2, aH1, aX};        // its input
        const int kprev[3] = {kH, kH, kIn};
        const uint32_t wl[3] = {aW3, aW2, 0u};
#pragma unroll 1
        for (int l = 0; l < 3; ++l)
        {
            relu_backward(tmem + dcol[l], hl[l], sDZ, red + kH * (2 - l), r, valid);
            tc_fence_before();
            fence_async_smem();
            __syncthreads();
            if (r == 0)
            {
                tc_fence_after();
                // dW_l [64 (+64 zero) x kprev] += dZ_l^T [128 x rows] * H_(l-1) [rows x kprev]
#pragma unroll
                for (int j = 0; j < kRows / 16; ++j)
                    mma_bf16(tmem + accc[l], desc_mnmajor(aDZ, kIn, j), desc_mnmajor(hprev[l], kprev[l], j),
                             idesc_bf16(kprev[l], true, true), (first && j == 0) ? 0u : 1u);
                // dH_(l-1) [rows x 64] = dZ_l [rows x 64] * W_l [64 x 64] (W_l's tile read MN-major)
                if (l < 2)
                {
#pragma unroll
                    for (int j = 0; j < kH / 16; ++j)
                        mma_bf16(tmem + dcol[l + 1], desc_kmajor(aDZ, kIn, j), desc_mnmajor(wl[l], kH, j),
                                 idesc_bf16(kH, false, true), j > 0);
                }
                mma_commit(bar);
            }
            ok = mbar_wait(bar, phase);
            phase ^= 1u;
            if (!ok) break;
            tc_fence_after();
        }
        first = false;
    }
    // accumulated dW1..dW3 (TMEM rows 0..63 = output units) and the shared-memory sums
    // into the global gradient
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (ok && !first && r < kH)
    {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
        for (int c = 0; c < kIn; c += 16)
        {
            float v[16];
            tmem_ld16(tmem + cW1 + lane_base + (uint32_t)c, v);
            for (int i = 0; i < 16; ++i) atomicAdd(&grad[oW1 + r * kIn + c + i], v[i]);
        }
#pragma unroll 1
        for (int c = 0; c < kH; c += 16)
        {
            float v[16];
            tmem_ld16(tmem + cW2 + lane_base + (uint32_t)c, v);
            for (int i = 0; i < 16; ++i) atomicAdd(&grad[oW2 + r * kH + c + i], v[i]);
            tmem_ld16(tmem + cW3 + lane_base + (uint32_t)c, v);
            for (int i = 0; i < 16; ++i) atomicAdd(&grad[oW3 + r * kH + c + i], v[i]);
        }
    }
    else if (ok && !first)
    {
        // warps 2 and 3 take part in no TMEM load of rows >= 64 (those rows are the zero padding)
    }
    __syncthreads();
    if (ok)
    {
        for (int i = r; i < kH; i += blockDim.x)
        {
            atomicAdd(&grad[oB1 + i], red[i]);
            atomicAdd(&grad[oB2 + i], red[kH + i]);
            atomicAdd(&grad[oB3 + i], red[2 * kH + i]);
        }
        for (int i = r; i < kOut; i += blockDim.x) atomicAdd(&grad[oB4 + i], red[3 * kH + i]);
        for (int i = r; i < kOut * kH; i += blockDim.x) atomicAdd(&grad[oW4 + i], red[3 * kH + kOutPad + i]);
        const float ls = warp_sum(loss_acc);
        if (lane == 0) atomicAdd(loss, ls);
    }
    if (!ok && err) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (r < 32) tmem_dealloc(tmem, 512);
}

// One Adam step (bias-corrected, step number t >= 1) on the FP32 parameters; clears grad.
static __global__ void k_mlp_adam(float* prm, float* grad, float* m, float* v, int t, float lr, float b1, float b2, float eps)
{
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x)
    {
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        grad[i] = 0.0f;
    }
}

} // namespace mlp
