// Host side of the learned refinement proposal's MLP (csrc/proposal.cuh): inference and
// gradients on caller-supplied samples, and a trainer (Adam on device) fed either with host
// samples or with the features and labels a simulation recorded on the device.
// No counterpart in the reference.
#include "../../include/mwdg2.h"
#include "proposal.cuh"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

void mwdg2_detail_set_last_error(const char* msg);
// Device features ([n][128] BF16) and labels ([n] bytes) the simulation recorded for its last
// step (csrc/sim.cu); MWDG2_ERR_STATE if it records none.
mwdg2_status mwdg2_detail_proposal_samples(mwdg2_sim* sim, const void** feats, const uint8_t** labels, int64_t* n,
                                           int* device);

namespace {

mwdg2_status fail(mwdg2_status st, const std::string& msg)
{
    mwdg2_detail_set_last_error(msg.c_str());
    return st;
}

#define CUDA_OK(call)                                                                                    \
    do                                                                                                   \
    {                                                                                                    \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return fail(MWDG2_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// FP32 -> BF16, round to nearest even (NaN kept quiet).
uint16_t to_bf16(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Device buffers released at scope exit.
struct DevBufs
{
    std::vector<void*> p;
    ~DevBufs() { for (void* q : p) cudaFree(q); }
    template <typename T> cudaError_t alloc(T*& out, size_t count)
    {
        void* v = nullptr;
        const cudaError_t e = cudaMalloc(&v, count * sizeof(T) + 16);
        if (e == cudaSuccess) p.push_back(v);
        out = static_cast<T*>(v);
        return e;
    }
};

constexpr size_t kFwdSmem = mlp::FwdSmem::Total + 1024;
constexpr size_t kTrainSmem = mlp::TrainSmem::Total + 1024;

cudaError_t set_smem_attrs()
{
    cudaError_t e = cudaFuncSetAttribute(mlp::k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
    return e;
}

// Host samples (FP32 features [n][113..128]) -> device BF16 rows of 128.
mwdg2_status upload_features(DevBufs& b, const float* feats, int nfeat, int64_t n, __nv_bfloat16*& d)
{
    std::vector<uint16_t> h((size_t)n * mlp::kIn, 0);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < nfeat && k < mlp::kIn; ++k) h[(size_t)i * mlp::kIn + k] = to_bf16(feats[(size_t)i * nfeat + k]);
    CUDA_OK(b.alloc(d, h.size()));
    CUDA_OK(cudaMemcpy(d, h.data(), h.size() * 2, cudaMemcpyHostToDevice));
    return MWDG2_OK;
}

mwdg2_status launch_train(const float* d_prm, const __nv_bfloat16* d_feats, const uint8_t* d_lab, int64_t n, float pos_w,
                          float* d_grad, float* d_loss, int* d_err, cudaStream_t st)
{
    const int64_t tiles = (n + mlp::kRows - 1) / mlp::kRows;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, sm_count()));
    mlp::k_mlp_train<<<grid, mlp::kRows, kTrainSmem, st>>>(d_prm, d_feats, d_lab, n, pos_w, d_grad, d_loss, d_err);
    CUDA_OK(cudaGetLastError());
    return MWDG2_OK;
}

} // namespace

struct mwdg2_trainer
{
    int device = 0;
    float lr = 1e-3f;
    int t = 0;
    float *prm = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    int* err = nullptr;
    cudaStream_t st = nullptr;
};

extern "C" {

mwdg2_status mwdg2_mlp_forward(const float* params, const float* feats, int nfeat, int64_t n, float threshold,
                               float* logits, uint8_t* proposal)
{
    if (!params || !feats || n < 0 || nfeat < 1 || nfeat > mlp::kIn)
        return fail(MWDG2_ERR_ARG, "mwdg2_mlp_forward: bad arguments");
    if (n == 0) return MWDG2_OK;
    CUDA_OK(set_smem_attrs());
    DevBufs b;
    float *d_prm = nullptr, *d_log = nullptr;
    uint8_t* d_prop = nullptr;
    int* d_err = nullptr;
    __nv_bfloat16* d_feat = nullptr;
    CUDA_OK(b.alloc(d_prm, mlp::kParams));
    CUDA_OK(cudaMemcpy(d_prm, params, sizeof(float) * mlp::kParams, cudaMemcpyHostToDevice));
    if (mwdg2_status s = upload_features(b, feats, nfeat, n, d_feat)) return s;
    CUDA_OK(b.alloc(d_log, (size_t)n * mlp::kOut));
    CUDA_OK(b.alloc(d_prop, (size_t)n * mlp::kOut));
    CUDA_OK(b.alloc(d_err, 1));
    CUDA_OK(cudaMemset(d_err, 0, sizeof(int)));
    const int64_t tiles = (n + mlp::kRows - 1) / mlp::kRows;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, 2 * sm_count()));
    mlp::k_mlp_forward<<<grid, mlp::kRows, kFwdSmem>>>(d_prm, d_feat, n, d_log, d_prop, threshold, d_err);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaDeviceSynchronize());
    int err = 0;
    CUDA_OK(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(MWDG2_ERR_TIMEOUT, "mwdg2_mlp_forward: a tensor-core wait ran out");
    if (logits) CUDA_OK(cudaMemcpy(logits, d_log, sizeof(float) * n * mlp::kOut, cudaMemcpyDeviceToHost));
    if (proposal) CUDA_OK(cudaMemcpy(proposal, d_prop, (size_t)n * mlp::kOut, cudaMemcpyDeviceToHost));
    return MWDG2_OK;
}

mwdg2_status mwdg2_mlp_grad(const float* params, const float* feats, int nfeat, const uint8_t* labels, int64_t n,
                            float pos_weight, float* grad, float* loss)
{
    if (!params || !feats || !labels || !grad || n <= 0 || nfeat < 1 || nfeat > mlp::kIn)
        return fail(MWDG2_ERR_ARG, "mwdg2_mlp_grad: bad arguments");
    CUDA_OK(set_smem_attrs());
    DevBufs b;
    float *d_prm = nullptr, *d_grad = nullptr, *d_loss = nullptr;
    uint8_t* d_lab = nullptr;
    int* d_err = nullptr;
    __nv_bfloat16* d_feat = nullptr;
    CUDA_OK(b.alloc(d_prm, mlp::kParams));
    CUDA_OK(cudaMemcpy(d_prm, params, sizeof(float) * mlp::kParams, cudaMemcpyHostToDevice));
    if (mwdg2_status s = upload_features(b, feats, nfeat, n, d_feat)) return s;
    CUDA_OK(b.alloc(d_lab, (size_t)n));
    CUDA_OK(cudaMemcpy(d_lab, labels, (size_t)n, cudaMemcpyHostToDevice));
    CUDA_OK(b.alloc(d_grad, mlp::kParams));
    CUDA_OK(cudaMemset(d_grad, 0, sizeof(float) * mlp::kParams));
    CUDA_OK(b.alloc(d_loss, 1));
    CUDA_OK(cudaMemset(d_loss, 0, sizeof(float)));
    CUDA_OK(b.alloc(d_err, 1));
    CUDA_OK(cudaMemset(d_err, 0, sizeof(int)));
    if (mwdg2_status s = launch_train(d_prm, d_feat, d_lab, n, pos_weight, d_grad, d_loss, d_err, nullptr)) return s;
    CUDA_OK(cudaDeviceSynchronize());
    int err = 0;
    CUDA_OK(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(MWDG2_ERR_TIMEOUT, "mwdg2_mlp_grad: a tensor-core wait ran out");
    CUDA_OK(cudaMemcpy(grad, d_grad, sizeof(float) * mlp::kParams, cudaMemcpyDeviceToHost));
    if (loss) CUDA_OK(cudaMemcpy(loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    return MWDG2_OK;
}

mwdg2_status mwdg2_trainer_create(const float* init_params, float lr, int device, mwdg2_trainer** out)
{
    if (!init_params || !out || !(lr > 0.0f)) return fail(MWDG2_ERR_ARG, "mwdg2_trainer_create: bad arguments");
    *out = nullptr;
    if (device >= 0) CUDA_OK(cudaSetDevice(device));
    auto* t = new mwdg2_trainer();
    CUDA_OK(cudaGetDevice(&t->device));
    t->lr = lr;
    auto alloc = [&](float*& p) { return cudaMalloc(&p, sizeof(float) * mlp::kParams); };
    cudaError_t e = alloc(t->prm);
    if (e == cudaSuccess) e = alloc(t->grad);
    if (e == cudaSuccess) e = alloc(t->m);
    if (e == cudaSuccess) e = alloc(t->v);
    if (e == cudaSuccess) e = cudaMalloc(&t->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&t->err, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&t->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpy(t->prm, init_params, sizeof(float) * mlp::kParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(t->grad, 0, sizeof(float) * mlp::kParams);
    if (e == cudaSuccess) e = cudaMemset(t->m, 0, sizeof(float) * mlp::kParams);
    if (e == cudaSuccess) e = cudaMemset(t->v, 0, sizeof(float) * mlp::kParams);
    if (e == cudaSuccess) e = cudaMemset(t->err, 0, sizeof(int));
    if (e == cudaSuccess) e = set_smem_attrs();
    if (e != cudaSuccess)
    {
        mwdg2_trainer_destroy(t);
        return fail(MWDG2_ERR_CUDA, std::string("mwdg2_trainer_create: ") + cudaGetErrorString(e));
    }
    *out = t;
    return MWDG2_OK;
}

// One Adam step on device samples (features [n][128] BF16, labels [n]).
static mwdg2_status trainer_step_device(mwdg2_trainer* t, const __nv_bfloat16* feats, const uint8_t* labels, int64_t n,
                                        float pos_weight, float* loss_out)
{
    CUDA_OK(cudaSetDevice(t->device));
    CUDA_OK(cudaMemsetAsync(t->loss, 0, sizeof(float), t->st));
    if (mwdg2_status s = launch_train(t->prm, feats, labels, n, pos_weight, t->grad, t->loss, t->err, t->st)) return s;
    ++t->t;
    mlp::k_mlp_adam<<<(mlp::kParams + 255) / 256, 256, 0, t->st>>>(t->prm, t->grad, t->m, t->v, t->t, t->lr, 0.9f, 0.999f,
                                                                  1e-8f);
    CUDA_OK(cudaGetLastError());
    float loss = 0.0f;
    int err = 0;
    CUDA_OK(cudaMemcpyAsync(&loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost, t->st));
    CUDA_OK(cudaMemcpyAsync(&err, t->err, sizeof(int), cudaMemcpyDeviceToHost, t->st));
    CUDA_OK(cudaStreamSynchronize(t->st));
    if (err) return fail(MWDG2_ERR_TIMEOUT, "mwdg2_trainer: a tensor-core wait ran out");
    if (loss_out) *loss_out = loss;
    return MWDG2_OK;
}

mwdg2_status mwdg2_trainer_step(mwdg2_trainer* t, const float* feats, int nfeat, const uint8_t* labels, int64_t n,
                                float pos_weight, float* loss_out)
{
    if (!t || !feats || !labels || n <= 0 || nfeat < 1 || nfeat > mlp::kIn)
        return fail(MWDG2_ERR_ARG, "mwdg2_trainer_step: bad arguments");
    CUDA_OK(cudaSetDevice(t->device));
    DevBufs b;
    __nv_bfloat16* d_feat = nullptr;
    uint8_t* d_lab = nullptr;
    if (mwdg2_status s = upload_features(b, feats, nfeat, n, d_feat)) return s;
    CUDA_OK(b.alloc(d_lab, (size_t)n));
    CUDA_OK(cudaMemcpy(d_lab, labels, (size_t)n, cudaMemcpyHostToDevice));
    return trainer_step_device(t, d_feat, d_lab, n, pos_weight, loss_out);
}

mwdg2_status mwdg2_trainer_observe(mwdg2_trainer* t, mwdg2_sim* sim, float pos_weight, float* loss_out)
{
    if (!t || !sim) return fail(MWDG2_ERR_ARG, "mwdg2_trainer_observe: null argument");
    const void* feats = nullptr;
    const uint8_t* labels = nullptr;
    int64_t n = 0;
    int dev = -1;
    if (mwdg2_status s = mwdg2_detail_proposal_samples(sim, &feats, &labels, &n, &dev)) return s;
    if (dev != t->device) return fail(MWDG2_ERR_ARG, "mwdg2_trainer_observe: the simulation is on another device");
    return trainer_step_device(t, static_cast<const __nv_bfloat16*>(feats), labels, n, pos_weight, loss_out);
}

mwdg2_status mwdg2_trainer_params(mwdg2_trainer* t, float* out)
{
    if (!t || !out) return fail(MWDG2_ERR_ARG, "mwdg2_trainer_params: null argument");
    CUDA_OK(cudaSetDevice(t->device));
    CUDA_OK(cudaStreamSynchronize(t->st));
    CUDA_OK(cudaMemcpy(out, t->prm, sizeof(float) * mlp::kParams, cudaMemcpyDeviceToHost));
    return MWDG2_OK;
}

void mwdg2_trainer_destroy(mwdg2_trainer* t)
{
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->st) cudaStreamSynchronize(t->st);
    for (float* p : {t->prm, t->grad, t->m, t->v, t->loss}) if (p) cudaFree(p);
    if (t->err) cudaFree(t->err);
    if (t->st) cudaStreamDestroy(t->st);
    delete t;
}

} // extern "C"
