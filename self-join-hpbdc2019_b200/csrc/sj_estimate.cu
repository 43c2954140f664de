// Learned result-size estimator: a 16 -> 64 -> 64 -> 2 ReLU MLP on per-cell
// features predicts log2(1 + distance calcs) and log2(1 + hits) of a cell.
// Forward, backward and Adam are plain FP32 CUDA-core kernels (the network is
// tiny).  The sampling estimator it replaces (GPU.cu:854-1065, which counts
// the hits of every 100th point) runs as the join's own count pass over
// tasks for the sampled points (sj_tasks.cu builds them, sj_api.cpp runs it).
#include <mutex>

#include "sj_internal.h"

namespace {

// ------------------------------------------------------------------ MLP ----
// parameter offsets
constexpr int OW1 = 0;
constexpr int OB1 = OW1 + SJ_NFEAT * SJ_HID;
constexpr int OW2 = OB1 + SJ_HID;
constexpr int OB2 = OW2 + SJ_HID * SJ_HID;
constexpr int OW3 = OB2 + SJ_HID;
constexpr int OB3 = OW3 + SJ_HID * SJ_NOUT;
constexpr int NP = OB3 + SJ_NOUT;
static_assert(NP == SJ_MLP_NPARAM, "parameter layout");

__device__ __forceinline__ void mlp_forward(const float *__restrict__ w, const float *x, float *z1, float *z2,
                                            float *y)
{
    for (int j = 0; j < SJ_HID; j++) {
        float s = w[OB1 + j];
#pragma unroll
        for (int i = 0; i < SJ_NFEAT; i++) s = fmaf(x[i], w[OW1 + i * SJ_HID + j], s);
        z1[j] = s;
    }
    for (int j = 0; j < SJ_HID; j++) {
        float s = w[OB2 + j];
        for (int i = 0; i < SJ_HID; i++) s = fmaf(fmaxf(z1[i], 0.f), w[OW2 + i * SJ_HID + j], s);
        z2[j] = s;
    }
#pragma unroll
    for (int o = 0; o < SJ_NOUT; o++) {
        float s = w[OB3 + o];
        for (int i = 0; i < SJ_HID; i++) s = fmaf(fmaxf(z2[i], 0.f), w[OW3 + i * SJ_NOUT + o], s);
        y[o] = s;
    }
}

__global__ void __launch_bounds__(128) k_mlp_infer(const float *__restrict__ feat, uint32_t m,
                                                   const float *__restrict__ wg, float *__restrict__ out)
{
    __shared__ float w[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) w[i] = wg[i];
    __syncthreads();
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    float x[SJ_NFEAT], z1[SJ_HID], z2[SJ_HID], y[SJ_NOUT];
    for (int i = 0; i < SJ_NFEAT; i++) x[i] = feat[(uint64_t)s * SJ_NFEAT + i];
    mlp_forward(w, x, z1, z2, y);
    for (int o = 0; o < SJ_NOUT; o++) out[(uint64_t)s * SJ_NOUT + o] = y[o];
}

// Per-sample forward + backward.  Loss = 1/(2m) * sum (y - t)^2.  Writes the
// activations and pre-activation gradients the weight gradients need.
__global__ void __launch_bounds__(128) k_mlp_backprop(const float *__restrict__ X, const float *__restrict__ Yt,
                                                      uint32_t m, const float *__restrict__ wg,
                                                      float *__restrict__ H1, float *__restrict__ G1,
                                                      float *__restrict__ H2, float *__restrict__ G2,
                                                      float *__restrict__ G3, float *__restrict__ loss)
{
    __shared__ float w[NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) w[i] = wg[i];
    __syncthreads();
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (s < m) {
        float x[SJ_NFEAT], z1[SJ_HID], z2[SJ_HID], y[SJ_NOUT], dy[SJ_NOUT], d2[SJ_HID];
        for (int i = 0; i < SJ_NFEAT; i++) x[i] = X[(uint64_t)s * SJ_NFEAT + i];
        mlp_forward(w, x, z1, z2, y);
        const float inv = 1.0f / (float)m;
        for (int o = 0; o < SJ_NOUT; o++) {
            float e = y[o] - Yt[(uint64_t)s * SJ_NOUT + o];
            l += 0.5f * e * e;
            dy[o] = e * inv;
            G3[(uint64_t)s * SJ_NOUT + o] = dy[o];
        }
        for (int i = 0; i < SJ_HID; i++) {
            float g = 0.f;
#pragma unroll
            for (int o = 0; o < SJ_NOUT; o++) g = fmaf(dy[o], w[OW3 + i * SJ_NOUT + o], g);
            d2[i] = z2[i] > 0.f ? g : 0.f;
            H2[(uint64_t)s * SJ_HID + i] = fmaxf(z2[i], 0.f);
            G2[(uint64_t)s * SJ_HID + i] = d2[i];
        }
        for (int i = 0; i < SJ_HID; i++) {
            float g = 0.f;
            for (int j = 0; j < SJ_HID; j++) g = fmaf(d2[j], w[OW2 + i * SJ_HID + j], g);
            H1[(uint64_t)s * SJ_HID + i] = fmaxf(z1[i], 0.f);
            G1[(uint64_t)s * SJ_HID + i] = z1[i] > 0.f ? g : 0.f;
        }
    }
    // loss reduction
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l / (float)m);
}

// grad[param] = sum over samples of (input activation) x (output gradient);
// one thread per parameter.  Inputs: X (m x 16), H1, H2 (m x 64);
// gradients: G1, G2 (m x 64), G3 (m x 2).
__global__ void __launch_bounds__(256) k_mlp_wgrad(const float *__restrict__ X, const float *__restrict__ H1,
                                                   const float *__restrict__ H2, const float *__restrict__ G1,
                                                   const float *__restrict__ G2, const float *__restrict__ G3,
                                                   uint32_t m, float *__restrict__ grad)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float *A = nullptr, *G = nullptr;
    int ai = -1, gj, aw = 0, gw;
    if (p < OB1) { A = X; aw = SJ_NFEAT; ai = (p - OW1) / SJ_HID; G = G1; gw = SJ_HID; gj = (p - OW1) % SJ_HID; }
    else if (p < OW2) { G = G1; gw = SJ_HID; gj = p - OB1; }
    else if (p < OB2) { A = H1; aw = SJ_HID; ai = (p - OW2) / SJ_HID; G = G2; gw = SJ_HID; gj = (p - OW2) % SJ_HID; }
    else if (p < OW3) { G = G2; gw = SJ_HID; gj = p - OB2; }
    else if (p < OB3) { A = H2; aw = SJ_HID; ai = (p - OW3) / SJ_NOUT; G = G3; gw = SJ_NOUT; gj = (p - OW3) % SJ_NOUT; }
    else { G = G3; gw = SJ_NOUT; gj = p - OB3; }
    float s = 0.f;
    for (uint32_t k = 0; k < m; k++) {
        float av = (ai >= 0) ? A[(uint64_t)k * aw + ai] : 1.0f;
        s = fmaf(av, G[(uint64_t)k * gw + gj], s);
    }
    grad[p] = s;
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ mm,
                       float *__restrict__ vv, int step, float lr)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float b1 = 0.9f, b2 = 0.999f, e = 1e-8f;
    float m = b1 * mm[p] + (1.f - b1) * g[p];
    float v = b2 * vv[p] + (1.f - b2) * g[p] * g[p];
    mm[p] = m;
    vv[p] = v;
    float mh = m / (1.f - powf(b1, (float)step));
    float vh = v / (1.f - powf(b2, (float)step));
    w[p] -= lr * mh / (sqrtf(vh) + e);
}

}  // namespace



cudaError_t sj_launch_mlp_infer(const float *feat, uint32_t nCells, const float *weights, float *out, cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_mlp_infer<<<(nCells + 127) / 128, 128, 0, s>>>(feat, nCells, weights, out); sj_note_launch();
    return cudaGetLastError();
}

// Scratch for one training/gradient call: H1, G1, H2, G2 (m x 64 each), G3 (m x 2).
static cudaError_t mlp_grad_impl(const float *x, const float *y, uint32_t m, const float *w, float *grad,
                                 float *lossOut, cudaStream_t s)
{
    float *buf = nullptr;
    size_t per = (size_t)m * (4 * SJ_HID + SJ_NOUT);
    cudaError_t e = cudaMallocAsync((void **)&buf, per * sizeof(float), s);
    if (e != cudaSuccess) return e;
    float *H1 = buf, *G1 = H1 + (size_t)m * SJ_HID, *H2 = G1 + (size_t)m * SJ_HID, *G2 = H2 + (size_t)m * SJ_HID,
          *G3 = G2 + (size_t)m * SJ_HID;
    cudaMemsetAsync(lossOut, 0, sizeof(float), s);
    k_mlp_backprop<<<(m + 127) / 128, 128, 0, s>>>(x, y, m, w, H1, G1, H2, G2, G3, lossOut); sj_note_launch();
    k_mlp_wgrad<<<(NP + 255) / 256, 256, 0, s>>>(x, H1, H2, G1, G2, G3, m, grad); sj_note_launch();
    e = cudaGetLastError();
    cudaFreeAsync(buf, s);
    return e;
}

cudaError_t sj_launch_mlp_grad(const float *x, const float *y, uint32_t m, const float *weights, float *grad,
                               float *lossOut, cudaStream_t s)
{
    return mlp_grad_impl(x, y, m, weights, grad, lossOut, s);
}

cudaError_t sj_launch_mlp_train_step(const float *x, const float *y, uint32_t m, float *weights, float *grad,
                                     float *adamM, float *adamV, int step, float lr, float *lossOut, cudaStream_t s)
{
    cudaError_t e = mlp_grad_impl(x, y, m, weights, grad, lossOut, s);
    if (e != cudaSuccess) return e;
    k_adam<<<(NP + 255) / 256, 256, 0, s>>>(weights, grad, adamM, adamV, step, lr); sj_note_launch();
    return cudaGetLastError();
}

// ------------------------------------------------- allocation-free gradient --
// Fixed scratch for sj_mlp_loss_grad_noalloc: the per-sample activations and
// gradients (H1, G1, H2, G2 of SJ_HID floats and G3 of SJ_NOUT floats) of at
// most SJ_MLP_NOALLOC_MAX_SAMPLES samples.  Every device that loads this
// library holds it (about 8.5 MB) until the process exits.
static __device__ __align__(256) float g_mlpNoallocScratch[SJ_MLP_NOALLOC_MAX_SAMPLES * (4 * SJ_HID + SJ_NOUT)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noallocMutex;
float *g_noallocScratchPtr[kMaxDevices] = {nullptr};
}  // namespace

extern "C" sj_status sj_mlp_loss_grad_noalloc(const float *x, const float *y, uint32_t m, const float *w, float *loss,
                                              float *grad, void *stream)
{
    if (!x || !y || !w || !loss || !grad || m == 0) {
        sj_set_error_message("sj_mlp_loss_grad_noalloc: null pointer or zero samples");
        return SJ_ERR_BAD_INPUT;
    }
    if (m > SJ_MLP_NOALLOC_MAX_SAMPLES) {
        sj_set_error_message("sj_mlp_loss_grad_noalloc: more samples than the fixed scratch holds "
                             "(limit SJ_MLP_NOALLOC_MAX_SAMPLES = 8192); split the batch");
        return SJ_ERR_BAD_INPUT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        sj_set_error_message("sj_mlp_loss_grad_noalloc: no usable current device");
        return SJ_ERR_CUDA;
    }
    float *scratch;
    {
        // first call on a device: resolve the device address of the scratch
        // array (a host-side name of a __device__ array is not a device pointer)
        std::lock_guard<std::mutex> lock(g_noallocMutex);
        if (!g_noallocScratchPtr[dev]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_mlpNoallocScratch);
            if (e != cudaSuccess || !ptr) {
                sj_set_error_message("sj_mlp_loss_grad_noalloc: cudaGetSymbolAddress failed");
                return SJ_ERR_CUDA;
            }
            g_noallocScratchPtr[dev] = (float *)ptr;
        }
        scratch = g_noallocScratchPtr[dev];
    }
    // an error left pending by earlier work on this thread is reported, not consumed,
    // so the error checks after the launches below see this call's launches only
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        sj_set_error_message("sj_mlp_loss_grad_noalloc: a CUDA error from earlier work is pending");
        return SJ_ERR_CUDA;
    }
    cudaStream_t s = (cudaStream_t)stream;
    float *H1 = scratch, *G1 = H1 + (size_t)m * SJ_HID, *H2 = G1 + (size_t)m * SJ_HID, *G2 = H2 + (size_t)m * SJ_HID,
          *G3 = G2 + (size_t)m * SJ_HID;
    // the loss is accumulated with atomics: it must start at zero; the scratch
    // rows are fully overwritten by every call
    e = cudaMemsetAsync(loss, 0, sizeof(float), s);
    if (e == cudaSuccess) {
        k_mlp_backprop<<<(m + 127) / 128, 128, 0, s>>>(x, y, m, w, H1, G1, H2, G2, G3, loss);
        sj_note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_mlp_wgrad<<<(NP + 255) / 256, 256, 0, s>>>(x, H1, H2, G1, G2, G3, m, grad);
        sj_note_launch();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        sj_set_error_message(cudaGetErrorString(e));
        return SJ_ERR_CUDA;
    }
    return SJ_OK;
}
