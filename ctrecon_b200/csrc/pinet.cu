// pinet.cu -- the learned PI-line initialiser: a small MLP that predicts each voxel's PI-line
// endpoints as the starting point of the FP64 Newton solve (pi.cu), trained on the GPU by the
// kernels below.
//
// Screw symmetry of the helix: rotating a point by alpha and lifting it by H alpha / 2 pi
// shifts both endpoints by alpha, so with normalised coordinates (x, y, z) = (X/R, Y/R, Z/H),
//   sb - 2 pi z  and  st - 2 pi z  depend only on  r = |(x, y)|  and  psi = atan2(y, x) - 2 pi z.
// On the axis they are -pi/2 and +pi/2. The network maps the features (r / 0.25, cos psi,
// sin psi) to 4 * (sb - 2 pi z + pi/2, st - 2 pi z - pi/2); it is independent of the scan's
// radius, pitch and sampling, and valid for r up to its training radius.
//
// Architecture 3 -> 64 -> 64 -> 64 -> 64 -> 2, SiLU after the hidden layers. Training keeps
// FP32 master weights (Adam); inference (pinet_infer.cu) runs BF16 weights with FP32
// accumulation. Training pairs come from the FP64 Newton solver converged to 1e-11 rad.
#include "internal.h"
#include "pi_device.cuh"
#include "pinet.h"

#include <cmath>
#include <vector>

namespace ctr {

namespace {

__device__ __forceinline__ float silu_f(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double uni(uint64_t k) { return ((k >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

// training pairs: area-uniform points in the disc of radius r_max at z = 0
__global__ void k_pairs(int n, double r_max, uint64_t seed, float* __restrict__ feat,
                        float* __restrict__ targ) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = mix64(seed ^ mix64((uint64_t)i));
    const double r = r_max * sqrt(uni(k));
    const double psi = 2 * kRefPi * uni(mix64(k));
    double sps, cps;
    sincos(psi, &sps, &cps);
    double sb, st;
    int it;
    pi_newton(r * cps, r * sps, 0.0, -0.5 * kRefPi, &sb, &st, &it);
    feat[3 * i + 0] = (float)(r * kPinetRInv);
    feat[3 * i + 1] = (float)cps;
    feat[3 * i + 2] = (float)sps;
    targ[2 * i + 0] = (float)((sb + 0.5 * kRefPi) * kPinetOutScale);
    targ[2 * i + 1] = (float)((st - 0.5 * kRefPi) * kPinetOutScale);
}

constexpr int kTB = 64;  // samples (threads) per block of the training step

// One block = 64 samples: forward, loss, backward, and this block's share of the parameter
// gradient (atomically added to grad). Shared memory holds the weights, the pre-activations
// z_l[i][sample] of the four hidden layers and the back-propagated deltas.
__global__ void __launch_bounds__(kTB) k_train_step(const float* __restrict__ theta,
                                                    const float* __restrict__ feat,
                                                    const float* __restrict__ targ, int n,
                                                    int first, float inv_batch,
                                                    float* __restrict__ grad,
                                                    float* __restrict__ loss) {
    extern __shared__ float sm[];
    float* W = sm;                          // kPinetParams
    float* zs = W + kPinetParamsPad;        // 4 x 64 x kTB
    float* dA = zs + 4 * kPinetH * kTB;     // 64 x kTB (delta of the current layer)
    float* dB = dA + kPinetH * kTB;         // 64 x kTB (delta of the layer below)
    float* a0 = dB + kPinetH * kTB;         // 3 x kTB
    const int t = threadIdx.x;
    for (int i = t; i < kPinetParams; i += kTB) W[i] = theta[i];
    const int s = first + blockIdx.x * kTB + t;
    const bool ok = s < n;
    float x0 = 0, x1 = 0, x2 = 0, y0 = 0, y1 = 0;
    if (ok) {
        x0 = feat[3 * s]; x1 = feat[3 * s + 1]; x2 = feat[3 * s + 2];
        y0 = targ[2 * s]; y1 = targ[2 * s + 1];
    }
    a0[0 * kTB + t] = x0; a0[1 * kTB + t] = x1; a0[2 * kTB + t] = x2;
    __syncthreads();
    // ---- forward
    {
        const float* W1 = W + pinet_offW(0);
        const float* b1 = W + pinet_offB(0);
        for (int o = 0; o < kPinetH; ++o)
            zs[o * kTB + t] = b1[o] + W1[o * 3] * x0 + W1[o * 3 + 1] * x1 + W1[o * 3 + 2] * x2;
    }
    float a[kPinetH];
    for (int l = 1; l < 4; ++l) {
        const float* zin = zs + (l - 1) * kPinetH * kTB;
        float* zout = zs + l * kPinetH * kTB;
#pragma unroll
        for (int i = 0; i < kPinetH; ++i) a[i] = silu_f(zin[i * kTB + t]);
        const float* Wl = W + pinet_offW(l);
        const float* bl = W + pinet_offB(l);
        for (int o = 0; o < kPinetH; ++o) {
            float acc = bl[o];
#pragma unroll
            for (int i = 0; i < kPinetH; ++i) acc = fmaf(Wl[o * kPinetH + i], a[i], acc);
            zout[o * kTB + t] = acc;
        }
    }
    {
        const float* z4 = zs + 3 * kPinetH * kTB;
#pragma unroll
        for (int i = 0; i < kPinetH; ++i) a[i] = silu_f(z4[i * kTB + t]);
    }
    const float* W5 = W + pinet_offW(4);
    const float* b5 = W + pinet_offB(4);
    float o0 = b5[0], o1 = b5[1];
#pragma unroll
    for (int i = 0; i < kPinetH; ++i) {
        o0 = fmaf(W5[i], a[i], o0);
        o1 = fmaf(W5[kPinetH + i], a[i], o1);
    }
    float d0 = ok ? (o0 - y0) : 0.f, d1 = ok ? (o1 - y1) : 0.f;
    float l2 = d0 * d0 + d1 * d1;
    for (int off = 16; off > 0; off >>= 1) l2 += __shfl_down_sync(0xffffffffu, l2, off);
    if ((t & 31) == 0) atomicAdd(loss, l2 * inv_batch);
    const float g0 = 2.f * d0 * inv_batch, g1 = 2.f * d1 * inv_batch;
    // output layer gradient: dW5[k][i] = sum_t g_k(t) a4_i(t); delta4 = W5^T g * silu'(z4)
    {
        const float* z4 = zs + 3 * kPinetH * kTB;
#pragma unroll
        for (int i = 0; i < kPinetH; ++i) {
            float v0 = g0 * a[i], v1 = g1 * a[i];
            for (int off = 16; off > 0; off >>= 1) {
                v0 += __shfl_down_sync(0xffffffffu, v0, off);
                v1 += __shfl_down_sync(0xffffffffu, v1, off);
            }
            if ((t & 31) == 0) {
                atomicAdd(&grad[pinet_offW(4) + i], v0);
                atomicAdd(&grad[pinet_offW(4) + kPinetH + i], v1);
            }
            dA[i * kTB + t] = (W5[i] * g0 + W5[kPinetH + i] * g1) * dsilu_f(z4[i * kTB + t]);
        }
        float v0 = g0, v1 = g1;
        for (int off = 16; off > 0; off >>= 1) {
            v0 += __shfl_down_sync(0xffffffffu, v0, off);
            v1 += __shfl_down_sync(0xffffffffu, v1, off);
        }
        if ((t & 31) == 0) {
            atomicAdd(&grad[pinet_offB(4)], v0);
            atomicAdd(&grad[pinet_offB(4) + 1], v1);
        }
    }
    __syncthreads();
    // hidden layers 4, 3, 2 (index l = 3, 2, 1): dW_l = delta_l a_{l-1}^T over the block's
    // samples (thread o owns row o), then delta_{l-1} = W_l^T delta_l * silu'(z_{l-1})
    float* dcur = dA;
    float* dnext = dB;
    float* aprev = a0 + 3 * kTB;  // 64 x kTB activations of the layer below
    for (int l = 3; l >= 1; --l) {
        const float* zprev = zs + (l - 1) * kPinetH * kTB;
        const float* Wl = W + pinet_offW(l);
        for (int i = 0; i < kPinetH; ++i) aprev[i * kTB + t] = silu_f(zprev[i * kTB + t]);
        __syncthreads();
        {
            const int o = t;  // kTB == kPinetH
            float gb = 0;
            for (int u = 0; u < kTB; ++u) gb += dcur[o * kTB + u];
            atomicAdd(&grad[pinet_offB(l) + o], gb);
            for (int i = 0; i < kPinetH; ++i) {
                float acc = 0;
                for (int u = 0; u < kTB; ++u) acc = fmaf(dcur[o * kTB + u], aprev[i * kTB + u], acc);
                atomicAdd(&grad[pinet_offW(l) + o * kPinetH + i], acc);
            }
        }
        for (int i = 0; i < kPinetH; ++i) {
            float acc = 0;
            for (int o = 0; o < kPinetH; ++o) acc = fmaf(Wl[o * kPinetH + i], dcur[o * kTB + t], acc);
            dnext[i * kTB + t] = acc * dsilu_f(zprev[i * kTB + t]);
        }
        __syncthreads();
        float* tmp = dcur; dcur = dnext; dnext = tmp;
    }
    // first layer: dW1[o][k] = sum_t delta1_o(t) x_k(t)
    {
        const int o = t;
        float gb = 0, gw0 = 0, gw1 = 0, gw2 = 0;
        for (int u = 0; u < kTB; ++u) {
            const float d = dcur[o * kTB + u];
            gb += d;
            gw0 = fmaf(d, a0[u], gw0);
            gw1 = fmaf(d, a0[kTB + u], gw1);
            gw2 = fmaf(d, a0[2 * kTB + u], gw2);
        }
        atomicAdd(&grad[pinet_offB(0) + o], gb);
        atomicAdd(&grad[pinet_offW(0) + o * 3 + 0], gw0);
        atomicAdd(&grad[pinet_offW(0) + o * 3 + 1], gw1);
        atomicAdd(&grad[pinet_offW(0) + o * 3 + 2], gw2);
    }
}

__global__ void k_adam(float* __restrict__ theta, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int n, float lr, float b1, float b2,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1 - b1) * gi;
    const float vi = b2 * v[i] + (1 - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

}  // namespace

// ---- host -----------------------------------------------------------------------------------
static size_t step_smem() {
    return (size_t)(kPinetParamsPad + 4 * kPinetH * kTB + 2 * kPinetH * kTB + 3 * kTB +
                    kPinetH * kTB) * sizeof(float);
}

Status pinet_init_params(std::vector<float>& theta, uint64_t seed) {
    theta.assign(kPinetParams, 0.f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < 5; ++l) {
        const int fan_in = pinet_in(l), fan_out = pinet_out(l);
        const double a = std::sqrt(3.0 / fan_in) * (l == 4 ? 0.1 : 1.0);
        for (int i = 0; i < fan_out * fan_in; ++i) theta[pinet_offW(l) + i] = (float)((2 * next() - 1) * a);
    }
    return Status::Ok();
}

Status pinet_ensure(ctrecon_ctx* ctx) {
    PinetState& P = ctx->pinet;
    if (P.theta.ptr) return Status::Ok();
    CTR_TRY(P.theta.ensure(kPinetParamsPad * sizeof(float), "network parameters"));
    CTR_TRY(P.adam_m.ensure(kPinetParamsPad * sizeof(float), "Adam state"));
    CTR_TRY(P.adam_v.ensure(kPinetParamsPad * sizeof(float), "Adam state"));
    CTR_TRY(P.grad.ensure(kPinetParamsPad * sizeof(float) + 64, "gradient"));
    std::vector<float> th;
    pinet_init_params(th, 12345);
    CTR_TRY(upload_now(P.theta.ptr, th.data(), kPinetParams * sizeof(float)));
    P.trained = false;
    return Status::Ok();
}

// loss and gradient of the current parameters on n samples (no update)
Status pinet_loss_grad(ctrecon_ctx* ctx, cudaStream_t s, const float* d_feat,
                       const float* d_targ, int n, float* d_grad, float* d_loss) {
    CTR_TRY(pinet_ensure(ctx));
    const size_t smem = step_smem();
    CTR_CUDA(cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CTR_CUDA(cudaMemsetAsync(d_grad, 0, kPinetParams * sizeof(float), s));
    CTR_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
    k_train_step<<<(n + kTB - 1) / kTB, kTB, smem, s>>>(ctx->pinet.theta.as<float>(), d_feat,
                                                        d_targ, n, 0, 1.f / n, d_grad, d_loss);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

Status pinet_train(ctrecon_ctx* ctx, cudaStream_t s, int n_pairs, int batch, int epochs,
                   double r_max, uint64_t seed, float* final_loss) {
    if (n_pairs < 1 || batch < 1 || epochs < 1 || !(r_max > 0 && r_max < 1))
        return make_status(CTRECON_ERR_INVALID_ARGUMENT, "pinet_train: bad arguments");
    CTR_TRY(pinet_ensure(ctx));
    PinetState& P = ctx->pinet;
    std::vector<float> th;
    pinet_init_params(th, seed);
    CTR_CUDA(cudaMemcpyAsync(P.theta.ptr, th.data(), kPinetParams * sizeof(float), cudaMemcpyHostToDevice, s));
    CTR_CUDA(cudaMemsetAsync(P.adam_m.ptr, 0, kPinetParams * sizeof(float), s));
    CTR_CUDA(cudaMemsetAsync(P.adam_v.ptr, 0, kPinetParams * sizeof(float), s));
    CTR_TRY(P.data.ensure((size_t)n_pairs * 5 * sizeof(float), "training pairs"));
    float* feat = P.data.as<float>();
    float* targ = feat + (size_t)n_pairs * 3;
    k_pairs<<<(n_pairs + 255) / 256, 256, 0, s>>>(n_pairs, r_max, seed, feat, targ);
    CTR_CUDA(cudaGetLastError());
    const size_t smem = step_smem();
    CTR_CUDA(cudaFuncSetAttribute(k_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    float* grad = P.grad.as<float>();
    float* loss = grad + kPinetParamsPad;
    const int steps_per_epoch = (n_pairs + batch - 1) / batch;
    const int total = steps_per_epoch * epochs;
    const float b1 = 0.9f, b2 = 0.999f, lr0 = 2e-3f, lr1 = 2e-5f;
    int step = 0;
    for (int e = 0; e < epochs; ++e) {
        for (int b = 0; b < steps_per_epoch; ++b, ++step) {
            const int first = b * batch;
            const int nb = std::min(batch, n_pairs - first);
            CTR_CUDA(cudaMemsetAsync(grad, 0, (kPinetParams + 16) * sizeof(float), s));
            k_train_step<<<(nb + kTB - 1) / kTB, kTB, smem, s>>>(P.theta.as<float>(), feat, targ,
                                                                first + nb, first, 1.f / nb, grad,
                                                                loss);
            const double frac = (double)step / std::max(1, total - 1);
            const float lr = (float)(lr1 + 0.5 * (lr0 - lr1) * (1 + std::cos(kRefPi * frac)));
            const int t = step + 1;
            k_adam<<<(kPinetParams + 255) / 256, 256, 0, s>>>(
                P.theta.as<float>(), P.adam_m.as<float>(), P.adam_v.as<float>(), grad,
                kPinetParams, lr, b1, b2, (float)(1 - std::pow(b1, t)), (float)(1 - std::pow(b2, t)));
        }
    }
    CTR_CUDA(cudaGetLastError());
    // final loss over the whole set at the trained parameters
    CTR_TRY(pinet_loss_grad(ctx, s, feat, targ, n_pairs, grad, loss));
    float l = 0;
    CTR_CUDA(cudaMemcpyAsync(&l, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CTR_CUDA(cudaStreamSynchronize(s));
    if (final_loss) *final_loss = l;
    P.r_max = r_max;
    P.trained = true;
    P.version++;
    return Status::Ok();
}

}  // namespace ctr

// ---- C ABI -----------------------------------------------------------------------------------
namespace ctr {
Status pinet_predict(ctrecon_ctx* ctx, cudaStream_t s, const float* d_feat, long long n,
                     float* d_out);
Status launch_pi_stats(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters);
void set_noctx_error(const std::string& m);
}  // namespace ctr

using namespace ctr;

static ctrecon_status pinet_finish(ctrecon_ctx* ctx, const Status& s) {
    if (!s.ok()) {
        if (ctx) ctx->last_error = s.msg;
        else set_noctx_error(s.msg);
    } else if (ctx) {
        ctx->last_error.clear();
    }
    return s.code;
}

#define PINET_GUARD(body)                                                                  \
    try {                                                                                  \
        body                                                                               \
    } catch (const std::exception& e) {                                                    \
        return pinet_finish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));             \
    }

extern "C" {

int ctrecon_pinet_num_params(void) { return kPinetParams; }

ctrecon_status ctrecon_pinet_train(ctrecon_ctx* ctx, void* stream, int n_pairs, int batch,
                                   int epochs, double r_max, uint64_t seed, float* final_loss) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        Status s = cudaSetDevice(ctx->device) == cudaSuccess
                       ? pinet_train(ctx, (cudaStream_t)stream, n_pairs, batch, epochs, r_max,
                                     seed, final_loss)
                       : make_status(CTRECON_ERR_CUDA, "cudaSetDevice failed");
        return pinet_finish(ctx, s);
    })
}

ctrecon_status ctrecon_pinet_get_params(ctrecon_ctx* ctx, float* host, int n) {
    if (!ctx || !host || n < kPinetParams) return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        cudaSetDevice(ctx->device);
        Status s = pinet_ensure(ctx);
        if (s.ok()) {
            // training runs on the caller's stream: wait for all of it
            cudaError_t e = cudaDeviceSynchronize();
            if (e == cudaSuccess)
                e = cudaMemcpy(host, ctx->pinet.theta.ptr, kPinetParams * sizeof(float),
                               cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) s = cuda_status(e, "network parameters");
        }
        return pinet_finish(ctx, s);
    })
}

ctrecon_status ctrecon_pinet_set_params(ctrecon_ctx* ctx, const float* host, int n,
                                        double r_max) {
    if (!ctx || !host || n < kPinetParams) return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        cudaSetDevice(ctx->device);
        Status s = pinet_ensure(ctx);
        if (s.ok()) {
            cudaError_t e = cudaDeviceSynchronize();  // no queued kernel still reads them
            if (e != cudaSuccess) s = cuda_status(e, "network parameters");
            else s = upload_now(ctx->pinet.theta.ptr, host, kPinetParams * sizeof(float));
        }
        if (s.ok()) {
            ctx->pinet.trained = true;
            ctx->pinet.r_max = r_max;
            ctx->pinet.version++;
        }
        return pinet_finish(ctx, s);
    })
}

ctrecon_status ctrecon_pinet_loss_grad(ctrecon_ctx* ctx, void* stream, const float* d_feat,
                                       const float* d_targ, int n, float* d_grad,
                                       float* d_loss) {
    if (!ctx || !d_feat || !d_targ || !d_grad || !d_loss || n < 1)
        return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        cudaSetDevice(ctx->device);
        return pinet_finish(ctx, pinet_loss_grad(ctx, (cudaStream_t)stream, d_feat, d_targ, n,
                                                 d_grad, d_loss));
    })
}

ctrecon_status ctrecon_pinet_predict(ctrecon_ctx* ctx, void* stream, const float* d_feat, int n,
                                     float* d_out) {
    if (!ctx || !d_feat || !d_out || n < 1) return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        cudaSetDevice(ctx->device);
        Status s = reset_device_flag(ctx, (cudaStream_t)stream);
        if (s.ok()) s = pinet_predict(ctx, (cudaStream_t)stream, d_feat, n, d_out);
        return pinet_finish(ctx, s);
    })
}

ctrecon_status ctrecon_pi_dev_stats(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                                    void* d_pitab, unsigned long long* d_updates,
                                    unsigned long long* d_iters) {
    if (!ctx || !g || !d_pitab) return CTRECON_ERR_INVALID_ARGUMENT;
    PINET_GUARD({
        cudaSetDevice(ctx->device);
        BPPlan* plan = nullptr;
        Status s = check_pitab_alignment(d_pitab);
        if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
        if (s.ok()) s = reset_device_flag(ctx, (cudaStream_t)stream);
        if (s.ok())
            s = launch_pi_stats(ctx, (cudaStream_t)stream, *plan, (PiRecord*)d_pitab, d_updates,
                                d_iters);
        return pinet_finish(ctx, s);
    })
}

}  // extern "C"
