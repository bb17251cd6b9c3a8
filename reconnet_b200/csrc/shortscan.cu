// Short-scan redundancy weights for fan-beam FBP (the reference's Python
// ParkerWeighting / RiessWeighting, python/ReconNet_no_tf.py:640-693), as
// device kernels.
//
// A fan-beam scan over beta in [0, pi + 2 gamma] measures some line integrals
// twice.  With the channel's fan angle alpha = ((u - (nu-1)/2) - off_a) * da
// (the sign convention of the reference's weighting functions) and gamma
// taken from the last view angle, gamma = (beta_last - pi) / 2:
//
//  * Parker (D. L. Parker, Med. Phys. 9(2), 1982): w = 1 where the ray is
//    measured once, and sin^2 ramps over the two doubly measured wedges,
//        w = sin^2(pi/4 * beta / (gamma - alpha))                beta < 2 gamma - 2 alpha
//        w = 1                                                   beta <= pi - 2 alpha
//        w = sin^2(pi/4 * (pi + 2 gamma - beta) / (gamma + alpha))  otherwise;
//  * Riess (C. Riess et al., "Novel redundancy weighting for short scans",
//    2013): the same ramps continued past the Parker wedges as 2 - w where
//    the conjugate ray falls outside the scan, then a Gaussian smoothing of
//    each view's weights along the channels (standard deviation sigma
//    channels, taps out to 4 sigma, edge values repeated), except for views
//    with theta < beta < pi + 2 gamma - theta, which keep the unsmoothed
//    weights.
//
// The reference evaluates that exception with
// `np.where(np.all((beta > theta, beta < pi + 2*gamma - theta)))`: np.all
// folds the two conditions into one scalar, so the index set is [0] when both
// hold and empty otherwise -- only channel 0 of those views keeps its
// unsmoothed weight.  riessMask = 0 reproduces that (parity with the
// reference); riessMask = 1 applies the exception to the whole view, the
// behaviour the published method describes.
//
// Parker weights are evaluated in FP64 (the reference uses float64 numpy),
// from FP64 pitch and offset: the Riess continuations jump where a wedge
// ends, so a channel angle rounded to FP32 can move a channel across that
// edge.
// The Riess pre-smoothing weights are rounded to FP32, as the reference
// stores them in a float32 array, and smoothed in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "rn_internal.h"

namespace rn {

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ double sin2(double x) {
    const double s = sin(x);
    return s * s;
}

// One thread per (channel, view); views along grid.y in a loop.
__global__ void parker_weights_kernel(float* __restrict__ w, const float* __restrict__ ang, int nu, int nview,
                                      double da, double off_a) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const double gamma = ((double)ang[nview - 1] - kPi) / 2;
    const double alpha = ((u - (nu - 1) / 2.0) - off_a) * da;
    for (int v = blockIdx.y; v < nview; v += gridDim.y) {
        const double beta = ang[v];
        double r;
        if (beta < 2 * gamma - 2 * alpha) r = sin2(kPi / 4 * beta / (gamma - alpha));
        else if (beta <= kPi - 2 * alpha) r = 1.0;
        else r = sin2(kPi / 4 * (kPi + 2 * gamma - beta) / (gamma + alpha));
        w[(long long)u * nview + v] = (float)r;
    }
}

// One CTA per view: the view's pre-smoothing weights and the Gaussian taps go
// to shared memory, then each thread smooths its channels.
__global__ void riess_weights_kernel(float* __restrict__ w, const float* __restrict__ ang, int nu, int nview,
                                     double da, double off_a, double sigma, int radius, double theta, int mask_all) {
    extern __shared__ double riess_smem[];
    double* taps = riess_smem;                                  // 2 radius + 1
    float* row = reinterpret_cast<float*>(taps + 2 * radius + 1);   // nu
    const double gamma = ((double)ang[nview - 1] - kPi) / 2;
    for (int k = threadIdx.x; k <= 2 * radius; k += blockDim.x) {
        const double x = (k - radius) / sigma;
        taps[k] = exp(-0.5 * x * x);
    }
    __syncthreads();
    __shared__ double tap_sum;
    if (threadIdx.x == 0) {
        double s = 0;
        for (int k = 0; k <= 2 * radius; k++) s += taps[k];
        tap_sum = s;
    }
    __syncthreads();
    const double inv_sum = 1.0 / tap_sum;
    for (int v = blockIdx.x; v < nview; v += gridDim.x) {
        const double beta = ang[v];
        for (int u = threadIdx.x; u < nu; u += blockDim.x) {
            const double alpha = ((u - (nu - 1) / 2.0) - off_a) * da;
            double r = 1.0;   // precedence: first wedge, its continuation, second wedge, its continuation
            if (beta < 2 * gamma - 2 * alpha) r = sin2(kPi / 4 * beta / (gamma - alpha));
            else if (beta < -2 * gamma + 2 * alpha) r = 2.0 - sin2(kPi / 4 * beta / (gamma - alpha));
            else if (beta > kPi - 2 * alpha) r = sin2(kPi / 4 * (kPi + 2 * gamma - beta) / (gamma + alpha));
            else if (beta > kPi + 2 * gamma + 2 * alpha)
                r = 2.0 - sin2(kPi / 4 * (kPi + 2 * gamma - beta) / (gamma + alpha));
            row[u] = (float)r;
        }
        __syncthreads();
        const bool keep = beta > theta && beta < kPi + 2 * gamma - theta;
        for (int u = threadIdx.x; u < nu; u += blockDim.x) {
            float out;
            if (keep && (mask_all || u == 0)) {
                out = row[u];
            } else {
                double acc = 0;
                for (int k = -radius; k <= radius; k++) {
                    const int j = min(max(u + k, 0), nu - 1);
                    acc += taps[k + radius] * (double)row[j];
                }
                out = (float)(acc * inv_sum);
            }
            w[(long long)u * nview + v] = out;
        }
        __syncthreads();
    }
}

int shortscan_weights_device(float* d_w, const float* d_ang, int nu, int nview, double da, double off_a, int kind,
                             double sigma, double theta, int riessMask, cudaStream_t st) {
    if (!d_w || !d_ang) return set_error(RN_ERR_ARG, "shortscan weights: null argument");
    if (nu <= 0 || nview <= 0 || !(da > 0)) return set_error(RN_ERR_ARG, "shortscan weights: sizes and pitch must be positive");
    if (kind == RN_WEIGHT_PARKER) {
        dim3 grid((unsigned)((nu + 255) / 256), (unsigned)std::min(nview, 65535));
        parker_weights_kernel<<<grid, 256, 0, st>>>(d_w, d_ang, nu, nview, da, off_a);
        RN_CUDA_TRY(cudaGetLastError());
        return RN_OK;
    }
    if (kind != RN_WEIGHT_RIESS) return set_error(RN_ERR_ARG, "shortscan weights: kind must be Parker (0) or Riess (1)");
    if (!(sigma > 0)) return set_error(RN_ERR_ARG, "shortscan weights: sigma must be positive");
    // scipy.ndimage.gaussian_filter1d's default reach: radius = int(4 sigma + 0.5)
    const int radius = (int)(4.0 * sigma + 0.5);
    const size_t smem = sizeof(double) * (2 * (size_t)radius + 1) + sizeof(float) * (size_t)nu;
    if (smem > 200 * 1024) return set_error(RN_ERR_ARG, "shortscan weights: too many channels or too wide a smoothing");
    RN_CUDA_TRY(cudaFuncSetAttribute(riess_weights_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    riess_weights_kernel<<<(unsigned)std::min(nview, 65535), 256, smem, st>>>(
        d_w, d_ang, nu, nview, da, off_a, sigma, radius, theta, riessMask ? 1 : 0);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

}  // namespace rn

using namespace rn;

extern "C" int rn_fan_shortscan_weights(float* d_w, const float* d_angles, int nu, int nview, double da, double off_a,
                                        int kind, double sigma, double theta, int riessMask, void* stream) {
    clear_error();
    return shortscan_weights_device(d_w, d_angles, nu, nview, da, off_a, kind, sigma, theta, riessMask,
                                    (cudaStream_t)stream);
}

extern "C" int rn_fan_shortscan_weights_host(float* w, const float* angles, int nu, int nview, double da,
                                             double off_a, int kind, double sigma, double theta, int riessMask) {
    clear_error();
    if (!w || !angles) return set_error(RN_ERR_ARG, "shortscan weights: null argument");
    if (nu <= 0 || nview <= 0) return set_error(RN_ERR_ARG, "shortscan weights: sizes must be positive");
    float* d_w = nullptr;
    float* d_a = nullptr;
    int st = RN_OK;
    const size_t nw = (size_t)nu * nview;
    if (cudaMalloc(&d_w, nw * sizeof(float)) != cudaSuccess || cudaMalloc(&d_a, (size_t)nview * sizeof(float)) != cudaSuccess) {
        st = set_error(RN_ERR_CUDA, "shortscan weights: device allocation failed");
    } else if (cudaMemcpy(d_a, angles, (size_t)nview * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        st = set_error(RN_ERR_CUDA, "shortscan weights: host to device copy failed");
    } else if ((st = shortscan_weights_device(d_w, d_a, nu, nview, da, off_a, kind, sigma, theta, riessMask, 0)) == RN_OK) {
        if (cudaMemcpy(w, d_w, nw * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            st = set_error(RN_ERR_CUDA, "shortscan weights: device to host copy failed");
    }
    if (d_w) cudaFree(d_w);
    if (d_a) cudaFree(d_a);
    return st;
}
