// Isotropic total-variation surrogate of the prior solver
// (PriorFunctionSolver/TVSQS.cu): the first and second derivatives of the
// separable quadratic surrogate of sum_p sqrt(|grad x|^2 + eps) with backward
// differences, in 2D (TVSQS.cu:8-93) and 3D (:160-265).
//
// For voxel p with backward differences d_k = x_p - x_{p - e_k} (0 on the low
// border) and forward differences f_k = x_p - x_{p + e_k} (0 on the high
// border):
//   var_p = sqrt(sum_k d_k^2 + eps)
//   s1_p  = sum_k d_k / var_p + sum_k f_k / var_{p + e_k}
//   s2_p  = ndim / var_p      + sum_k 1 / var_{p + e_k}
// where var_{p + e_k} is replaced by var_p on the high border.  The reference
// writes var in one launch and reads it back in a second; here one pass
// recomputes the neighbours' var from the image (a 13-point stencil in 3D,
// 7 in 2D, served by L1), so DRAM sees one read of the image and the three
// writes.
#include <cuda_runtime.h>

#include <algorithm>

#include "rn_internal.h"

namespace rn {

template <int kDims>
__global__ void tv_iso_kernel(float* __restrict__ s1, float* __restrict__ s2, float* __restrict__ var,
                              const float* __restrict__ img, int nx, int ny, int nz, int nc, long long n,
                              float eps) {
    const long long sz = nc, sy = (long long)nz * nc, sx = (long long)ny * sy;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        long long q = i / nc;
        const int z = (int)(q % nz);
        q /= nz;
        const int y = (int)(q % ny);
        q /= ny;
        const int x = (int)(q % nx);
        const float* p = img + i;
        // var at p + (ox, oy, oz) (offsets 0 or +1), given its value xo
        auto var_at = [&](int ox, int oy, int oz, float xo) -> float {
            const float* c = p + ox * sx + oy * sy + oz * sz;
            float s = 0.f;
            if (x + ox > 0) {
                const float d = xo - __ldg(c - sx);
                s = fmaf(d, d, s);
            }
            if (y + oy > 0) {
                const float d = xo - __ldg(c - sy);
                s = fmaf(d, d, s);
            }
            if (kDims == 3 && z + oz > 0) {
                const float d = xo - __ldg(c - sz);
                s = fmaf(d, d, s);
            }
            return sqrtf(s + eps);
        };
        const float x0 = __ldg(p);
        const float v = var_at(0, 0, 0, x0);
        const float dx0 = x > 0 ? x0 - __ldg(p - sx) : 0.f;
        const float dy0 = y > 0 ? x0 - __ldg(p - sy) : 0.f;
        const float dz0 = (kDims == 3 && z > 0) ? x0 - __ldg(p - sz) : 0.f;
        float a = (dx0 + dy0 + dz0) / v, b = (float)kDims / v;
        if (x < nx - 1) {
            const float xp = __ldg(p + sx);
            const float vx = var_at(1, 0, 0, xp);
            a += (x0 - xp) / vx;
            b += 1.f / vx;
        } else {
            b += 1.f / v;
        }
        if (y < ny - 1) {
            const float yp = __ldg(p + sy);
            const float vy = var_at(0, 1, 0, yp);
            a += (x0 - yp) / vy;
            b += 1.f / vy;
        } else {
            b += 1.f / v;
        }
        if (kDims == 3) {
            if (z < nz - 1) {
                const float zp = __ldg(p + sz);
                const float vz = var_at(0, 0, 1, zp);
                a += (x0 - zp) / vz;
                b += 1.f / vz;
            } else {
                b += 1.f / v;
            }
        }
        s1[i] = a;
        s2[i] = b;
        if (var) var[i] = v;
    }
}

}  // namespace rn

using namespace rn;

extern "C" {

int rn_tv_iso_sqs(float* d_s1, float* d_s2, float* d_var, const float* d_img, int nb, int nx, int ny, int nz, int nc,
                  float eps, int ndim, void* stream) {
    clear_error();
    if (!d_s1 || !d_s2 || !d_img) return set_error(RN_ERR_ARG, "null argument");
    if (nb <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || nc <= 0) return set_error(RN_ERR_ARG, "sizes must be positive");
    if (ndim != 2 && ndim != 3) return set_error(RN_ERR_ARG, "ndim must be 2 or 3");
    if (ndim == 2 && nz != 1) return set_error(RN_ERR_ARG, "2D total variation takes nz = 1");
    const long long n = (long long)nb * nx * ny * nz * nc;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    cudaStream_t st = (cudaStream_t)stream;
    if (ndim == 2)
        tv_iso_kernel<2><<<blocks, 256, 0, st>>>(d_s1, d_s2, d_var, d_img, nx, ny, 1, nc, n, eps);
    else
        tv_iso_kernel<3><<<blocks, 256, 0, st>>>(d_s1, d_s2, d_var, d_img, nx, ny, nz, nc, n, eps);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

int rn_tv_iso_sqs_host(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nz, int nc,
                       float eps, int ndim) {
    clear_error();
    if (!s1 || !s2 || !var || !img) return set_error(RN_ERR_ARG, "null argument");
    if (nb <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || nc <= 0) return set_error(RN_ERR_ARG, "sizes must be positive");
    const size_t n = (size_t)nb * nx * ny * nz * nc;
    float* d = nullptr;
    RN_CUDA_TRY(cudaMalloc(&d, n * 4 * sizeof(float)));
    cudaStream_t st = nullptr;
    int s = RN_OK;
    cudaError_t e = cudaMemcpyAsync(d, img, n * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) s = set_cuda_error(e, "copy to device");
    if (s == RN_OK) s = rn_tv_iso_sqs(d + n, d + 2 * n, d + 3 * n, d, nb, nx, ny, nz, nc, eps, ndim, st);
    if (s == RN_OK) {
        cudaMemcpyAsync(s1, d + n, n * sizeof(float), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(s2, d + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(var, d + 3 * n, n * sizeof(float), cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = set_cuda_error(e, "rn_tv_iso_sqs_host");
    }
    cudaFree(d);
    return s;
}

}  // extern "C"
