// Tomosynthesis distance-driven projector pair (flat detector with detU = x,
// detV = y, main axis z), restating DistanceDrivenTomo::ProjectionTomo /
// BackprojectionTomo (ReconNet4D/DistanceDriven3D.cu:37-663):
//   FP: per ray, for every z plane at integer z, the source-to-detector
//       rectangle [x1,x2] x [y1,y2] spanned by the cell's edge rays is
//       integrated with a 2D summed-area table (4 bilinear corner lookups),
//       normalised by its area, and the sum is scaled by
//       dz / |dz_src-det| * |src - det|;
//   BP: the sinogram is pre-weighted by the same length factor, a (u, v)
//       summed-area table is built per view, and every voxel integrates the
//       detector rectangle spanned by its projected faces.
// The summed-area tables are FP64 (as in the reference) so that corner
// differences keep full precision; each (b, c) volume is processed by one
// launch sequence on the caller's stream.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "rn_internal.h"

namespace rn {

struct TomoDims {
    int nb, nc, nx, ny, nz;
    float dx, dy, dz, cx, cy, cz;
    int nu, nview, nv;
    float du, dv, off_u, off_v;
};

// SAT of one (b, c) volume, layout [z][x][y] with x in [0,nx], y in [0,ny].
__global__ void tomo_sat_rows(double* __restrict__ sat, const float* __restrict__ img, TomoDims d, int b, int c) {
    // one thread per (z, x): prefix along y for image column x (into row x+1)
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nz * d.nx) return;
    int z = i / d.nx, x = i - (i / d.nx) * d.nx;
    double* row = sat + ((long long)z * (d.nx + 1) + (x + 1)) * (d.ny + 1);
    const float* src = img + (long long)b * d.nx * d.ny * d.nz * d.nc + (long long)x * d.ny * d.nz * d.nc +
                       (long long)z * d.nc + c;
    double acc = 0.0;
    row[0] = 0.0;
    for (int y = 0; y < d.ny; y++) {
        acc += (double)src[(long long)y * d.nz * d.nc];
        row[y + 1] = acc;
    }
    if (x == 0) {
        double* r0 = sat + (long long)z * (d.nx + 1) * (d.ny + 1);
        for (int y = 0; y <= d.ny; y++) r0[y] = 0.0;
    }
}

__global__ void tomo_sat_cols(double* __restrict__ sat, TomoDims d) {
    // one thread per (z, y): prefix along x
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nz * (d.ny + 1)) return;
    int z = i / (d.ny + 1), y = i - (i / (d.ny + 1)) * (d.ny + 1);
    double* base = sat + (long long)z * (d.nx + 1) * (d.ny + 1) + y;
    double acc = 0.0;
    for (int x = 1; x <= d.nx; x++) {
        acc += base[(long long)x * (d.ny + 1)];
        base[(long long)x * (d.ny + 1)] = acc;
    }
}

// Clamp_float + bilinear interpolation of InterpolateXY / InterpolateUV
// (DistanceDriven3D.cu:75-135, :493-517) on an (n0 x n1) grid, row stride s0.
__device__ __forceinline__ double sat_bilinear(const double* __restrict__ a, float x, float y, int n0, int n1,
                                               long long s0) {
    x = x < 0.f ? 0.f : (x >= (float)n0 ? (float)(n0 - 1) : x);
    y = y < 0.f ? 0.f : (y >= (float)n1 ? (float)(n1 - 1) : y);
    int i0 = (int)x, j0 = (int)y;
    int i1 = min(i0 + 1, n0 - 1), j1 = min(j0 + 1, n1 - 1);
    double wx = (double)(x - (float)i0), wy = (double)(y - (float)j0);
    return a[i0 * s0 + j0] * (1 - wx) * (1 - wy) + a[i1 * s0 + j0] * wx * (1 - wy) + a[i0 * s0 + j1] * (1 - wx) * wy +
           a[i1 * s0 + j1] * wx * wy;
}

__global__ void tomo_fp_kernel(float* __restrict__ prj, const double* __restrict__ sat,
                               const float* __restrict__ detCenter, const float* __restrict__ src, TomoDims d, int b,
                               int c) {
    int iu = blockIdx.x * blockDim.x + threadIdx.x;
    int iview = blockIdx.y;
    int iv = blockIdx.z * blockDim.y + threadIdx.y;
    if (iu >= d.nu || iv >= d.nv) return;
    const float* dc = detCenter + 3 * iview;
    const float* sp = src + 3 * iview;
    float u = (iu - d.off_u - (d.nu - 1) / 2.0f) * d.du;
    float v = (iv - d.off_v - (d.nv - 1) / 2.0f) * d.dv;
    auto img_x = [&](float px) { return (px - d.cx) / d.dx + d.nx / 2.0f; };
    auto img_y = [&](float py) { return (py - d.cy) / d.dy + d.ny / 2.0f; };
    auto img_z = [&](float pz) { return (pz - d.cz) / d.dz + d.nz / 2.0f; };
    float sx = img_x(sp[0]), sy = img_y(sp[1]), sz = img_z(sp[2]);
    float xa = img_x(dc[0] + u - d.du / 2), xb = img_x(dc[0] + u + d.du / 2);
    float ya = img_y(dc[1] + v - d.dv / 2), yb = img_y(dc[1] + v + d.dv / 2);
    float zd = img_z(dc[2]);
    if (xa > xb) { float t = xa; xa = xb; xb = t; }
    if (ya > yb) { float t = ya; ya = yb; yb = t; }
    float rx1 = (xa - sx) / (zd - sz), rx2 = (xb - sx) / (zd - sz);
    float ry1 = (ya - sy) / (zd - sz), ry2 = (yb - sy) / (zd - sz);
    const long long plane = (long long)(d.nx + 1) * (d.ny + 1);
    double val = 0.0;
    for (int iz = 0; iz < d.nz; iz++) {
        float x1 = sx + rx1 * (iz - sz), x2 = sx + rx2 * (iz - sz);
        float y1 = sy + ry1 * (iz - sz), y2 = sy + ry2 * (iz - sz);
        const double* a = sat + iz * plane;
        double q = sat_bilinear(a, x2, y2, d.nx + 1, d.ny + 1, d.ny + 1) +
                   sat_bilinear(a, x1, y1, d.nx + 1, d.ny + 1, d.ny + 1) -
                   sat_bilinear(a, x2, y1, d.nx + 1, d.ny + 1, d.ny + 1) -
                   sat_bilinear(a, x1, y2, d.nx + 1, d.ny + 1, d.ny + 1);
        val += q / ((double)(x2 - x1) * (double)(y2 - y1));
    }
    double ddx = (double)sp[0] - (dc[0] + u), ddy = (double)sp[1] - (dc[1] + v), ddz = (double)sp[2] - dc[2];
    val *= (double)d.dz / fabs(ddz) * sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
    prj[(long long)b * d.nu * d.nview * d.nv * d.nc + ((long long)iu * d.nview + iview) * d.nv * d.nc +
        (long long)iv * d.nc + c] = (float)val;
}

// Weighted (u, v) SAT per view, layout [view][u in 0..nu][v in 0..nv].
// weight_all = 0 applies the length weight to view 0 only, as the reference's
// pre-weight launch does (its grid has one row of views,
// DistanceDriven3D.cu:612-621); 1 weights every view.
__global__ void tomo_bp_sat_u(double* __restrict__ sat, const float* __restrict__ prj,
                              const float* __restrict__ detCenter, const float* __restrict__ src, TomoDims d, int b,
                              int c, int weight_all) {
    // one thread per (view, v): prefix along u of the weighted projections
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nview * d.nv) return;
    int view = i / d.nv, iv = i - (i / d.nv) * d.nv;
    const float* dc = detCenter + 3 * view;
    const float* sp = src + 3 * view;
    double* base = sat + (long long)view * (d.nu + 1) * (d.nv + 1) + (iv + 1);
    double acc = 0.0;
    if (iv == 0)
        for (int u = 0; u <= d.nu; u++) sat[(long long)view * (d.nu + 1) * (d.nv + 1) + (long long)u * (d.nv + 1)] = 0;
    base[0] = 0.0;
    float v = (iv - d.off_v - (d.nv - 1) / 2.0f) * d.dv;
    for (int iu = 0; iu < d.nu; iu++) {
        float u = (iu - d.off_u - (d.nu - 1) / 2.0f) * d.du;
        double ddx = (double)sp[0] - (dc[0] + u), ddy = (double)sp[1] - (dc[1] + v), ddz = (double)sp[2] - dc[2];
        double w = (weight_all || view == 0) ? (double)d.dz / fabs(ddz) * sqrt(ddx * ddx + ddy * ddy + ddz * ddz)
                                             : 1.0;
        acc += w * (double)prj[(long long)b * d.nu * d.nview * d.nv * d.nc +
                               ((long long)iu * d.nview + view) * d.nv * d.nc + (long long)iv * d.nc + c];
        base[(long long)(iu + 1) * (d.nv + 1)] = acc;
    }
}

__global__ void tomo_bp_sat_v(double* __restrict__ sat, TomoDims d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nview * (d.nu + 1)) return;
    double* row = sat + (long long)i * (d.nv + 1);
    double acc = 0.0;
    for (int v = 1; v <= d.nv; v++) {
        acc += row[v];
        row[v] = acc;
    }
}

__global__ void tomo_bp_kernel(float* __restrict__ img, const double* __restrict__ sat,
                               const float* __restrict__ detCenter, const float* __restrict__ src, TomoDims d, int b,
                               int c) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    int iz = blockIdx.z;
    if (ix >= d.nx || iy >= d.ny) return;
    float x = (ix - (d.nx - 1) / 2.0f) * d.dx + d.cx;
    float y = (iy - (d.ny - 1) / 2.0f) * d.dy + d.cy;
    float z = (iz - (d.nz - 1) / 2.0f) * d.dz + d.cz;
    double val = 0.0;
    const long long vstride = (long long)(d.nu + 1) * (d.nv + 1);
    for (int view = 0; view < d.nview; view++) {
        const float* dc = detCenter + 3 * view;
        const float* sp = src + 3 * view;
        // ProjectConeToDetCart (DistanceDriven3D.cu:478-489)
        float r = (dc[2] - sp[2]) / (z - sp[2]);
        float u1 = (sp[0] - dc[0] + r * (x - d.dx / 2 - sp[0])) / d.du + d.off_u + (d.nu - 1) / 2.0f;
        float u2 = (sp[0] - dc[0] + r * (x + d.dx / 2 - sp[0])) / d.du + d.off_u + (d.nu - 1) / 2.0f;
        float v1 = (sp[1] - dc[1] + r * (y - d.dy / 2 - sp[1])) / d.dv + d.off_v + (d.nv - 1) / 2.0f;
        float v2 = (sp[1] - dc[1] + r * (y + d.dy / 2 - sp[1])) / d.dv + d.off_v + (d.nv - 1) / 2.0f;
        const double* a = sat + view * vstride;
        double q = sat_bilinear(a, u2, v2, d.nu + 1, d.nv + 1, d.nv + 1) -
                   sat_bilinear(a, u2, v1, d.nu + 1, d.nv + 1, d.nv + 1) +
                   sat_bilinear(a, u1, v1, d.nu + 1, d.nv + 1, d.nv + 1) -
                   sat_bilinear(a, u1, v2, d.nu + 1, d.nv + 1, d.nv + 1);
        val += q / ((double)(u2 - u1) * (double)(v2 - v1));
    }
    img[(long long)b * d.nx * d.ny * d.nz * d.nc + (((long long)ix * d.ny + iy) * d.nz + iz) * d.nc + c] = (float)val;
}

static int tomo_validate(const TomoDims& d) {
    if (d.nb <= 0 || d.nc <= 0 || d.nx <= 0 || d.ny <= 0 || d.nz <= 0 || d.nu <= 0 || d.nview <= 0 || d.nv <= 0)
        return set_error(RN_ERR_ARG, "tomo: sizes must be positive");
    if (!(d.dx > 0 && d.dy > 0 && d.dz > 0 && d.du > 0 && d.dv > 0))
        return set_error(RN_ERR_ARG, "tomo: pixel and detector sizes must be positive");
    return RN_OK;
}

int tomo_project(float* d_prj, const float* d_img, const float* d_dc, const float* d_src, const TomoDims& d,
                 double* d_sat, cudaStream_t st) {
    RN_TRY(tomo_validate(d));
    for (int b = 0; b < d.nb; b++)
        for (int c = 0; c < d.nc; c++) {
            tomo_sat_rows<<<(d.nz * d.nx + 127) / 128, 128, 0, st>>>(d_sat, d_img, d, b, c);
            tomo_sat_cols<<<(d.nz * (d.ny + 1) + 127) / 128, 128, 0, st>>>(d_sat, d);
            dim3 blk(32, 4);
            dim3 grd((d.nu + 31) / 32, d.nview, (d.nv + 3) / 4);
            tomo_fp_kernel<<<grd, blk, 0, st>>>(d_prj, d_sat, d_dc, d_src, d, b, c);
        }
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

int tomo_backproject(float* d_img, const float* d_prj, const float* d_dc, const float* d_src, const TomoDims& d,
                     double* d_sat, int weight_all, cudaStream_t st) {
    RN_TRY(tomo_validate(d));
    for (int b = 0; b < d.nb; b++)
        for (int c = 0; c < d.nc; c++) {
            tomo_bp_sat_u<<<(d.nview * d.nv + 127) / 128, 128, 0, st>>>(d_sat, d_prj, d_dc, d_src, d, b, c,
                                                                          weight_all);
            tomo_bp_sat_v<<<(d.nview * (d.nu + 1) + 127) / 128, 128, 0, st>>>(d_sat, d);
            dim3 blk(32, 8);
            dim3 grd((d.nx + 31) / 32, (d.ny + 7) / 8, d.nz);
            tomo_bp_kernel<<<grd, blk, 0, st>>>(d_img, d_sat, d_dc, d_src, d, b, c);
        }
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

static TomoDims tomo_dims(int nb, int nc, int nx, int ny, int nz, float dx, float dy, float dz, float cx, float cy,
                          float cz, int nu, int nview, int nv, float du, float dv, float off_u, float off_v) {
    TomoDims d;
    d.nb = nb; d.nc = nc; d.nx = nx; d.ny = ny; d.nz = nz;
    d.dx = dx; d.dy = dy; d.dz = dz; d.cx = cx; d.cy = cy; d.cz = cz;
    d.nu = nu; d.nview = nview; d.nv = nv;
    d.du = du; d.dv = dv; d.off_u = off_u; d.off_v = off_v;
    return d;
}

// Host-call scratch: grow-only device buffers guarded by a mutex.
struct TomoHost {
    std::mutex mu;
    cudaStream_t st = nullptr;
    void* buf[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t cap[5] = {0, 0, 0, 0, 0};
    int ensure(int i, size_t bytes) {
        if (bytes <= cap[i]) return RN_OK;
        if (buf[i]) cudaFree(buf[i]);
        buf[i] = nullptr;
        cap[i] = 0;
        cudaError_t e = cudaMalloc(&buf[i], bytes);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc");
        cap[i] = bytes;
        return RN_OK;
    }
};
static TomoHost g_tomo;

static int host_tomo(bool fp, float* out, const float* in, const float* dc, const float* sp, const TomoDims& d) {
    RN_TRY(tomo_validate(d));
    std::lock_guard<std::mutex> lk(g_tomo.mu);
    if (!g_tomo.st) RN_CUDA_TRY(cudaStreamCreateWithFlags(&g_tomo.st, cudaStreamNonBlocking));
    cudaStream_t st = g_tomo.st;
    size_t ni = (size_t)d.nb * d.nx * d.ny * d.nz * d.nc, np = (size_t)d.nb * d.nu * d.nview * d.nv * d.nc;
    size_t nsat = fp ? (size_t)d.nz * (d.nx + 1) * (d.ny + 1) : (size_t)d.nview * (d.nu + 1) * (d.nv + 1);
    RN_TRY(g_tomo.ensure(0, ni * 4));
    RN_TRY(g_tomo.ensure(1, np * 4));
    RN_TRY(g_tomo.ensure(2, (size_t)d.nview * 12));
    RN_TRY(g_tomo.ensure(3, (size_t)d.nview * 12));
    RN_TRY(g_tomo.ensure(4, nsat * 8));
    float* dimg = (float*)g_tomo.buf[0];
    float* dprj = (float*)g_tomo.buf[1];
    RN_CUDA_TRY(cudaMemcpyAsync(g_tomo.buf[2], dc, (size_t)d.nview * 12, cudaMemcpyHostToDevice, st));
    RN_CUDA_TRY(cudaMemcpyAsync(g_tomo.buf[3], sp, (size_t)d.nview * 12, cudaMemcpyHostToDevice, st));
    if (fp) {
        RN_CUDA_TRY(cudaMemcpyAsync(dimg, in, ni * 4, cudaMemcpyHostToDevice, st));
        RN_TRY(tomo_project(dprj, dimg, (float*)g_tomo.buf[2], (float*)g_tomo.buf[3], d, (double*)g_tomo.buf[4], st));
        RN_CUDA_TRY(cudaMemcpyAsync(out, dprj, np * 4, cudaMemcpyDeviceToHost, st));
    } else {
        RN_CUDA_TRY(cudaMemcpyAsync(dprj, in, np * 4, cudaMemcpyHostToDevice, st));
        RN_TRY(tomo_backproject(dimg, dprj, (float*)g_tomo.buf[2], (float*)g_tomo.buf[3], d, (double*)g_tomo.buf[4],
                                0, st));
        RN_CUDA_TRY(cudaMemcpyAsync(out, dimg, ni * 4, cudaMemcpyDeviceToHost, st));
    }
    RN_CUDA_TRY(cudaStreamSynchronize(st));
    return RN_OK;
}

}  // namespace rn

using namespace rn;

extern "C" {

int rn_tomo_sat_bytes(int nx, int ny, int nz, int nu, int nview, int nv, size_t* fp_bytes, size_t* bp_bytes) {
    if (fp_bytes) *fp_bytes = (size_t)nz * (nx + 1) * (ny + 1) * 8;
    if (bp_bytes) *bp_bytes = (size_t)nview * (nu + 1) * (nv + 1) * 8;
    return RN_OK;
}

int rn_tomo_project(float* d_prj, const float* d_img, const float* d_detCenter, const float* d_src, double* d_sat,
                    int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, float cx,
                    float cy, float cz, int nu, int nview, int nv, float du, float dv, float off_u, float off_v,
                    void* stream) {
    clear_error();
    if (!d_prj || !d_img || !d_detCenter || !d_src || !d_sat) return set_error(RN_ERR_ARG, "null argument");
    return tomo_project(d_prj, d_img, d_detCenter, d_src,
                        tomo_dims(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv,
                                  off_u, off_v),
                        d_sat, (cudaStream_t)stream);
}

int rn_tomo_backproject(float* d_img, const float* d_prj, const float* d_detCenter, const float* d_src, double* d_sat,
                        int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, float cx,
                        float cy, float cz, int nu, int nview, int nv, float du, float dv, float off_u, float off_v,
                        int weightAllViews, void* stream) {
    clear_error();
    if (!d_prj || !d_img || !d_detCenter || !d_src || !d_sat) return set_error(RN_ERR_ARG, "null argument");
    return tomo_backproject(d_img, d_prj, d_detCenter, d_src,
                            tomo_dims(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv,
                                      off_u, off_v),
                            d_sat, weightAllViews ? 1 : 0, (cudaStream_t)stream);
}

void cDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                   int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz,
                                   float cx, float cy, float cz, int nu, int nview, int nv, float du, float dv,
                                   float off_u, float off_v) {
    clear_error();
    if (!prj || !img || !detCenter || !src) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_tomo(true, prj, img, detCenter, src,
              tomo_dims(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v));
}

void cDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                       int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy,
                                       float dz, float cx, float cy, float cz, int nu, int nview, int nv, float du,
                                       float dv, float off_u, float off_v) {
    clear_error();
    if (!prj || !img || !detCenter || !src) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_tomo(false, img, prj, detCenter, src,
              tomo_dims(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v));
}

}  // extern "C"
