// Tomosynthesis distance-driven projector pair (flat detector with detU = x,
// detV = y, main axis z), restating DistanceDrivenTomo::ProjectionTomo /
// BackprojectionTomo (ReconNet4D/DistanceDriven3D.cu:37-663):
//   FP: per ray, for every z plane at integer z, the source-to-detector
//       rectangle [x1,x2] x [y1,y2] spanned by the cell's edge rays is
//       integrated over the piecewise-constant plane (the reference reads 4
//       bilinear corners of a 2D summed-area table), normalised by its area,
//       and the sum is scaled by dz / |dz_src-det| * |src - det|;
//   BP: the sinogram is pre-weighted by the same length factor, and every
//       voxel integrates the detector rectangle spanned by its projected faces.
// The FP integral comes from FP64 row-prefix tables (rows_integral): the rows
// a rectangle overlaps, each weighted by its overlap, the same quantity in
// exact arithmetic as the reference's summed-area-table corner form.  The BP
// reads the FP64 (u, v) summed-area table, as the reference does, with the
// corners shared between neighbouring voxels.  Each (b, c) volume is
// processed by one launch sequence on the caller's stream.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "rn_device.cuh"
#include "rn_internal.h"

namespace rn {

struct TomoDims {
    int nb, nc, nx, ny, nz;
    float dx, dy, dz, cx, cy, cz;
    int nu, nview, nv;
    float du, dv, off_u, off_v;
};

// ---------------------------------------------------------------------------
// Tables (FP64).  FP: per z plane, row prefixes along x of image row y,
// layout [z][y + 1][x] (x fastest, x in [0, nx]); a rectangle integral is the
// sum over the rows it overlaps (rows_integral), which equals the reference's
// summed-area-table corner form.  BP: per view, row prefixes along u of the
// length-weighted projections, layout [view][v + 1][u] (u fastest, u in
// [0, nu]), then summed along v in place (tomo_bp_sat_v) into the (u, v)
// summed-area table.  Rows run along the axis that the lanes of the main
// kernels walk, so their reads are coalesced.
// Row prefixes are built by a tiled pass that reads the source along its
// contiguous axis, transposes 32 x 32 tiles through shared memory and scans
// along the row with warp scans (carry across tiles).
// ---------------------------------------------------------------------------

// Row prefixes R[z][y + 1][x + 1] = sum_{x' <= x} img[x'][y][z].  Block
// (32, 8): blockIdx.x = y, blockIdx.y = a tile of 32 planes.
__global__ void __launch_bounds__(256) tomo_sat_x(double* __restrict__ sat, const float* __restrict__ img, TomoDims d,
                                                  int b, int c) {
    __shared__ float tile[32][33];
    const int y = blockIdx.x, z0 = blockIdx.y * 32;
    const int lane = threadIdx.x, w = threadIdx.y;
    const long long plane = (long long)(d.nx + 1) * (d.ny + 1), row = d.nx + 1;
    const long long sx = (long long)d.ny * d.nz * d.nc;   // img stride along x
    const float* base = img + (long long)b * d.nx * sx + (long long)y * d.nz * d.nc + c;
    double carry[4] = {0.0, 0.0, 0.0, 0.0};
    for (int x0 = 0; x0 < d.nx; x0 += 32) {
#pragma unroll
        for (int k = 0; k < 4; k++) {   // rows x0 + w + 8k, lanes along z (contiguous)
            const int x = x0 + w + 8 * k, z = z0 + lane;
            tile[w + 8 * k][lane] = (x < d.nx && z < d.nz) ? base[(long long)x * sx + (long long)z * d.nc] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; k++) {   // plane z0 + w + 8k, lanes along x
            const int zz = w + 8 * k, z = z0 + zz;
            const double v = (double)tile[lane][zz];
            const double incl = warp_incl_scan(v);
            if (z < d.nz && x0 + lane < d.nx) sat[z * plane + (y + 1) * row + (x0 + lane + 1)] = carry[k] + incl;
            carry[k] += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncthreads();
    }
    // column x = 0 of row y + 1, and row y = 0 of the tile's planes
    const int z = z0 + lane;
    if (w == 0 && z < d.nz) sat[z * plane + (y + 1) * row] = 0.0;
    if (y == 0)
        for (int zz = w; zz < 32 && z0 + zz < d.nz; zz += 8)
            for (int x = lane; x <= d.nx; x += 32) sat[(z0 + zz) * plane + x] = 0.0;
}

// Length weight of detector cell (u, v) of a view (PreweightBPCartKernelXY,
// DistanceDriven3D.cu:409-431).
__device__ __forceinline__ double tomo_len_weight(const float* dc, const float* sp, float u, float v, float dz) {
    const double ddx = (double)sp[0] - (dc[0] + u), ddy = (double)sp[1] - (dc[1] + v), ddz = (double)sp[2] - dc[2];
    return (double)dz / fabs(ddz) * sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
}

// Weighted row prefixes R[view][v + 1][u + 1] = sum_{u' <= u} w p(u', v).
// weight_all = 0 applies the length weight to view 0 only, as the reference's
// pre-weight launch does (its grid has one row of views,
// DistanceDriven3D.cu:612-621); 1 weights every view.  Block (32, 8):
// blockIdx.x = a tile of 32 detector rows v, blockIdx.y = view.
__global__ void __launch_bounds__(256) tomo_bp_sat_u(double* __restrict__ sat, const float* __restrict__ prj,
                                                     const float* __restrict__ detCenter,
                                                     const float* __restrict__ src, TomoDims d, int b, int c,
                                                     int weight_all) {
    __shared__ double tile[32][33];
    const int v0 = blockIdx.x * 32, view = blockIdx.y;
    const int lane = threadIdx.x, w = threadIdx.y;
    const float* dc = detCenter + 3 * view;
    const float* sp = src + 3 * view;
    const bool weighted = weight_all || view == 0;
    const long long vplane = (long long)(d.nu + 1) * (d.nv + 1), row = d.nu + 1;
    double* S = sat + view * vplane;
    const long long su = (long long)d.nview * d.nv * d.nc;   // prj stride along u
    const float* base = prj + (long long)b * d.nu * su + (long long)view * d.nv * d.nc + c;
    double carry[4] = {0.0, 0.0, 0.0, 0.0};
    for (int u0 = 0; u0 < d.nu; u0 += 32) {
#pragma unroll
        for (int k = 0; k < 4; k++) {   // cells u0 + w + 8k, lanes along v (contiguous)
            const int iu = u0 + w + 8 * k, iv = v0 + lane;
            double val = 0.0;
            if (iu < d.nu && iv < d.nv) {
                val = (double)base[(long long)iu * su + (long long)iv * d.nc];
                if (weighted) {
                    const float u = (iu - d.off_u - (d.nu - 1) / 2.0f) * d.du;
                    const float v = (iv - d.off_v - (d.nv - 1) / 2.0f) * d.dv;
                    val *= tomo_len_weight(dc, sp, u, v, d.dz);
                }
            }
            tile[w + 8 * k][lane] = val;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; k++) {   // row v0 + w + 8k, lanes along u
            const int vv = w + 8 * k, iv = v0 + vv;
            const double incl = warp_incl_scan(tile[lane][vv]);
            if (iv < d.nv && u0 + lane < d.nu) S[(iv + 1) * row + (u0 + lane + 1)] = carry[k] + incl;
            carry[k] += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncthreads();
    }
    const int iv = v0 + lane;
    if (w == 0 && iv < d.nv) S[(iv + 1) * row] = 0.0;
    if (blockIdx.x == 0)
        for (int u = lane + 32 * w; u <= d.nu; u += 256) S[u] = 0.0;
}

// In place along v: T[view][k][u] = sum_{k' <= k} R[view][k'][u], the (u, v)
// summed-area table of the weighted projections (row 0 stays 0), the
// quantity of the reference's AccumulateUVAlongVKernel (DistanceDriven3D.cu:459-475).
// A warp scans 32 u columns (lanes along u, coalesced) down all rows, loading
// 8 rows ahead of the running sum.  Block (32, 4): blockIdx.x * 4 + warp = a
// strip of 32 columns, blockIdx.y = view.
__global__ void __launch_bounds__(128) tomo_bp_sat_v(double* __restrict__ sat, TomoDims d) {
    const int u = (blockIdx.x * 4 + threadIdx.y) * 32 + threadIdx.x;
    // the two pad entries after the last view's table (read with weight 0
    // by the backprojection's u + 1 neighbour at u = nu)
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.y == 0 && threadIdx.x < 2)
        sat[(long long)d.nview * (d.nu + 1) * (d.nv + 1) + threadIdx.x] = 0.0;
    if (u > d.nu) return;
    const long long row = d.nu + 1;
    double* T = sat + (long long)blockIdx.y * row * (d.nv + 1) + u;
    double acc = 0.0;
    for (int k0 = 1; k0 <= d.nv; k0 += 8) {
        double v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = k0 + i <= d.nv ? T[(k0 + i) * row] : 0.0;
#pragma unroll
        for (int i = 0; i < 8; i++)
            if (k0 + i <= d.nv) {
                acc += v[i];
                T[(k0 + i) * row] = acc;
            }
    }
}

// Clamp_float + the index / weight of one coordinate of InterpolateXY /
// InterpolateUV (DistanceDriven3D.cu:75-135, :493-517) on a grid of n points.
struct Lerp {
    int i0, i1;
    double w;
};
// The index and the fraction come from a round-down add against 1.5 * 2^23
// (exact for 0 <= x < 2^22) instead of conversions on the XU pipe; a NaN
// coordinate clamps to 0.
__device__ __forceinline__ Lerp lerp_at(float x, int n) {
    x = fminf(fmaxf(x, 0.f), (float)(n - 1));
    const float y = __fadd_rd(x, 12582912.0f);
    Lerp l;
    l.i0 = __float_as_int(y) - 0x4B400000;
    l.i1 = min(l.i0 + 1, n - 1);
    l.w = (double)(x - (y - 12582912.0f));
    return l;
}
// Integral over [y1, y2] (clamped to [0, n]; the result changes sign when
// y2 < y1) of the row prefixes of a table R[row j + 1][col], interpolated
// linearly at the column lc: the summed-area-table difference S(c, y2) -
// S(c, y1) written as the rows that [y1, y2] overlaps, each weighted by its
// overlap.  Equal to the bilinear corner form of InterpolateXY / UV in exact
// arithmetic, with one or two rows instead of four corner reads.
__device__ __forceinline__ double rows_integral(const double* __restrict__ R, const Lerp& lc, float y1, float y2, int n,
                                                long long row) {
    float lo = fminf(y1, y2), hi = fmaxf(y1, y2);
    lo = fminf(fmaxf(lo, 0.f), (float)n);
    hi = fminf(fmaxf(hi, 0.f), (float)n);
    double acc = 0.0;
    // rows j < n overlapped by [lo, hi]; j and its float value fj from a
    // round-down add, as in lerp_at
    const float y = __fadd_rd(lo, 12582912.0f);
    float fj = y - 12582912.0f;
    const double* r = R + (long long)(__float_as_int(y) - 0x4B400000 + 1) * row;
#pragma unroll 4
    for (; fj < hi; fj += 1.f, r += row) {
        const float ov = fminf(hi, fj + 1.f) - fmaxf(lo, fj);
        acc += (r[lc.i0] * (1 - lc.w) + r[lc.i1] * lc.w) * (double)ov;
    }
    return y2 >= y1 ? acc : -acc;
}

// FP: lane i of a warp owns detector column iu = 31 blockIdx.x + i and its
// left cell edge; lane 31 only supplies the right edge of lane 30's cell.  A
// warp handles one detector row v of one view, and per z plane each lane
// evaluates D = S(x_e, y2) - S(x_e, y1) at its edge from the rows [y1, y2]
// overlaps, so the rectangle integral of a cell is D(next lane) - D(this
// lane): two reads per overlapped row instead of the reference's 16 corner
// reads.  The rectangle's area is (x_{e+1} - x_e)(y2 - y1) = drx dry
// (z - sz)^2, exact for the straight edge rays.
__global__ void __launch_bounds__(128) tomo_fp_kernel(float* __restrict__ prj, const double* __restrict__ sat,
                                                      const float* __restrict__ detCenter,
                                                      const float* __restrict__ src, TomoDims d, int b, int c) {
    const int lane = threadIdx.x;
    const int iu = blockIdx.x * 31 + lane;
    const int iview = blockIdx.y;
    const int iv = blockIdx.z * blockDim.y + threadIdx.y;
    if (iv >= d.nv) return;   // warp-uniform
    const float* dc = detCenter + 3 * iview;
    const float* sp = src + 3 * iview;
    const float u = (iu - d.off_u - (d.nu - 1) / 2.0f) * d.du;
    const float v = (iv - d.off_v - (d.nv - 1) / 2.0f) * d.dv;
    auto img_x = [&](float px) { return (px - d.cx) / d.dx + d.nx / 2.0f; };
    auto img_y = [&](float py) { return (py - d.cy) / d.dy + d.ny / 2.0f; };
    auto img_z = [&](float pz) { return (pz - d.cz) / d.dz + d.nz / 2.0f; };
    const float sx = img_x(sp[0]), sy = img_y(sp[1]), sz = img_z(sp[2]);
    const float zd = img_z(dc[2]);
    const float xe = img_x(dc[0] + u - d.du / 2);
    const float ya = img_y(dc[1] + v - d.dv / 2), yb = img_y(dc[1] + v + d.dv / 2);
    const float rxe = (xe - sx) / (zd - sz);
    const float rya = (ya - sy) / (zd - sz), ryb = (yb - sy) / (zd - sz);
    const float drx = __shfl_down_sync(0xffffffffu, rxe, 1) - rxe;   // signed, as are D and dry
    const float k = 1.0f / (drx * (ryb - rya));
    const long long plane = (long long)(d.nx + 1) * (d.ny + 1), row = d.nx + 1;
    float val = 0.f;
    for (int iz = 0; iz < d.nz; iz++) {
        const float t = (float)iz - sz;
        const Lerp lx = lerp_at(sx + rxe * t, d.nx + 1);
        const double D = rows_integral(sat + iz * plane, lx, sy + rya * t, sy + ryb * t, d.ny, row);
        const double q = __shfl_down_sync(0xffffffffu, D, 1) - D;
        val = fmaf((float)q, __fdividef(k, t * t), val);
    }
    if (lane < 31 && iu < d.nu) {
        val *= (float)tomo_len_weight(dc, sp, u, v, d.dz);
        prj[(long long)b * d.nu * d.nview * d.nv * d.nc + ((long long)iu * d.nview + iview) * d.nv * d.nc +
            (long long)iv * d.nc + c] = val;
    }
}

// BP: lane i of a warp owns voxel column ix = 31 blockIdx.y + i and its left
// face; lane 31 only supplies the right face of lane 30's voxel.  A warp
// handles kTomoBpRows consecutive voxels y0 .. y0 + 7 of one z plane.  Per
// view each lane evaluates the (u, v) summed-area table T of the weighted
// projections, bilinearly (InterpolateUV, DistanceDriven3D.cu:493-517), at
// its face's detector coordinate u_e (ProjectConeToDetCart, :478-489) and the
// detector coordinates f_0 .. f_8 of the 8 voxels' v faces (the same for
// every lane of the warp): D_j = T(u_e, f_(j+1)) - T(u_e, f_j), and the
// voxel's rectangle integral is D_j(next lane) - D_j(this lane), divided by
// its area r^2 dx dy / (du dv).  The reference reads 4 corners of 4 bilinear
// samples per voxel and view; sharing corners between neighbouring voxels
// in x (shuffles) and in y (the face between them) leaves 4 table reads per
// voxel and view, all independent of one another.
constexpr int kTomoBpRows = 8;

__global__ void __launch_bounds__(256) tomo_bp_kernel(float* __restrict__ img, const double* __restrict__ sat,
                                                      const float* __restrict__ detCenter,
                                                      const float* __restrict__ src, TomoDims d, int b, int c) {
    // z runs fastest over the grid, so the CTAs resident at a time cover few
    // (x, y) columns and their detector footprints in all views stay in L2
    const int lane = threadIdx.x;
    const int iz = blockIdx.x;
    const int ix = blockIdx.y * 31 + lane;
    const int y0 = (blockIdx.z * blockDim.y + threadIdx.y) * kTomoBpRows;
    if (y0 >= d.ny) return;   // warp-uniform
    const int ny_w = min(kTomoBpRows, d.ny - y0);
    const float xf = (ix - (d.nx - 1) / 2.0f) * d.dx + d.cx - d.dx / 2;
    const float yb = (y0 - (d.ny - 1) / 2.0f) * d.dy + d.cy - d.dy / 2;   // lower face of voxel y0
    const float z = (iz - (d.nz - 1) / 2.0f) * d.dz + d.cz;
    const float cu = d.off_u + (d.nu - 1) / 2.0f, cv = d.off_v + (d.nv - 1) / 2.0f;
    const float aunit = d.dx * d.dy / (d.du * d.dv);
    const float idu = 1.0f / d.du, idv = 1.0f / d.dv;
    const long long vplane = (long long)(d.nu + 1) * (d.nv + 1);
    const int row = d.nu + 1;
    float acc[kTomoBpRows];
#pragma unroll
    for (int j = 0; j < kTomoBpRows; j++) acc[j] = 0.f;
    for (int view = 0; view < d.nview; view++) {
        const float* dc = detCenter + 3 * view;
        const float* sp = src + 3 * view;
        const float r = (dc[2] - sp[2]) / (z - sp[2]);
        const float ue = fmaf(sp[0] - dc[0] + r * (xf - sp[0]), idu, cu);
        const float ov0 = sp[1] - dc[1], wgt = __fdividef(1.0f, r * r * aunit);
        // u_e clamped to [0, nu]: column iu and its neighbour iu + 1 with
        // weight wu (at u_e = nu the neighbour is the next row's zero column
        // or a pad entry, with weight 0)
        const float uc = fminf(fmaxf(ue, 0.f), (float)d.nu);
        const float uy = __fadd_rd(uc, 12582912.0f);
        const double wu = (double)(uc - (uy - 12582912.0f)), wu1 = 1.0 - wu;
        const double* Tu = sat + view * vplane + (__float_as_int(uy) - 0x4B400000);
        // T(u_e, f_j) at the lower face of voxel y0 + j, from table rows k0
        // and k1 = k0 + 1 (clamped); a face whose k0 is the previous face's
        // k1 (the row index is the same for the whole warp) reuses that row
        int kp = -1;
        double ep = 0.0;
        auto tface = [&](int j) {
            const float f = fmaf(ov0 + r * (fmaf((float)j, d.dy, yb) - sp[1]), idv, cv);
            const Lerp lv = lerp_at(f, d.nv + 1);
            double a;
            if (lv.i0 == kp) {
                a = ep;
            } else {
                const double* t0 = Tu + lv.i0 * row;
                a = t0[0] * wu1 + t0[1] * wu;
            }
            const double* t1 = Tu + lv.i1 * row;
            const double e = t1[0] * wu1 + t1[1] * wu;
            kp = lv.i1;
            ep = e;
            return fma(e - a, lv.w, a);
        };
        double tprev = tface(0);
#pragma unroll
        for (int j = 0; j < kTomoBpRows; j++) {
            if (j < ny_w) {   // warp-uniform
                const double t = tface(j + 1);
                const double D = t - tprev;
                const double q = __shfl_down_sync(0xffffffffu, D, 1) - D;
                acc[j] = fmaf((float)q, wgt, acc[j]);
                tprev = t;
            }
        }
    }
    if (lane < 31 && ix < d.nx) {
        float* out = img + (long long)b * d.nx * d.ny * d.nz * d.nc + (((long long)ix * d.ny + y0) * d.nz + iz) * d.nc + c;
#pragma unroll
        for (int j = 0; j < kTomoBpRows; j++)
            if (j < ny_w) out[(long long)j * d.nz * d.nc] = acc[j];
    }
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
            tomo_sat_x<<<dim3(d.ny, (d.nz + 31) / 32), dim3(32, 8), 0, st>>>(d_sat, d_img, d, b, c);
            dim3 blk(32, 4);
            dim3 grd((d.nu + 30) / 31, d.nview, (d.nv + 3) / 4);
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
            tomo_bp_sat_u<<<dim3((d.nv + 31) / 32, d.nview), dim3(32, 8), 0, st>>>(d_sat, d_prj, d_dc, d_src, d, b,
                                                                                    c, weight_all);
            tomo_bp_sat_v<<<dim3((d.nu + 1 + 127) / 128, d.nview), dim3(32, 4), 0, st>>>(d_sat, d);
            dim3 blk(32, 8);
            dim3 grd(d.nz, (d.nx + 30) / 31, (d.ny + 8 * kTomoBpRows - 1) / (8 * kTomoBpRows));
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
    size_t nsat = fp ? (size_t)d.nz * (d.nx + 1) * (d.ny + 1) : (size_t)d.nview * (d.nu + 1) * (d.nv + 1) + 2;
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
    if (bp_bytes) *bp_bytes = ((size_t)nview * (nu + 1) * (nv + 1) + 2) * 8;   // + 2 pad entries
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
