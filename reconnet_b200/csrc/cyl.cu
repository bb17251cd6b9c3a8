// Cylindrical-detector cone-beam distance-driven pair on a circular orbit.
//
// The reference has no kernel for this geometry: its DistanceDriven3D.cu
// (DDFPConeKernelXY :139-227, DDBPConeCartKernelXY :519-559) is a flat,
// axis-aligned tomosynthesis pair whose main axis is always z.  This pair
// generalises its rectangle-footprint form and the fan DD geometry
// (DistanceDriven.cu:64-196: fan angle a = (-(u - (nu-1)/2) - off_a) da,
// source (dso sin t, -dso cos t), view classes by |cos t| > |sin t| in float)
// to a 360-degree orbit and a cylindrical detector:
//
//  * X-class views (rays mostly along y) take the voxel rows y = const as
//    planes, Y-class views the columns x = const.  On plane k, cell (u, v)
//    covers the rectangle [l(a_u - da/2), l(a_u + da/2)] x [s_v- dc, s_v+ dc]
//    in (lateral, z): l(a) the in-plane position of the fan ray at angle a,
//    s = height / dsd the rise of a detector-row edge per mm of in-plane
//    distance, dc the in-plane distance of the cell's central ray to the
//    plane.  Per plane the cell adds the mean of the voxels over the
//    rectangle (overlaps in voxel units) times the central ray's path length
//    through the plane's slab, L = dmain sqrt(1 + R_c^2) sqrt(1 + s_c^2).
//  * The backprojection is the exact transpose, in gather form (no atomics).
//
// The FP64 CPU oracle (oracle/oracle.cpp, cyl_view_terms) evaluates the same
// sum voxel by voxel.
//
// Forward projection: the volume's z prefix sums (one FP64-accumulated
// table per call, cyl_zprefix_kernel) turn a row's integral over z on one
// voxel column into the difference of the prefix at its two edges, read with
// linear interpolation inside a voxel.  A warp owns one detector column u
// and 32 rows: its lanes hold the rows' lower edges, and the 33rd edge,
// closing lane 31's row, is evaluated by every lane alongside.  On each
// plane the column's lateral footprint covers 1-3 voxel columns, the same
// for every lane; each lane reads the prefix at its edge on each of them
// (lanes read neighbouring entries of one column: two or three sectors per
// warp), weights it by the lateral overlap, and a row's value is the
// difference of two neighbouring lanes' sums (one shuffle), so every edge is
// evaluated once per plane.
//
// Backprojection: per view, the sinogram column u becomes a row table of
// prefix sums of L p along v (cyl_table_kernel).  The gather runs in
// launches over chunks of views whose tables stay in L2 (each voxel adds its
// chunk's sum to the previous chunks').  A warp owns 128 voxels along z of
// one (x, y) column, four per lane, so the lateral work of a view (the
// voxel's fan-angle range, the candidate cells u whose footprint meets its
// lateral extent on its plane, their overlaps) is done once for the whole
// column and the loop over candidates does not diverge.  For each candidate
// the voxel edges map linearly to detector-row coordinates, the row table
// gives the prefix of L p at each edge, and a voxel's share is the
// difference of its two edges' prefixes (one shuffle).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "rn_internal.h"

namespace rn {

struct CylView {
    double sx, sy;      // source (mm)
    float theta;        // view angle (rad)
    int xcls;           // 1: main axis y (planes are voxel rows y = const)
};

struct CylDims {
    int nb, nx, ny, nz, nu, nview, nv;
    double dx, dy, dz, cx, cy, cz;
    double da, off_a, dv, off_v, dsd;
    long long vol_stride, prj_stride;
};

constexpr int kCylFpWarps = 8;   // detector columns per forward-projection CTA
constexpr int kCylRows = 32;     // detector rows per warp (its 32 lanes' edges and one more)
constexpr int kCylBpWarps = 8;   // voxel columns per backprojection CTA
constexpr int kCylBpZ = 4;       // voxels per lane along z (a warp covers 128)

__device__ __forceinline__ float warp_scan_f(float v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// z prefix sums of the volume, one column (b, x, y) per warp: entry j of
// nz + 1 holds the sum of voxels j' < j, accumulated in FP64.
__global__ void cyl_zprefix_kernel(float* __restrict__ zp, const float* __restrict__ vol, CylDims d) {
    const int lane = threadIdx.x & 31;
    const long long col = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (col >= (long long)d.nb * d.nx * d.ny) return;   // whole warp
    const long long b = col / ((long long)d.nx * d.ny), xy = col % ((long long)d.nx * d.ny);
    const float* v = vol + b * d.vol_stride + xy * d.nz;
    float* o = zp + col * (d.nz + 1);
    double carry = 0;
    for (int j0 = 0; j0 < d.nz; j0 += 32) {
        const int j = j0 + lane;
        double x = j < d.nz ? (double)v[j] : 0.0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += t;
        }
        // inclusive sum up to j -> the prefix before j + 1
        if (j < d.nz) o[j + 1] = (float)(carry + x);
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) o[0] = 0.f;
}

// The prefix of a z column at zeta (voxel units from the volume's bottom),
// linear inside each voxel.
__device__ __forceinline__ float z_prefix(const float* __restrict__ c, float zeta, int nz) {
    if (zeta <= 0.f) return 0.f;
    if (zeta >= (float)nz) return __ldg(c + nz);
    const int m = (int)zeta;
    const float a = __ldg(c + m), b = __ldg(c + m + 1);
    return fmaf(zeta - (float)m, b - a, a);
}

__global__ void __launch_bounds__(32 * kCylFpWarps) cyl_fp_kernel(float* __restrict__ prj,
                                                                 const float* __restrict__ zp,
                                                                 const CylView* __restrict__ views,
                                                                 const double* __restrict__ redge,
                                                                 const float* __restrict__ inplane,
                                                                 const float* __restrict__ sedge,
                                                                 const float* __restrict__ rowlen, CylDims d) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = blockIdx.x * kCylFpWarps + warp;
    if (u >= d.nu) return;                                   // whole warp
    const int g0 = blockIdx.y * kCylRows;
    const int e = g0 + lane;
    const float s_lane = sedge[min(e, d.nv)];
    const float s_top = sedge[min(g0 + 32, d.nv)];           // the 33rd edge, closing lane 31's row
    const float inv_dz = (float)(1.0 / d.dz), zoff = (float)(d.nz / 2.0 - d.cz / d.dz);
    for (int bz = blockIdx.z; bz < d.nview * d.nb; bz += gridDim.z) {
        const int iv = bz % d.nview, b = bz / d.nview;
        const CylView V = views[iv];
        const bool xc = V.xcls != 0;
        const int nplane = xc ? d.ny : d.nx, nlat = xc ? d.nx : d.ny;
        const double dmain = xc ? d.dy : d.dx, dlat = xc ? d.dx : d.dy;
        const double cmain = xc ? d.cy : d.cx, clat = xc ? d.cx : d.cy;
        const double smain = xc ? V.sy : V.sx, slat = xc ? V.sx : V.sy;
        const double R0 = redge[(long long)iv * (d.nu + 1) + u], R1 = redge[(long long)iv * (d.nu + 1) + u + 1];
        const float inp = inplane[(long long)iv * d.nu + u];
        const double inv_dlat = 1.0 / dlat;
        const double lat_off = nlat / 2.0 - clat * inv_dlat;
        // footprint width x in-plane distance: |R1 - R0| inp D^2 / dlat
        const float wfac = (float)(fabs(R1 - R0) * inv_dlat) * inp;
        const float* zb = zp + (long long)b * d.nx * d.ny * (d.nz + 1);
        // the columns of plane k along the lateral axis: x-class planes are
        // rows y = k (columns x = i), y-class planes columns x = k
        const long long cstride = (long long)(xc ? d.ny : 1) * (d.nz + 1);
        const long long pstride = (long long)(xc ? 1 : d.ny) * (d.nz + 1);
        const float szl = s_lane * inp * inv_dz, szt = s_top * inp * inv_dz;
        float acc = 0.f;
        for (int k = 0; k < nplane; k++) {
            const double D = (k + 0.5 - nplane / 2.0) * dmain + cmain - smain;
            const double la = fma(R0, D, slat) * inv_dlat + lat_off, lb = fma(R1, D, slat) * inv_dlat + lat_off;
            const double lo = fmin(la, lb), hi = fmax(la, lb);
            const int i0 = (int)fmax(floor(lo), 0.0), i1 = (int)fmin(floor(hi), (double)(nlat - 1));
            if (i0 > i1) continue;
            const float aD = (float)fabs(D);
            const float zeta = fmaf(szl, aD, zoff);
            const float ztop = fmaf(szt, aD, zoff);
            const float z_first = __shfl_sync(0xffffffffu, zeta, 0);
            if (ztop <= 0.f || z_first >= (float)d.nz) continue;   // every row edge outside the volume
            const float* cp = zb + k * pstride;
            float Q = 0.f, Qt = 0.f;
            for (int i = i0; i <= i1; i++) {
                const float ox = (float)(fmin(hi, i + 1.0) - fmax(lo, (double)i));
                const float* c = cp + i * cstride;
                Q = fmaf(ox, z_prefix(c, zeta, d.nz), Q);
                Qt = fmaf(ox, z_prefix(c, ztop, d.nz), Qt);
            }
            float Qn = __shfl_down_sync(0xffffffffu, Q, 1);
            if (lane == 31) Qn = Qt;
            acc = fmaf(Qn - Q, __frcp_rn(wfac * aD * aD), acc);
        }
        if (e < d.nv) {
            const float ds = sedge[e + 1] - sedge[e];
            const float L = (float)dmain * inp * rowlen[e];
            prj[(long long)b * d.prj_stride + ((long long)u * d.nview + iv) * d.nv + e] = acc * L * (float)d.dz / ds;
        }
    }
}

// Row tables of the backprojection: per (batch, view, column u), entry r of
// nv + 1 holds (sum over rows v < r of L p, L p of row r), built in FP64.
__global__ void cyl_table_kernel(float2* __restrict__ tab, const float* __restrict__ prj, const CylView* __restrict__ views,
                                 const float* __restrict__ inplane, const float* __restrict__ rowlen, CylDims d) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)d.nb * d.nview * d.nu;
    if (t >= n) return;
    const int iv = (int)(t % d.nview);
    const long long r = t / d.nview;
    const int u = (int)(r % d.nu), b = (int)(r / d.nu);
    const double dmain = views[iv].xcls ? d.dy : d.dx;
    const double lu = dmain * inplane[(long long)iv * d.nu + u];
    const float* p = prj + (long long)b * d.prj_stride + ((long long)u * d.nview + iv) * d.nv;
    float2* out = tab + (((long long)b * d.nview + iv) * d.nu + u) * (d.nv + 1);
    double C = 0;
    for (int v = 0; v < d.nv; v++) {
        const double w = lu * rowlen[v] * (double)p[v];
        out[v] = make_float2((float)C, (float)w);
        C += w;
    }
    out[d.nv] = make_float2((float)C, 0.f);
}

__device__ __forceinline__ float row_prefix(const float2* __restrict__ t, float rho, int nv) {
    if (rho <= 0.f) return 0.f;
    if (rho >= (float)nv) return __ldg(&t[nv].x);
    const int r = (int)rho;
    const float2 c = __ldg(&t[r]);
    return fmaf(c.y, rho - (float)r, c.x);
}

__global__ void __launch_bounds__(32 * kCylBpWarps) cyl_bp_kernel(float* __restrict__ vol, const float2* __restrict__ tab,
                                                                 const CylView* __restrict__ views,
                                                                 const double* __restrict__ redge,
                                                                 const double* __restrict__ inv_dr,
                                                                 const float* __restrict__ inv_inp, CylDims d,
                                                                 int v_begin, int v_end, int accumulate) {
    constexpr int Z = kCylBpZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long column = (long long)blockIdx.x * kCylBpWarps + warp;
    if (column >= (long long)d.nx * d.ny) return;              // whole warp
    const int ix = (int)(column / d.ny), iy = (int)(column % d.ny);
    const int b = blockIdx.z;
    const int zbase = blockIdx.y * 32 * Z;
    // z (mm) of the voxel edges zbase + lane + 32 q and of the warp's top edge
    float ze[Z];
#pragma unroll
    for (int q = 0; q < Z; q++) ze[q] = (float)((zbase + lane + 32 * q - d.nz / 2.0) * d.dz + d.cz);
    const float ztop = (float)((zbase + 32 * Z - d.nz / 2.0) * d.dz + d.cz);
    const float zlast = (float)((min(d.nz, zbase + 32 * Z) - d.nz / 2.0) * d.dz + d.cz);
    const float zfirst = (float)((zbase - d.nz / 2.0) * d.dz + d.cz);
    const float rho0 = (float)(d.nv / 2.0 - d.off_v);
    const float dsd_dv = (float)(d.dsd / d.dv);
    const double two_pi = 6.283185307179586;
    float acc[Z];
#pragma unroll
    for (int q = 0; q < Z; q++) acc[q] = 0.f;
    for (int iv = v_begin; iv < v_end; iv++) {
        const CylView V = views[iv];
        const bool xc = V.xcls != 0;
        const int k = xc ? iy : ix, i = xc ? ix : iy;
        const int nplane = xc ? d.ny : d.nx, nlat = xc ? d.nx : d.ny;
        const double dmain = xc ? d.dy : d.dx, dlat = xc ? d.dx : d.dy;
        const double cmain = xc ? d.cy : d.cx, clat = xc ? d.cx : d.cy;
        const double smain = xc ? V.sy : V.sx, slat = xc ? V.sx : V.sy;
        const double pm = (k + 0.5 - nplane / 2.0) * dmain + cmain;
        const double D = pm - smain;
        const double lat0 = (i - nlat / 2.0) * dlat + clat;
        // fan angles of the rays through the voxel's lateral faces -> edge coordinates
        float e01[2];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const double lat = lat0 + q * dlat;
            const float px = (float)((xc ? lat : pm) - V.sx), py = (float)((xc ? pm : lat) - V.sy);
            float a = atan2f(px, py) + V.theta;
            a -= (float)two_pi * rintf(a * (float)(1.0 / two_pi));
            e01[q] = -a / (float)d.da - (float)d.off_a + (d.nu - 1) * 0.5f + 0.5f;
        }
        const float elo = fminf(e01[0], e01[1]) - 0.01f, ehi = fmaxf(e01[0], e01[1]) + 0.01f;
        const int ulo = (int)fmaxf(floorf(elo), 0.f), uhi = (int)fminf(floorf(ehi), (double)(d.nu - 1));
        const double inv_dlat = 1.0 / dlat;
        const double lat_off = nlat / 2.0 - clat * inv_dlat;
        // footprint width on this plane: |R1 - R0| |D| / dlat
        const double wD = dlat / fabs(D);
        const float inv_aD = (float)(1.0 / fabs(D));
        const double* Rv = redge + (long long)iv * (d.nu + 1);
        const float2* tv = tab + ((long long)b * d.nview + iv) * (long long)d.nu * (d.nv + 1);
        for (int u = ulo; u <= uhi; u++) {
            const double la = fma(Rv[u], D, slat) * inv_dlat + lat_off, lb = fma(Rv[u + 1], D, slat) * inv_dlat + lat_off;
            const double lo = fmin(la, lb), hi = fmax(la, lb);
            const double ov = fmin(hi, i + 1.0) - fmax(lo, (double)i);
            if (ov <= 0) continue;
            const float inv = dsd_dv * inv_aD * inv_inp[(long long)iv * d.nu + u];
            // the warp's z run against the detector rows: skip if it misses them
            if (fmaf(zlast, inv, rho0) <= 0.f || fmaf(zfirst, inv, rho0) >= (float)d.nv) continue;
            const float w = (float)(ov * wD * inv_dr[(long long)iv * d.nu + u]);
            const float2* t = tv + (long long)u * (d.nv + 1);
            // prefixes at every edge; a voxel's integral is the next edge's minus its own
            float P[Z];
#pragma unroll
            for (int q = 0; q < Z; q++) P[q] = row_prefix(t, fmaf(ze[q], inv, rho0), d.nv);
            const float Ptop = row_prefix(t, fmaf(ztop, inv, rho0), d.nv);
#pragma unroll
            for (int q = 0; q < Z; q++) {
                float Pn = __shfl_down_sync(0xffffffffu, P[q], 1);
                const float P0 = __shfl_sync(0xffffffffu, q + 1 < Z ? P[q + 1 < Z ? q + 1 : q] : Ptop, 0);
                if (lane == 31) Pn = q + 1 < Z ? P0 : Ptop;
                acc[q] = fmaf(w, Pn - P[q], acc[q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Z; q++) {
        const int j = zbase + lane + 32 * q;
        if (j < d.nz) {
            float* o = vol + (long long)b * d.vol_stride + ((long long)ix * d.ny + iy) * d.nz + j;
            *o = accumulate ? *o + acc[q] : acc[q];
        }
    }
}

}  // namespace rn

using namespace rn;

struct rn_cyl_plan {
    RnCylGeom g;
    CylDims d;
    int device = 0;
    CylView* d_views = nullptr;
    double* d_redge = nullptr;    // [nview][nu+1] lateral slope of each fan edge ray
    float* d_inplane = nullptr;   // [nview][nu] sqrt(1 + R_c^2) of each cell's central ray
    float* d_sedge = nullptr;     // [nv+1] row-edge rise per mm of in-plane distance
    float* d_rowlen = nullptr;    // [nv] sqrt(1 + s_c^2) of each row's central ray
    double* d_invdr = nullptr;    // [nview][nu] 1 / |R_{u+1} - R_u|
    float* d_invinp = nullptr;    // [nview][nu] 1 / sqrt(1 + R_c^2)
    int bp_chunk = 0;             // views per backprojection launch (their row tables stay in L2)
    float2* d_tab = nullptr;      // backprojection row tables [nb][nview][nu][nv+1]
    float* d_zp = nullptr;        // forward-projection z prefix sums [nb][nx][ny][nz+1]
    long long launches = 0;
};

static int cyl_check(const RnCylGeom* g) {
    if (!g) return set_error(RN_ERR_ARG, "cyl: null geometry");
    if (g->nBatches <= 0 || g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->nu <= 0 || g->nview <= 0 || g->nv <= 0)
        return set_error(RN_ERR_ARG, "cyl: sizes must be positive");
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0 && g->da > 0 && g->dv > 0 && g->dsd > 0 && g->dso > 0))
        return set_error(RN_ERR_ARG, "cyl: pitches and distances must be positive");
    const double hx = 0.5 * g->nx * g->dx + std::fabs(g->cx), hy = 0.5 * g->ny * g->dy + std::fabs(g->cy);
    if (g->dso <= std::sqrt(hx * hx + hy * hy))
        return set_error(RN_ERR_ARG, "cyl: the source orbit must lie outside the volume");
    if ((double)g->nu * g->da >= 3.0)
        return set_error(RN_ERR_ARG, "cyl: the fan must be narrower than 3 rad");
    return RN_OK;
}

extern "C" int rn_cyl_plan_create(rn_cyl_plan** out, const RnCylGeom* g, const float* host_deg, void* stream) {
    clear_error();
    if (!out || !host_deg) return set_error(RN_ERR_ARG, "cyl: null argument");
    *out = nullptr;
    RN_TRY(cyl_check(g));
    cudaStream_t st = (cudaStream_t)stream;
    rn_cyl_plan* p = new rn_cyl_plan();
    p->g = *g;
    cudaGetDevice(&p->device);
    CylDims& d = p->d;
    d.nb = g->nBatches; d.nx = g->nx; d.ny = g->ny; d.nz = g->nz;
    d.nu = g->nu; d.nview = g->nview; d.nv = g->nv;
    d.dx = g->dx; d.dy = g->dy; d.dz = g->dz; d.cx = g->cx; d.cy = g->cy; d.cz = g->cz;
    d.da = g->da; d.off_a = g->off_a; d.dv = g->dv; d.off_v = g->off_v; d.dsd = g->dsd;
    d.vol_stride = (long long)g->nx * g->ny * g->nz;
    d.prj_stride = (long long)g->nu * g->nview * g->nv;
    const int nu = g->nu, nv = g->nv, nview = g->nview;
    std::vector<CylView> views(nview);
    std::vector<double> redge((size_t)nview * (nu + 1));
    std::vector<float> inplane((size_t)nview * nu), sedge(nv + 1), rowlen(nv), invinp((size_t)nview * nu);
    std::vector<double> invdr((size_t)nview * nu);
    for (int iv = 0; iv < nview; iv++) {
        const float tf = host_deg[iv];
        const double t = (double)tf;
        const bool xc = std::fabs(std::cos(tf)) > std::fabs(std::sin(tf));   // the reference's float class rule
        views[iv] = CylView{g->dso * std::sin(t), -g->dso * std::cos(t), tf, xc ? 1 : 0};
        auto slope = [&](double a) {
            const double ph = a - t;
            return xc ? std::sin(ph) / std::cos(ph) : std::cos(ph) / std::sin(ph);
        };
        for (int e = 0; e <= nu; e++)
            redge[(size_t)iv * (nu + 1) + e] = slope((-((e - 0.5) - (nu - 1) / 2.0) - g->off_a) * g->da);
        for (int u = 0; u < nu; u++) {
            const double Rc = slope((-(u - (nu - 1) / 2.0) - g->off_a) * g->da);
            inplane[(size_t)iv * nu + u] = (float)std::sqrt(1 + Rc * Rc);
            invinp[(size_t)iv * nu + u] = (float)(1.0 / std::sqrt(1 + Rc * Rc));
            invdr[(size_t)iv * nu + u] =
                1.0 / std::fabs(redge[(size_t)iv * (nu + 1) + u + 1] - redge[(size_t)iv * (nu + 1) + u]);
        }
    }
    for (int e = 0; e <= nv; e++) sedge[e] = (float)(((e - 0.5) - (nv - 1) / 2.0 + g->off_v) * g->dv / g->dsd);
    for (int v = 0; v < nv; v++) {
        const double sc = ((double)v - (nv - 1) / 2.0 + g->off_v) * g->dv / g->dsd;
        rowlen[v] = (float)std::sqrt(1 + sc * sc);
    }
    const size_t tab_elems = (size_t)g->nBatches * nview * nu * (nv + 1);
    auto fail = [&](cudaError_t e, const char* what) {
        rn_cyl_plan_destroy(p);
        return set_cuda_error(e, what);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&p->d_views, sizeof(CylView) * nview)) != cudaSuccess) return fail(e, "cyl: view records");
    if ((e = cudaMalloc(&p->d_redge, sizeof(double) * redge.size())) != cudaSuccess) return fail(e, "cyl: edge table");
    if ((e = cudaMalloc(&p->d_inplane, sizeof(float) * inplane.size())) != cudaSuccess) return fail(e, "cyl: cells");
    if ((e = cudaMalloc(&p->d_sedge, sizeof(float) * sedge.size())) != cudaSuccess) return fail(e, "cyl: rows");
    if ((e = cudaMalloc(&p->d_rowlen, sizeof(float) * rowlen.size())) != cudaSuccess) return fail(e, "cyl: rows");
    if ((e = cudaMalloc(&p->d_tab, sizeof(float2) * tab_elems)) != cudaSuccess) return fail(e, "cyl: row tables");
    if ((e = cudaMalloc(&p->d_zp, sizeof(float) * (size_t)g->nBatches * g->nx * g->ny * (g->nz + 1))) != cudaSuccess)
        return fail(e, "cyl: z prefix sums");
    if ((e = cudaMalloc(&p->d_invdr, sizeof(double) * invdr.size())) != cudaSuccess) return fail(e, "cyl: cells");
    if ((e = cudaMalloc(&p->d_invinp, sizeof(float) * invinp.size())) != cudaSuccess) return fail(e, "cyl: cells");
    if ((e = cudaMemcpyAsync(p->d_views, views.data(), sizeof(CylView) * nview, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_redge, redge.data(), sizeof(double) * redge.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_inplane, inplane.data(), sizeof(float) * inplane.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_sedge, sedge.data(), sizeof(float) * sedge.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_rowlen, rowlen.data(), sizeof(float) * rowlen.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_invdr, invdr.data(), sizeof(double) * invdr.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_invinp, invinp.data(), sizeof(float) * invinp.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail(e, "cyl: table upload");
    // backprojection launches take views in chunks whose row tables (nu x
    // (nv + 1) float2 each) fill about 24 MB, well inside the 126 MB L2
    p->bp_chunk = (int)std::max<long long>(1, (24ll << 20) / ((long long)nu * (nv + 1) * 8 * g->nBatches));
    // the host vectors go out of scope: finish the copies first
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cyl: table upload");
    *out = p;
    return RN_OK;
}

extern "C" int rn_cyl_plan_destroy(rn_cyl_plan* p) {
    if (!p) return RN_OK;
    cudaFree(p->d_views);
    cudaFree(p->d_redge);
    cudaFree(p->d_inplane);
    cudaFree(p->d_sedge);
    cudaFree(p->d_rowlen);
    cudaFree(p->d_tab);
    cudaFree(p->d_zp);
    cudaFree(p->d_invdr);
    cudaFree(p->d_invinp);
    delete p;
    return RN_OK;
}

extern "C" long long rn_cyl_plan_launches(const rn_cyl_plan* p) { return p ? p->launches : 0; }

extern "C" int rn_cyl_project(rn_cyl_plan* p, float* d_prj, const float* d_vol, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_vol) return set_error(RN_ERR_ARG, "cyl: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const CylDims& d = p->d;
    const long long ncol = (long long)d.nb * d.nx * d.ny;
    cyl_zprefix_kernel<<<(unsigned)((ncol * 32 + 255) / 256), 256, 0, st>>>(p->d_zp, d_vol, d);
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    dim3 grid((unsigned)((d.nu + kCylFpWarps - 1) / kCylFpWarps), (unsigned)((d.nv + kCylRows - 1) / kCylRows),
              (unsigned)std::min<long long>((long long)d.nview * d.nb, 65535));
    cyl_fp_kernel<<<grid, 32 * kCylFpWarps, 0, st>>>(d_prj, p->d_zp, p->d_views, p->d_redge, p->d_inplane,
                                                    p->d_sedge, p->d_rowlen, d);
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

extern "C" int rn_cyl_backproject(rn_cyl_plan* p, float* d_vol, const float* d_prj, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_vol) return set_error(RN_ERR_ARG, "cyl: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const CylDims& d = p->d;
    const long long nt = (long long)d.nb * d.nview * d.nu;
    cyl_table_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(p->d_tab, d_prj, p->d_views, p->d_inplane,
                                                                    p->d_rowlen, d);
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    if (d.nb > 65535) return set_error(RN_ERR_ARG, "cyl: too many batches");
    dim3 grid((unsigned)(((long long)d.nx * d.ny + kCylBpWarps - 1) / kCylBpWarps),
              (unsigned)((d.nz + 32 * kCylBpZ - 1) / (32 * kCylBpZ)), (unsigned)d.nb);
    for (int v0 = 0; v0 < d.nview; v0 += p->bp_chunk) {
        const int v1 = std::min(d.nview, v0 + p->bp_chunk);
        cyl_bp_kernel<<<grid, 32 * kCylBpWarps, 0, st>>>(d_vol, p->d_tab, p->d_views, p->d_redge, p->d_invdr,
                                                        p->d_invinp, d, v0, v1, v0 > 0 ? 1 : 0);
        p->launches++;
        RN_CUDA_TRY(cudaGetLastError());
    }
    return RN_OK;
}
