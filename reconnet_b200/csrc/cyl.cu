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
constexpr int kCylRows = 64;     // detector rows per forward-projection warp (two per lane)
constexpr int kCylBpWarps = 8;   // voxel columns per backprojection CTA
constexpr int kCylBpZ = 2;       // voxels per lane along z (a warp covers 64)
constexpr float kCylFloorBias = 12582912.0f;   // 1.5 * 2^23: adding it rounds to an integer
constexpr int kCylFloorBiasBits = 0x4B400000;

// Band-limited z prefix sums of the volume, one column (b, x, y) per warp.
// Entry j of the band (nbz entries) holds the sum of the column's voxels
// between z = max(zlo, 0) and z = clamp(zlo + j, 0, nz) (voxel units), so that
// linear interpolation between entries is the column's exact integral up to
// any height, constant below the volume and above it.  The band [zlo, zlo +
// nbz - 1] covers every row edge of every view (the plan bounds it on the
// host), and accumulation is FP64.
__global__ void cyl_zprefix_kernel(float* __restrict__ zp, const float* __restrict__ vol, CylDims d, int zlo,
                                   int nbz) {
    const int lane = threadIdx.x & 31;
    const long long col = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (col >= (long long)d.nb * d.nx * d.ny) return;   // whole warp
    const long long b = col / ((long long)d.nx * d.ny), xy = col % ((long long)d.nx * d.ny);
    const float* v = vol + b * d.vol_stride + xy * d.nz;
    float* o = zp + col * nbz;
    const int z0 = max(zlo, 0), z1 = min(zlo + nbz - 1, d.nz);   // heights stored as running sums
    double carry = 0;
    for (int j0 = z0; j0 < z1; j0 += 32) {
        const int j = j0 + lane;   // voxel j: the entry at height j + 1 holds the sum up to it
        double x = j < z1 ? (double)v[j] : 0.0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += t;
        }
        if (j < z1) o[j + 1 - zlo] = (float)(carry + x);
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    // heights at or below max(zlo, 0) hold 0, heights above min(zhi, nz) the total
    const float tot = (float)carry;
    for (int j = lane; j < nbz; j += 32) {
        const int z = zlo + j;
        if (z <= z0) o[j] = 0.f;
        else if (z > z1) o[j] = tot;
    }
}

// Forward projection.  A warp owns one detector column u and 64 rows; lane l
// holds rows 2l and 2l + 1, so it evaluates their three edges.  Per plane k
// the column's lateral footprint [lo, hi] (voxel units) is affine in k, and
// so is each edge's height on the plane; the heights' cells and fractions are
// computed once per plane and serve every voxel column the footprint meets.
__global__ void __launch_bounds__(32 * kCylFpWarps) cyl_fp_kernel(float* __restrict__ prj,
                                                                 const float* __restrict__ zp,
                                                                 const CylView* __restrict__ views,
                                                                 const double* __restrict__ redge,
                                                                 const float* __restrict__ inplane,
                                                                 const float* __restrict__ sedge,
                                                                 const float* __restrict__ rowlen, CylDims d,
                                                                 int zlo, int nbz) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = blockIdx.x * kCylFpWarps + warp;
    if (u >= d.nu) return;                                   // whole warp
    const int g0 = blockIdx.y * kCylRows;
    const int e0 = g0 + 2 * lane;
    float sl[3];
#pragma unroll
    for (int q = 0; q < 3; q++) sl[q] = sedge[min(e0 + q, d.nv)];
    const float s_bot = sedge[min(g0, d.nv)], s_top = sedge[min(g0 + kCylRows, d.nv)];
    const float inv_dz = (float)(1.0 / d.dz);
    const float zoffb = (float)(d.nz / 2.0 - d.cz / d.dz) - (float)zlo;   // band coordinates
    const float zvol0 = -(float)zlo, zvol1 = (float)(d.nz - zlo);         // the volume's bottom and top
    const unsigned mmax = (unsigned)(nbz - 2);
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
        // plane k sits at D(k) = D0 + k dmain from the source along the main
        // axis (one sign for every plane: the source is outside the volume);
        // the footprint's edges are affine in D
        const double D0 = (0.5 - nplane / 2.0) * dmain + cmain - smain;
        const double la0 = fma(R0, D0, slat) * inv_dlat + lat_off, dla = R0 * dmain * inv_dlat;
        const double lb0 = fma(R1, D0, slat) * inv_dlat + lat_off, dlb = R1 * dmain * inv_dlat;
        const bool aless = la0 < lb0;
        const double lo0 = aless ? la0 : lb0, dlo = aless ? dla : dlb;
        const double hi0 = aless ? lb0 : la0, dhi = aless ? dlb : dla;
        // footprint width x in-plane distance: |R1 - R0| inp D^2 / dlat
        const float wfac = (float)(fabs(R1 - R0) * inv_dlat) * inp;
        const float* zb = zp + (long long)b * d.nx * d.ny * nbz;
        // voxel column (lateral i, plane k): x-class planes are rows y = k
        const long long cstride = (long long)(xc ? d.ny : 1) * nbz;
        const long long pstride = (long long)(xc ? 1 : d.ny) * nbz;
        float sz[3];
#pragma unroll
        for (int q = 0; q < 3; q++) sz[q] = sl[q] * inp * inv_dz;
        const float szb = s_bot * inp * inv_dz, szt = s_top * inp * inv_dz;
        float acc0 = 0.f, acc1 = 0.f;
        // Planes go in groups of 32: lane l first works out plane k0 + l's
        // lateral terms (the footprint's voxel columns and end fractions, the
        // distance |D| and the plane weight), which are the same for every
        // row, and the warp then walks the group's planes with them
        // broadcast by shuffles.
        for (int k0 = 0; k0 < nplane; k0 += 32) {
            int l_lo = 0, l_hi = -1;     // footprint cells: floor(lo), floor(hi); l_hi < l_lo: skip
            float l_flo = 0.f, l_fhi = 0.f, l_aD = 1.f, l_w = 0.f;
            {
                const int k = k0 + lane;
                if (k < nplane) {
                    const double D = fma((double)k, dmain, D0);
                    const double lo = fma((double)k, dlo, lo0), hi = fma((double)k, dhi, hi0);
                    const double flo_d = floor(lo), fhi_d = floor(hi);
                    const int ilo = (int)flo_d, ihi = (int)fhi_d;
                    const float aD = (float)fabs(D);
                    // the footprint meets the volume laterally, and the
                    // warp's rows meet its z extent
                    if (max(ilo, 0) <= min(ihi, nlat - 1) && fmaf(szt, aD, zoffb) > zvol0 &&
                        fmaf(szb, aD, zoffb) < zvol1) {
                        l_lo = ilo;
                        l_hi = ihi;
                        l_flo = (float)(lo - flo_d);
                        l_fhi = (float)(hi - fhi_d);
                        l_aD = aD;
                        l_w = __frcp_rn(wfac * aD * aD);
                    }
                }
            }
            const int nk = min(32, nplane - k0);
            for (int j = 0; j < nk; j++) {
                const int ilo = __shfl_sync(0xffffffffu, l_lo, j), ihi = __shfl_sync(0xffffffffu, l_hi, j);
                if (ihi < ilo) continue;                                 // warp-uniform
                const int i0 = max(ilo, 0), i1 = min(ihi, nlat - 1);
                const float flo = __shfl_sync(0xffffffffu, l_flo, j), fhi = __shfl_sync(0xffffffffu, l_fhi, j);
                const float aD = __shfl_sync(0xffffffffu, l_aD, j), w = __shfl_sync(0xffffffffu, l_w, j);
                // each edge's cell m and fraction f in the band
                unsigned m[3];
                float f[3];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const float z = fmaf(sz[q], aD, zoffb);
                    const float y = __fadd_rd(z, kCylFloorBias);
                    const int mi = __float_as_int(y) - kCylFloorBiasBits;
                    f[q] = z - (y - kCylFloorBias);
                    m[q] = min((unsigned)max(mi, 0), mmax);
                }
                const float* cp = zb + (k0 + j) * pstride;
                float Q0 = 0.f, Q1 = 0.f, Q2 = 0.f;
                for (int i = i0; i <= i1; i++) {
                    const float ox = (i == ihi ? fhi : 1.f) - (i == ilo ? flo : 0.f);
                    const float* c = cp + i * cstride;
                    float a0 = __ldg(c + m[0]), b0 = __ldg(c + m[0] + 1);
                    float a1 = __ldg(c + m[1]), b1 = __ldg(c + m[1] + 1);
                    float a2 = __ldg(c + m[2]), b2 = __ldg(c + m[2] + 1);
                    Q0 = fmaf(ox, fmaf(f[0], b0 - a0, a0), Q0);
                    Q1 = fmaf(ox, fmaf(f[1], b1 - a1, a1), Q1);
                    Q2 = fmaf(ox, fmaf(f[2], b2 - a2, a2), Q2);
                }
                acc0 = fmaf(Q1 - Q0, w, acc0);
                acc1 = fmaf(Q2 - Q1, w, acc1);
            }
        }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int e = e0 + q;
            if (e < d.nv) {
                const float ds = sedge[e + 1] - sedge[e];
                const float L = (float)dmain * inp * rowlen[e];
                prj[(long long)b * d.prj_stride + ((long long)u * d.nview + iv) * d.nv + e] =
                    (q ? acc1 : acc0) * L * (float)d.dz / ds;
            }
        }
    }
}

// Row tables of the backprojection: per (batch, view, column u), nv + 2
// entries: entry r + 1 holds (sum over rows v < r of L p, L p of row r) for
// r < nv, built in FP64; entry 0 = (0, 0) and entry nv + 1 = (total, 0) are
// guards, so that a height below the detector reads 0 and one above it the
// total without a branch.
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
    float2* out = tab + (((long long)b * d.nview + iv) * d.nu + u) * (d.nv + 2);
    double C = 0;
    out[0] = make_float2(0.f, 0.f);
    for (int v = 0; v < d.nv; v++) {
        const double w = lu * rowlen[v] * (double)p[v];
        out[v + 1] = make_float2((float)C, (float)w);
        C += w;
    }
    out[d.nv + 1] = make_float2((float)C, 0.f);
}

// The prefix of L p at detector-row coordinate rho of a row table (linear
// inside each row, 0 below the detector, the total above it).
__device__ __forceinline__ float row_prefix(const float2* __restrict__ t, float rho, int nv) {
    const float y = __fadd_rd(rho, kCylFloorBias);
    const int m = min(max(__float_as_int(y) - kCylFloorBiasBits, -1), nv);
    const float2 c = __ldg(&t[m + 1]);
    return fmaf(c.y, rho - (y - kCylFloorBias), c.x);
}

// The candidate cells u of one view for the voxel column (ix, iy): those
// whose footprint on the column's plane overlaps the voxel laterally and whose
// rows reach the warp's z run [zfirst, zlast] (mm).  For each, emit(u, w,
// inv) with w the lateral overlap weight and inv the detector rows per mm of
// height on the plane.
template <class Emit>
__device__ __forceinline__ void cyl_bp_candidates(const CylView& V, int iv, int ix, int iy, const CylDims& d,
                                                  const double* __restrict__ redge, const float* __restrict__ inv_dr,
                                                  const float* __restrict__ inv_inp, float zfirst, float zlast,
                                                  Emit&& emit) {
    const float rho0 = (float)(d.nv / 2.0 - d.off_v);
    const float dsd_dv = (float)(d.dsd / d.dv);
    const float inv_da = (float)(1.0 / d.da), e_off = (float)(-d.off_a + (d.nu - 1) * 0.5 + 0.5);
    const double two_pi = 6.283185307179586;
    const bool xc = V.xcls != 0;
    const int k = xc ? iy : ix, i = xc ? ix : iy;
    const int nplane = xc ? d.ny : d.nx, nlat = xc ? d.nx : d.ny;
    const double dmain = xc ? d.dy : d.dx, dlat = xc ? d.dx : d.dy;
    const double cmain = xc ? d.cy : d.cx, clat = xc ? d.cx : d.cy;
    const double smain = xc ? V.sy : V.sx, slat = xc ? V.sx : V.sy;
    const double D = (k + 0.5 - nplane / 2.0) * dmain + cmain - smain;
    // the voxel's lower lateral face, relative to the source
    const double lf = (i - nlat / 2.0) * dlat + clat - slat;
    // fan angle of the ray through the voxel's lateral centre, and the
    // half-width of the voxel's angular range to first order: |D| / r^2 per
    // mm of lateral offset.  The candidate range is widened by the bound of
    // the second-order term, (dlat / 2)^2 / (2 r^2) rad, twice over, and 0.01
    // cells; every candidate's overlap is then exact.
    const float pl = (float)(lf + 0.5 * dlat), pD = (float)D;
    const float px = xc ? pl : pD, py = xc ? pD : pl;
    float a = atan2f(px, py) + V.theta;
    a -= (float)two_pi * rintf(a * (float)(1.0 / two_pi));
    const float inv_r2 = __frcp_rn(fmaf(px, px, py * py));
    const float dl = (float)dlat;
    const float half = 0.5f * dl * fabsf(pD) * inv_r2 * inv_da;
    const float slack = fmaf(0.25f * dl * dl * inv_r2, inv_da, 0.01f);
    const float ec = fmaf(-a, inv_da, e_off);
    const int ulo = (int)fmaxf(floorf(ec - half - slack), 0.f);
    const int uhi = (int)fminf(floorf(ec + half + slack), (float)(d.nu - 1));
    const float inv_aD = __frcp_rn(fabsf(pD));
    const float wD = dl * inv_aD;
    const double inv_dlat = 1.0 / dlat;
    const double* Rv = redge + (long long)iv * (d.nu + 1);
    // lateral position of edge e on this plane relative to the voxel's lower
    // face, in voxel units
    float xe = (float)((fma(Rv[ulo], D, -lf)) * inv_dlat);
    for (int u = ulo; u <= uhi; u++) {
        const float xn = (float)((fma(Rv[u + 1], D, -lf)) * inv_dlat);
        const float lo = fminf(xe, xn), hi = fmaxf(xe, xn);
        xe = xn;
        const float ov = fminf(hi, 1.f) - fmaxf(lo, 0.f);
        if (ov <= 0.f) continue;
        const float inv = dsd_dv * inv_aD * inv_inp[(long long)iv * d.nu + u];
        // the warp's z run against the detector rows: skip if it misses them
        if (fmaf(zlast, inv, rho0) <= 0.f || fmaf(zfirst, inv, rho0) >= (float)d.nv) continue;
        emit(u, ov * wD * inv_dr[(long long)iv * d.nu + u], inv);
    }
}

constexpr int kCylBpSlots = 8;   // candidates kept per (voxel column, view)

// Backprojection.  A warp owns the voxels vz0 + 64 blockIdx.y + [0, 64) of
// one (x, y) column, two per lane.  Views go in groups of 32: first each lane
// finds the candidate cells of one view of the group (the lateral work, once
// per view instead of once per lane), into a per-warp list in shared memory;
// then the warp walks the group's views and candidates together, each lane
// reading the row tables at its voxels' edges.  A view with more candidates
// than the list holds is redone by the whole warp.
__global__ void __launch_bounds__(32 * kCylBpWarps) cyl_bp_kernel(float* __restrict__ vol, const float2* __restrict__ tab,
                                                                 const CylView* __restrict__ views,
                                                                 const double* __restrict__ redge,
                                                                 const float* __restrict__ inv_dr,
                                                                 const float* __restrict__ inv_inp, CylDims d,
                                                                 int v_begin, int v_end, int accumulate, int vz0,
                                                                 int vz1) {
    constexpr int Z = kCylBpZ;
    __shared__ float4 s_cand[kCylBpWarps][kCylBpSlots][32];   // (w, inv, view * nu + u) per slot and view
    __shared__ int s_cnt[kCylBpWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long column = (long long)blockIdx.x * kCylBpWarps + warp;
    if (column >= (long long)d.nx * d.ny) return;              // whole warp
    const int ix = (int)(column / d.ny), iy = (int)(column % d.ny);
    const int b = blockIdx.z;
    // Only voxels vz0 <= j < vz1 can meet a detector row (the plan bounds the
    // rows' heights over every view and plane); the first launch of a
    // backprojection writes 0 to the rest of the column.
    if (!accumulate && blockIdx.y == 0) {
        float* o = vol + (long long)b * d.vol_stride + ((long long)ix * d.ny + iy) * d.nz;
        for (int j = lane; j < d.nz; j += 32)
            if (j < vz0 || j >= vz1) o[j] = 0.f;
    }
    const int zbase = vz0 + blockIdx.y * 32 * Z;
    // lane holds voxels zbase + Z lane + q; z (mm) of their Z + 1 edges
    float ze[Z + 1];
#pragma unroll
    for (int q = 0; q <= Z; q++) ze[q] = (float)((zbase + Z * lane + q - d.nz / 2.0) * d.dz + d.cz);
    const float zlast = (float)((min(vz1, zbase + 32 * Z) - d.nz / 2.0) * d.dz + d.cz);
    const float zfirst = (float)((zbase - d.nz / 2.0) * d.dz + d.cz);
    const float rho0 = (float)(d.nv / 2.0 - d.off_v);
    const long long tab_b = (long long)b * d.nview * d.nu;
    float acc[Z];
#pragma unroll
    for (int q = 0; q < Z; q++) acc[q] = 0.f;
    // one candidate: the prefixes at the lane's Z + 1 edges; a voxel's
    // integral is the difference of its two edges'
    auto add = [&](int vu, float w, float inv) {
        const float2* t = tab + (tab_b + vu) * (d.nv + 2);
        float P[Z + 1];
#pragma unroll
        for (int q = 0; q <= Z; q++) P[q] = row_prefix(t, fmaf(ze[q], inv, rho0), d.nv);
#pragma unroll
        for (int q = 0; q < Z; q++) acc[q] = fmaf(w, P[q + 1] - P[q], acc[q]);
    };
    for (int v0 = v_begin; v0 < v_end; v0 += 32) {
        // lateral work: lane l takes view v0 + l
        {
            const int iv = v0 + lane;
            int n = 0;
            if (iv < v_end) {
                const CylView V = views[iv];
                cyl_bp_candidates(V, iv, ix, iy, d, redge, inv_dr, inv_inp, zfirst, zlast,
                                  [&](int u, float w, float inv) {
                                      if (n < kCylBpSlots)
                                          s_cand[warp][n][lane] = make_float4(w, inv, __int_as_float(iv * d.nu + u), 0.f);
                                      n++;
                                  });
            }
            s_cnt[warp][lane] = n <= kCylBpSlots ? n : -1;
        }
        __syncwarp();
        const int nj = min(32, v_end - v0);
        for (int j = 0; j < nj; j++) {
            const int cnt = s_cnt[warp][j];
            if (cnt >= 0) {
                for (int c = 0; c < cnt; c++) {
                    const float4 e = s_cand[warp][c][j];
                    add(__float_as_int(e.z), e.x, e.y);
                }
            } else {   // more candidates than the list holds: the warp redoes the view
                const int iv = v0 + j;
                const CylView V = views[iv];
                cyl_bp_candidates(V, iv, ix, iy, d, redge, inv_dr, inv_inp, zfirst, zlast,
                                  [&](int u, float w, float inv) { add(iv * d.nu + u, w, inv); });
            }
        }
        __syncwarp();   // the list is rewritten for the next group
    }
#pragma unroll
    for (int q = 0; q < Z; q++) {
        const int j = zbase + Z * lane + q;
        if (j < vz1) {
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
    float* d_invdr = nullptr;     // [nview][nu] 1 / |R_{u+1} - R_u|
    float* d_invinp = nullptr;    // [nview][nu] 1 / sqrt(1 + R_c^2)
    int bp_chunk = 0;             // views per backprojection launch (their row tables stay in L2)
    float2* d_tab = nullptr;      // backprojection row tables [nb][nview][nu][nv+2]
    float* d_zp = nullptr;        // forward-projection z prefix band [nb][nx][ny][nbz]
    int zlo = 0, nbz = 0;         // the band: heights zlo .. zlo + nbz - 1 (voxel units)
    int vz0 = 0, vz1 = 0;         // voxels that can meet a detector row: vz0 <= j < vz1
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
    std::vector<float> invdr((size_t)nview * nu);
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
                (float)(1.0 / std::fabs(redge[(size_t)iv * (nu + 1) + u + 1] - redge[(size_t)iv * (nu + 1) + u]));
        }
    }
    for (int e = 0; e <= nv; e++) sedge[e] = (float)(((e - 0.5) - (nv - 1) / 2.0 + g->off_v) * g->dv / g->dsd);
    for (int v = 0; v < nv; v++) {
        const double sc = ((double)v - (nv - 1) / 2.0 + g->off_v) * g->dv / g->dsd;
        rowlen[v] = (float)std::sqrt(1 + sc * sc);
    }
    const size_t tab_elems = (size_t)g->nBatches * nview * nu * (nv + 2);
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
    // The forward projection's z prefix band.  A row edge of rise s sits, on
    // a plane, at height s r / dz + zoff, r the in-plane distance from the
    // source to where the cell's central ray meets the plane.  Both passes
    // use a plane only where the cell's footprint meets the volume, so r is
    // at most the distance from the source to the volume's in-plane box
    // grown by one voxel and one footprint width (and at least the distance
    // to that box); the band spans s r / dz + zoff over those extremes, with
    // one cell of margin each side, cut to one height below and above the
    // volume, where the prefix is constant.
    {
        // a footprint's lateral width on a plane is |D| da (1 + R^2) to first
        // order, R the lateral slope of its rays
        double rsl = 0.0;
        for (double r : redge) rsl = std::max(rsl, std::fabs(r));
        const double grow = std::max(g->dx, g->dy) + (g->dso + std::hypot(0.5 * g->nx * g->dx + std::fabs(g->cx),
                                                                          0.5 * g->ny * g->dy + std::fabs(g->cy))) *
                                                        g->da * (1 + rsl * rsl) * 1.5;
        const double bx0 = -0.5 * g->nx * g->dx + g->cx - grow, bx1 = 0.5 * g->nx * g->dx + g->cx + grow;
        const double by0 = -0.5 * g->ny * g->dy + g->cy - grow, by1 = 0.5 * g->ny * g->dy + g->cy + grow;
        double rmin = 1e300, rmax = 0.0;
        for (int iv = 0; iv < nview; iv++) {
            const double sx = views[iv].sx, sy = views[iv].sy;
            for (double x : {bx0, bx1})
                for (double y : {by0, by1}) rmax = std::max(rmax, std::hypot(x - sx, y - sy));
            const double qx = std::min(std::max(sx, bx0), bx1), qy = std::min(std::max(sy, by0), by1);
            rmin = std::min(rmin, std::hypot(qx - sx, qy - sy));
        }
        const double smin = sedge[0], smax = sedge[nv];
        double pmin = std::min(smin * rmin, smin * rmax), pmax = std::max(smax * rmin, smax * rmax);
        if (!(pmin > -1e9)) pmin = -1e9;   // unbounded footprints: the whole volume
        if (!(pmax < 1e9)) pmax = 1e9;
        const double zoff = g->nz / 2.0 - g->cz / g->dz;
        long long zlo = (long long)std::floor(pmin / g->dz + zoff) - 1;
        long long zhi = (long long)std::ceil(pmax / g->dz + zoff) + 1;
        zlo = std::max<long long>(zlo, -1);
        zhi = std::min<long long>(zhi, (long long)g->nz + 1);
        if (zhi < zlo + 1) zhi = zlo + 1;
        p->zlo = (int)zlo;
        p->nbz = (int)(zhi - zlo + 1);
        // voxel j spans heights [j, j + 1]: those inside the band's heights
        p->vz0 = (int)std::max<long long>(zlo, 0);
        p->vz1 = (int)std::max<long long>(std::min<long long>(zhi, g->nz), p->vz0 + 1);
    }
    if ((e = cudaMalloc(&p->d_zp, sizeof(float) * (size_t)g->nBatches * g->nx * g->ny * p->nbz)) != cudaSuccess)
        return fail(e, "cyl: z prefix sums");
    if ((e = cudaMalloc(&p->d_invdr, sizeof(float) * invdr.size())) != cudaSuccess) return fail(e, "cyl: cells");
    if ((e = cudaMalloc(&p->d_invinp, sizeof(float) * invinp.size())) != cudaSuccess) return fail(e, "cyl: cells");
    if ((e = cudaMemcpyAsync(p->d_views, views.data(), sizeof(CylView) * nview, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_redge, redge.data(), sizeof(double) * redge.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_inplane, inplane.data(), sizeof(float) * inplane.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_sedge, sedge.data(), sizeof(float) * sedge.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_rowlen, rowlen.data(), sizeof(float) * rowlen.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_invdr, invdr.data(), sizeof(float) * invdr.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(p->d_invinp, invinp.data(), sizeof(float) * invinp.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail(e, "cyl: table upload");
    // backprojection launches take views in chunks whose row tables (nu x
    // (nv + 2) float2 each) fill about 24 MB, well inside the 126 MB L2
    p->bp_chunk = (int)std::max<long long>(1, (24ll << 20) / ((long long)nu * (nv + 2) * 8 * g->nBatches));
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
    cyl_zprefix_kernel<<<(unsigned)((ncol * 32 + 255) / 256), 256, 0, st>>>(p->d_zp, d_vol, d, p->zlo, p->nbz);
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    dim3 grid((unsigned)((d.nu + kCylFpWarps - 1) / kCylFpWarps), (unsigned)((d.nv + kCylRows - 1) / kCylRows),
              (unsigned)std::min<long long>((long long)d.nview * d.nb, 65535));
    cyl_fp_kernel<<<grid, 32 * kCylFpWarps, 0, st>>>(d_prj, p->d_zp, p->d_views, p->d_redge, p->d_inplane,
                                                    p->d_sedge, p->d_rowlen, d, p->zlo, p->nbz);
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
              (unsigned)((p->vz1 - p->vz0 + 32 * kCylBpZ - 1) / (32 * kCylBpZ)), (unsigned)d.nb);
    for (int v0 = 0; v0 < d.nview; v0 += p->bp_chunk) {
        const int v1 = std::min(d.nview, v0 + p->bp_chunk);
        cyl_bp_kernel<<<grid, 32 * kCylBpWarps, 0, st>>>(d_vol, p->d_tab, p->d_views, p->d_redge, p->d_invdr,
                                                        p->d_invinp, d, v0, v1, v0 > 0 ? 1 : 0, p->vz0, p->vz1);
        p->launches++;
        RN_CUDA_TRY(cudaGetLastError());
    }
    return RN_OK;
}
