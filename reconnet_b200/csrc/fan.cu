// Distance-driven fan-beam projector pair for sm_100a.
//
// Forward projection (restates DDFPFanKernelX/Y, ReconNet4D/DistanceDriven.cu:64-196):
//   prj(u, view) = L_u * sum_lines [P_l(x_{u+1}(l)) - P_l(x_u(l))] / (x_{u+1}(l) - x_u(l))
// where l runs over the image rows (X-class views) or columns (Y-class),
// x_e(l) is where the ray through detector-cell edge e crosses line l, and
// P_l is the exact integral of the line's pixel values from 0 to x.  The
// reference samples its prefix texture at row *boundaries* with a 50/50
// blend of the two neighbouring rows (tex3D at integer y, border mode); the
// line arrays built here are exactly those blended rows.
//
// Design:
//   * line prologue: one warp per line, FP64 prefix split into hi/lo floats
//     (so prefix differences keep full precision), written once per call;
//   * FP kernel: one CTA per (slice, view class, 4 views); lines are staged
//     into shared memory in chunks with bulk async copies (cp.async.bulk +
//     mbarrier, double buffered); each thread integrates whole rays across
//     the staged lines; per-ray accumulators live in shared memory;
//   * BP: edge tables (FP64 prefix of the weighted sinogram, hi/lo) built per
//     call, then a gather-form kernel (no atomics): each thread owns a 4x4
//     pixel block and accumulates all views in registers; per-view table
//     windows are staged with bulk async copies.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "rn_device.cuh"
#include "rn_internal.h"

namespace rn {

// ---------------------------------------------------------------------------
// Tunables.
// ---------------------------------------------------------------------------
// FP CTA shape per mode: DD runs 24 warps of 6 ray groups (80 registers),
// Siddon, whose band step needs more registers, 16 warps of 8 groups
template <bool kSiddon>
struct FpCfg {
    static constexpr int threads = kSiddon ? 512 : 768;
    static constexpr int groups = kSiddon ? 8 : 6;   // groups of 31 rays per warp (at most)
    static constexpr int warps = threads / 32;
};
constexpr int kFpViews = 4;          // views per FP CTA (at most)
constexpr int kFpMaxLines = 16;      // lines per staged chunk (upper bound)
constexpr int kSmemBudget = 227 * 1024;


constexpr int kBpViews = 8;          // views per staged chunk

__host__ __device__ inline long long align4(long long v) { return (v + 3) & ~3ll; }

// ---------------------------------------------------------------------------
// Geometry: per-edge slopes r_e (FP64).  X-class: r = tan(gamma_e - theta)*dy/dx
// (= (D.x - S.x)/(D.y - S.y) in image units, DistanceDriven.cu:89-113);
// Y-class: r = cot(gamma_e - theta)*dx/dy.
// ---------------------------------------------------------------------------
__global__ void edge_slope_kernel(double* edges, const double2* view_cs, const int* view_x, const double2* edge_sc,
                                  int total_views, int nu, double dx, double dy) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)total_views * (nu + 1);
    if (i >= n) return;
    int v = (int)(i / (nu + 1));
    int e = (int)(i - (long long)v * (nu + 1));
    double2 cs = view_cs[v];     // (cos theta, sin theta)
    double2 sc = edge_sc[e];     // (sin gamma, cos gamma)
    double sn = sc.x * cs.x - sc.y * cs.y;   // sin(gamma - theta)
    double cn = sc.y * cs.x + sc.x * cs.y;   // cos(gamma - theta)
    edges[i] = view_x[v] ? (sn * dy) / (cn * dx) : (cn * dx) / (sn * dy);
}

// ---------------------------------------------------------------------------
// Line prologue: for each FP slice, X lines (image rows, boundary l between
// rows l-1 and l) and Y lines (columns).  Entry k of a line holds the prefix
// P[k] = sum_{i<k} a_i (summed in FP64) and the value a_k (a_n = 0).
// Band mode (Siddon): P as (hi, lo) floats in `hl`, a_k in `la`, entry j at
// line_pos(j) (one unused slot per 16 entries, against bank conflicts); the
// band integrals need prefix differences across a fraction of one cell.  DD
// mode: (P rounded to FP32, a_k) packed in `hl` at entry j, `la` unused; a DD
// footprint spans about a cell, so the prefix's FP32 rounding moves a
// projection by ~1e-7 relative (independent roundings over the lines a ray
// crosses).
// ---------------------------------------------------------------------------
__global__ void fan_lines_kernel(const float* __restrict__ img, const FpSlice* __restrict__ fps, int s_begin, int ns,
                                 FanDims d, float2* __restrict__ hl, float* __restrict__ la, long long slot_elems,
                                 int band) {
    __shared__ __align__(16) float s_lines_a[8][128];
    __shared__ __align__(16) double s_lines_p[8][128];
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int per_slice = d.ny + d.nx;
    if (warp >= ns * per_slice) return;
    int si = warp / per_slice;
    int li = warp - si * per_slice;
    const FpSlice fs = fps[s_begin + si];
    bool xl = li < d.ny;
    int l = xl ? li : li - d.ny;
    int n = xl ? d.nx : d.ny;
    int lp = xl ? d.lpx : d.lpy;
    const int M = d.margin;
    long long base = (long long)si * slot_elems + (xl ? (long long)l * d.spx : (long long)d.ny * d.spx + (long long)l * d.spy);
    float2* ohl = hl + base;    // entry j (at line_pos(j) in band mode, j for DD) holds position k = j - M
    float* ola = la + base;
    // blended value of rows (l-1, l) [X] or columns (l-1, l) [Y] at position k;
    // band mode (Siddon): row / column l itself
    auto value = [&](int k) -> float {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            float w = fs.img_w[j];
            if (w == 0.f) continue;
            const float* p = img + fs.img_off[j];
            float v1, v0 = 0.f;
            if (xl) {
                v1 = __ldg(p + (long long)k * d.isx + (long long)l * d.isy);
                if (l > 0) v0 = __ldg(p + (long long)k * d.isx + (long long)(l - 1) * d.isy);
            } else {
                v1 = __ldg(p + (long long)l * d.isx + (long long)k * d.isy);
                if (l > 0) v0 = __ldg(p + (long long)(l - 1) * d.isx + (long long)k * d.isy);
            }
            s += w * (band ? v1 : 0.5f * v0 + 0.5f * v1);
        }
        return s;
    };
    // Blocks of 128 positions: loaded and stored coalesced (position 32c +
    // lane), scanned with each lane owning 4 consecutive positions (4 lane,
    // .., 4 lane + 3, exchanged through shared memory), so one warp scan
    // serves 128 positions.
    const int wib = (threadIdx.x >> 5) & 7;
    float* sa = s_lines_a[wib];
    double* sp = s_lines_p[wib];
    double carry = 0.0;
    for (int k0 = 0; k0 < n; k0 += 128) {
        float v[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = k0 + 32 * c + lane;
            v[c] = k < n ? value(k) : 0.f;
            sa[32 * c + lane] = v[c];
        }
        __syncwarp();
        const float4 q = reinterpret_cast<const float4*>(sa)[lane];
        const double p1 = (double)q.x, p2 = p1 + (double)q.y, p3 = p2 + (double)q.z, p4 = p3 + (double)q.w;
        const double incl = warp_incl_scan(p4);
        const double pre = carry + (incl - p4);   // exclusive prefix at position 4 lane
        reinterpret_cast<double2*>(sp)[2 * lane] = make_double2(pre, pre + p1);
        reinterpret_cast<double2*>(sp)[2 * lane + 1] = make_double2(pre + p2, pre + p3);
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = k0 + 32 * c + lane;
            if (k < n) {
                if (band) {
                    ohl[line_pos(k + M)] = split_double(sp[32 * c + lane]);
                    ola[line_pos(k + M)] = v[c];
                } else {
                    ohl[k + M] = make_float2((float)sp[32 * c + lane], v[c]);
                }
            }
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();   // the next block overwrites sa and sp
    }
    // margins: P = 0 before the line, P = total from position n on
    const float2 tot = band ? split_double(carry) : make_float2((float)carry, 0.f);
    for (int j = lane; j < M; j += 32) {
        ohl[band ? line_pos(j) : j] = make_float2(0.f, 0.f);
        if (band) ola[line_pos(j)] = 0.f;
    }
    for (int j = n + M + lane; j < lp; j += 32) {
        ohl[band ? line_pos(j) : j] = tot;
        if (band) ola[line_pos(j)] = 0.f;
    }
}

// ---------------------------------------------------------------------------
// FP kernel.
//
// One CTA = (slice, view class, up to kFpViews views), 16 warps.  A warp
// owns groups of 31 adjacent rays of one view: lane i evaluates the prefix
// integral at cell edge e0+i and takes edge e0+i+1 from its neighbour with a
// shuffle, so every edge is evaluated once.  Group accumulators and line
// ranges stay in registers for the whole kernel.  Lines are staged R at a
// time into a double buffer by bulk async copies.  Per chunk, an edge's
// position at the chunk's first line is rebuilt from a per-edge table (the
// line-0 position as integer cell + offset, the slope as hi/lo floats) and
// split into an integer cell and a small FP32 offset, so per-line positions
// carry ~1e-6 cells of rounding.  A group
// visits only the lines where one of its footprints overlaps the image.  The
// line arrays carry `margin` zero-valued padding entries on both sides and
// positions beyond them clamp to the ends, so a footprint that misses a line
// adds exactly zero and no per-ray masking is needed.
// ---------------------------------------------------------------------------
constexpr int kFpGroupRays = 31;
// shared-memory header: barriers and view data (128 B), then the per-line
// factors 1 / (l - perp) of two chunks; the per-edge table follows
constexpr int kFpHeader = 128 + 2 * (int)sizeof(float) * kFpViews * kFpMaxLines;
static_assert(kFpHeader % 16 == 0, "per-edge table must be 16-byte aligned");
constexpr float kFloorBias = 12582912.0f;   // 1.5 * 2^23
constexpr int kFloorBiasBits = 0x4B400000;

struct FpParams {
    const ViewGeo* views;
    const double* edges;
    const float2* cell;
    const int* perm;
    const GeoSet* sets;
    const FpSlice* fps;
    const int4* work;
    const float2* hl;
    const float* la;
    long long slot_elems;
    int slot_base;     // first FP slice of the current wave
    float* prj;
    int* err;
    FanDims d;
    int R;             // lines per chunk
    int vt;            // views per CTA (size of the per-edge table)
    long long spin;    // polls of a chunk wait before it gives up (the plan's spin limit)
};

// Active line range [lb, le) of the footprint between edge slopes ra, rb
// (positions x(l) = par + r (l - perp)) over [0, n], visiting one extra line
// on each side against FP64 rounding; 0 if empty, else lb << 16 | le.
__device__ __forceinline__ int fp_ray_range(double ra, double rb, double par, double perp, int nlines, double n) {
    double lm = 0.5 * nlines;
    bool aHi = (par + ra * (lm - perp)) >= (par + rb * (lm - perp));   // the edges meet only at the source
    double rh = aHi ? ra : rb, rl = aHi ? rb : ra;
    double lo_l = -1e30, hi_l = 1e30;
    if (rh > 0) lo_l = fmax(lo_l, perp - par / rh);          // hi(l) > 0
    else if (rh < 0) hi_l = fmin(hi_l, perp - par / rh);
    else if (!(par > 0)) hi_l = -1e30;
    if (rl > 0) hi_l = fmin(hi_l, perp + (n - par) / rl);    // lo(l) < n
    else if (rl < 0) lo_l = fmax(lo_l, perp + (n - par) / rl);
    else if (!(par < n)) hi_l = -1e30;
    double lb = fmax(0.0, floor(lo_l)), le = fmin((double)nlines, floor(hi_l) + 2.0);
    return (le > lb) ? (((int)lb << 16) | (int)le) : 0;
}

template <bool kSiddon>
__global__ void __launch_bounds__(FpCfg<kSiddon>::threads, 1) fan_fp_kernel(FpParams p) {
    constexpr int kFpThreads = FpCfg<kSiddon>::threads, kFpGroups = FpCfg<kSiddon>::groups;
    constexpr int kFpWarps = FpCfg<kSiddon>::warps;
    extern __shared__ __align__(128) unsigned char smem[];
    const int4 w = p.work[blockIdx.x];
    const int s = w.x, xcls = w.y, vbegin = w.z, vcount = w.w;
    const FpSlice fs = p.fps[s];
    const GeoSet gs = p.sets[fs.set];
    const int nu = p.d.nu;
    const int nlines = xcls ? p.d.ny : p.d.nx;
    const int lp = xcls ? p.d.lpx : p.d.lpy;   // entries per line
    const int sp = xcls ? p.d.spx : p.d.spy;   // line stride (padded)
    const int R = p.R;
    const long long slot = (long long)(s - p.slot_base) * p.slot_elems + (xcls ? 0ll : (long long)p.d.ny * p.d.spx);
    const float2* ghl = p.hl + slot;
    const float* gla = p.la + slot;

    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    int* s_gv = reinterpret_cast<int*>(smem + 16);                  // kFpViews
    int* s_vl = s_gv + kFpViews;                                    // set-local view index
    double* s_par = reinterpret_cast<double*>(smem + 64);           // kFpViews
    double* s_perp = s_par + kFpViews;                              // kFpViews
    float* s_g = reinterpret_cast<float*>(smem + 128);              // 2 x kFpViews x kFpMaxLines
    float4* s_edge = reinterpret_cast<float4*>(smem + kFpHeader);
    size_t off = kFpHeader + sizeof(float4) * (size_t)p.vt * (nu + 1);
    off = (off + 127) & ~size_t(127);
    // double buffer: buffer b holds R lines of float2 entries ((P, a) packed
    // for DD; (hi, lo) then R lines of values for Siddon)
    const size_t hl_bytes = (size_t)R * sp * sizeof(float2), la_bytes = kSiddon ? (size_t)R * sp * sizeof(float) : 0;
    unsigned char* const buf0 = smem + off;
    const size_t buf_bytes = hl_bytes + la_bytes;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if (tid < vcount) {
        int vl = p.perm[gs.view_off + vbegin + tid];
        int gv = gs.view_off + vl;
        s_vl[tid] = vl;
        s_gv[tid] = gv;
        s_par[tid] = p.views[gv].par;
        s_perp[tid] = p.views[gv].perp;
    }
    __syncthreads();
    // per-edge positions at line 0 (padded) and slopes, as hi/lo floats
    const double M = (double)p.d.margin;
    for (int i = tid; i < vcount * (nu + 1); i += kFpThreads) {
        int v = i / (nu + 1);
        int e = i - v * (nu + 1);
        double r = p.edges[(long long)s_gv[v] * (nu + 1) + e];
        double X0 = s_par[v] - r * s_perp[v] + M;
        double Xi0 = floor(X0);
        float rh = (float)r;
        s_edge[i] = make_float4((float)(X0 - Xi0), __int_as_float((int)Xi0), rh, (float)(r - (double)rh));
    }
    // ray groups of this warp: own ray range (per lane) and the group's
    // union range (warp-uniform)
    const int ngpv = (nu + kFpGroupRays - 1) / kFpGroupRays;    // groups per view
    const int ngroups = vcount * ngpv;
    const double n_d = (double)(xcls ? p.d.nx : p.d.ny);
    // per group: line range (lb << 16 | le) and this lane's edge-table slot
    // (view << 16 | entry), fixed for the whole kernel
    int urng[kFpGroups], gslot[kFpGroups];
    float acc[kFpGroups];
#pragma unroll
    for (int k = 0; k < kFpGroups; k++) {
        acc[k] = 0.f;
        urng[k] = 0;
        gslot[k] = 0;
        const int grp = warp + k * kFpWarps;
        if (grp < ngroups) {   // warp-uniform
            const int v = grp / ngpv;
            const int u = (grp - v * ngpv) * kFpGroupRays + lane;
            gslot[k] = (v << 16) | (v * (nu + 1) + min(u, nu));
            int rng = 0;
            if (lane < kFpGroupRays && u < nu) {
                const double* ed = p.edges + (long long)s_gv[v] * (nu + 1);
                rng = fp_ray_range(ed[u], ed[kSiddon ? u : u + 1], s_par[v], s_perp[v], nlines, n_d);
            }
            int lb = rng ? (rng >> 16) : 0x7fffffff;
            int le = rng ? (rng & 0xffff) : 0;
            lb = __reduce_min_sync(0xffffffffu, lb);
            le = __reduce_max_sync(0xffffffffu, le);
            urng[k] = (le > lb) ? ((lb << 16) | le) : 0;
        }
    }
    __syncthreads();

    const int nchunks = (nlines + R - 1) / R;
    auto issue = [&](int c) {
        int b = c & 1;
        int l0 = c * R;
        int rc = min(R, nlines - l0);
        uint32_t bh = (uint32_t)((size_t)rc * sp * sizeof(float2));
        uint32_t ba = kSiddon ? (uint32_t)((size_t)rc * sp * sizeof(float)) : 0u;
        unsigned char* dst = buf0 + b * buf_bytes;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bars[b], bh + ba);
        bulk_g2s(dst, ghl + (long long)l0 * sp, bh, &bars[b]);
        if (kSiddon) bulk_g2s(dst + hl_bytes, gla + (long long)l0 * sp, ba, &bars[b]);
    };
    // per-line factors 1 / (l - perp) of chunk c into slot c & 1
    auto line_factors = [&](int c) {
        if (!kSiddon && tid < vcount * R) {
            const int v = tid / R, j = tid - (tid / R) * R;
            s_g[(c & 1) * kFpViews * kFpMaxLines + v * kFpMaxLines + j] =
                (float)(1.0 / ((double)(c * R + j) - s_perp[v]));
        }
    };
    if (tid == 0) issue(0);
    line_factors(0);

    // One barrier per chunk: after it every warp has finished chunk c - 1, so
    // buffer (c + 1) & 1 and factor slot (c + 1) & 1 may be refilled.
    const unsigned lpm1 = (unsigned)(lp - 1);
    bool ok = true;
    for (int c = 0; c < nchunks; c++) {
        const int b = c & 1;
        const int l0 = c * R;
        const int rc = min(R, nlines - l0);
        if (!mbar_wait(&bars[b], (uint32_t)((c >> 1) & 1), p.spin)) ok = false;
        if (!__syncthreads_and(ok)) {
            // chunk c's bulk copy is the only one in flight (chunk c + 1 is
            // issued after this barrier): the issuing thread waits for it,
            // bounded, so no copy lands in shared memory after the CTA exits
            if (tid == 0) {
                atomicExch(p.err, RN_ERR_TIMEOUT);
                mbar_wait(&bars[b], (uint32_t)((c >> 1) & 1));
            }
            ok = false;
            break;
        }
        if (tid == 0 && c + 1 < nchunks) issue(c + 1);
        const float2* HL = reinterpret_cast<const float2*>(buf0 + b * buf_bytes);
        const float* LA = reinterpret_cast<const float*>(buf0 + b * buf_bytes + hl_bytes);
        const float fl0 = (float)l0;
        // edge position of group k's lane at the chunk's first line, Xi0 + Xf0 +
        // (rhi + rlo) l0, split into an integer cell Xi (floor bias folded in)
        // and a small offset Xf with error-free steps: rhi l0 = pr + pe exactly,
        // pr = floor(pr) + pf exactly.  Per-line positions then stay below ~50
        // cells and keep ~1e-6 cells of precision.
        auto setup = [&](int k, int& Xi, float& Xf, float& r, const float*& g) {
            const float4 E = s_edge[gslot[k] & 0xffff];
            const float pr = E.z * fl0;
            const float pe = fmaf(E.z, fl0, -pr);
            const float py = __fadd_rd(pr, kFloorBias);
            const float pf = pr - (py - kFloorBias);
            Xi = __float_as_int(E.y) + (__float_as_int(py) - kFloorBiasBits) - kFloorBiasBits;
            Xf = (E.x + pf) + fmaf(E.w, fl0, pe);
            r = E.z;
            g = s_g + b * kFpViews * kFpMaxLines + (gslot[k] >> 16) * kFpMaxLines;
        };
        // prefix integral at this lane's edge on line j and the footprint
        // difference with the next lane's edge: cell kk and fraction f of the
        // padded position, floored by a round-down add against 1.5*2^23, and
        // one packed (P, a) entry read.  Positions beyond the padded line
        // clamp to its ends, where the prefix is 0 or the line total and the
        // value 0, so a ray that misses line j adds exactly 0.
        auto footprint = [&](float jf, int Xi, float Xf, float r, const float2* hrow) -> float {
            const float x = fmaf(r, jf, Xf);
            const float y = __fadd_rd(x, kFloorBias);
            const unsigned kk = min((unsigned)max(__float_as_int(y) + Xi, 0), lpm1);
            const unsigned pos = kk;
            const float f = x - (y - kFloorBias);
            const float2 h = hrow[pos];
            const float P = fmaf(f, h.y, h.x);
            return __shfl_down_sync(0xffffffffu, P, 1) - P;
        };
        // Siddon (kSiddon): lane = ray.  On band j (image row / column j, not
        // blended) the ray runs from its position at boundary j to boundary
        // j + 1; the band adds the integral of the row over that interval
        // divided by the interval's signed width r, taken from the two
        // positions' cells.  The second position is formed from the first's
        // fraction plus r, so the width keeps ~1e-7 cells of precision, and a
        // ray that stays inside one cell adds that cell's value exactly (also
        // for r = 0).  The epilogue multiplies by the ray length per band.
        auto band = [&](float jf, int Xi, float Xf, float r, float ir, const float2* hrow, const float* arow) -> float {
            const float x = fmaf(r, jf, Xf);
            const float y = __fadd_rd(x, kFloorBias);
            const int ka = __float_as_int(y) + Xi;
            const float fa = x - (y - kFloorBias);
            const float t = fa + r;
            const float yt = __fadd_rd(t, kFloorBias);
            const int kb = ka + (__float_as_int(yt) - kFloorBiasBits);
            const float fb = t - (yt - kFloorBias);
            const unsigned ua = min((unsigned)max(ka, 0), lpm1), ub = min((unsigned)max(kb, 0), lpm1);
            const unsigned pa = ua + (ua >> 4), pb = ub + (ub >> 4);
            const float2 ha = hrow[pa], hb = hrow[pb];
            const float aa = arow[pa];
            const float d = (hb.x - ha.x) + (fmaf(fb, arow[pb], hb.y) - fmaf(fa, aa, ha.y));
            return ka == kb ? aa : d * ir;
        };
        auto single = [&](int k, int J0, int J1) {
            int Xi;
            float Xf, r;
            const float* g;
            setup(k, Xi, Xf, r, g);
            const float2* hrow = HL + J0 * sp;
            const float* arow = LA + J0 * sp;
            float a = acc[k];
            float jf = (float)J0;
            if constexpr (kSiddon) {
                const float ir = 1.0f / r;
                for (int j = J0; j < J1; j++, jf += 1.f, hrow += sp, arow += sp)
                    a += band(jf, Xi, Xf, r, ir, hrow, arow);
            } else {
                for (int j = J0; j < J1; j++, jf += 1.f, hrow += sp)
                    a = fmaf(footprint(jf, Xi, Xf, r, hrow), g[j], a);
            }
            acc[k] = a;
        };
        // groups in pairs: where both have lines in this chunk, one loop over
        // the union of their ranges runs two independent chains (a group adds
        // exactly 0 on lines outside its range)
#pragma unroll
        for (int k = 0; k < kFpGroups; k += 2) {
            const int J0a = max((urng[k] >> 16) - l0, 0), J1a = min((urng[k] & 0xffff) - l0, rc);
            const int J0b = max((urng[k + 1] >> 16) - l0, 0), J1b = min((urng[k + 1] & 0xffff) - l0, rc);
            if (J0a < J1a && J0b < J1b) {   // warp-uniform
                int Xia, Xib;
                float Xfa, Xfb, ra, rb;
                const float *ga, *gb;
                setup(k, Xia, Xfa, ra, ga);
                setup(k + 1, Xib, Xfb, rb, gb);
                const int J0 = min(J0a, J0b), J1 = max(J1a, J1b);
                const float2* hrow = HL + J0 * sp;
                const float* arow = LA + J0 * sp;
                float aa = acc[k], ab = acc[k + 1];
                float jf = (float)J0;
                if constexpr (kSiddon) {
                    const float ira = 1.0f / ra, irb = 1.0f / rb;
                    for (int j = J0; j < J1; j++, jf += 1.f, hrow += sp, arow += sp) {
                        aa += band(jf, Xia, Xfa, ra, ira, hrow, arow);
                        ab += band(jf, Xib, Xfb, rb, irb, hrow, arow);
                    }
                } else {
                    for (int j = J0; j < J1; j++, jf += 1.f, hrow += sp) {
                        aa = fmaf(footprint(jf, Xia, Xfa, ra, hrow), ga[j], aa);
                        ab = fmaf(footprint(jf, Xib, Xfb, rb, hrow), gb[j], ab);
                    }
                }
                acc[k] = aa;
                acc[k + 1] = ab;
            } else if (J0a < J1a) {
                single(k, J0a, J1a);
            } else if (J0b < J1b) {
                single(k + 1, J0b, J1b);
            }
        }
        if (c + 1 < nchunks) line_factors(c + 1);
    }
    if (!ok) return;

    // epilogue: scale by L_u / (r_{u+1} - r_u) and store
    const float lenA = xcls ? p.d.dy : p.d.dx;
#pragma unroll
    for (int k = 0; k < kFpGroups; k++) {
        const int grp = warp + k * kFpWarps;
        if (grp >= ngroups) continue;
        const int v = grp / ngpv;
        const int u = (grp - v * ngpv) * kFpGroupRays + lane;
        if (lane >= kFpGroupRays || u >= nu) continue;
        const int gv = s_gv[v];
        const double* ed = p.edges + (long long)gv * (nu + 1);
        float scale;
        if constexpr (kSiddon) {
            // ray length per band: r cells along the band, one band across
            const double along = xcls ? p.d.dx : p.d.dy, across = xcls ? p.d.dy : p.d.dx;
            scale = (float)sqrt(ed[u] * ed[u] * along * along + across * across);
        } else {
            const float dr = (float)(ed[u + 1] - ed[u]);
            const ViewGeo& vg = p.views[gv];
            const float2 cs = p.cell[u];   // (cos a, sin a)
            const float Lw = xcls ? lenA / fabsf(vg.cosd * cs.x + vg.sind * cs.y)
                                  : lenA / fabsf(vg.sind * cs.x - vg.cosd * cs.y);
            scale = Lw / dr;
        }
        p.prj[fs.prj_off + (long long)u * fs.su + (long long)s_vl[v] * fs.sview] = acc[k] * scale;
    }
}

// ---------------------------------------------------------------------------
// BP edge tables.  One warp per (BP slice, view); 8 consecutive views per CTA
// so that the u-strided sinogram reads of neighbouring views share sectors.
//   matched (type 2): W_u = prj * L_u; entry e < nu = {Qhi, Qlo, W_e/(r_{e+1}-r_e), r_e}
//   reference (0/1):  W_u = prj * (L_u if type 0); entry k <= nu = {Uhi, Ulo, W_k, 0}
// with Q/U the FP64 prefix over u; stored at index e+1 after a guard entry.
// ---------------------------------------------------------------------------
__global__ void fan_table_kernel(const float* __restrict__ prj, const BpSlice* __restrict__ bps, int s_begin,
                                 int ns, const GeoSet* __restrict__ sets, const ViewGeo* __restrict__ views,
                                 const double* __restrict__ edges, const float2* __restrict__ cell, FanDims d,
                                 int type, float4* __restrict__ tab, long long tab_base) {
    int warp = threadIdx.x >> 5;
    int lane = threadIdx.x & 31;
    int si = blockIdx.y;
    if (si >= ns) return;
    const BpSlice bs = bps[s_begin + si];
    const GeoSet gs = sets[bs.set];
    int vl = blockIdx.x * 8 + warp;
    if (vl >= gs.nview) return;
    int gv = gs.view_off + vl;
    const ViewGeo vg = views[gv];
    const int nu = d.nu;
    const double* ed = edges + (long long)gv * (nu + 1);
    // per view: index 0 is a guard entry (prefix 0, slope 0), index e+1 holds
    // edge / cell e, index nu+1 the total with slope 0; indices outside the
    // detector therefore evaluate to 0 or the total without clamping
    float4* out = tab + (bs.table_off - tab_base) + (long long)vl * (nu + 2);
    if (lane == 0) out[0] = make_float4(0.f, 0.f, 0.f, type == RN_TYPE_MATCHED ? (float)ed[0] : 0.f);
    out += 1;
    const float lenA = vg.xcls ? d.dy : d.dx;
    double carry = 0.0;
    for (int u0 = 0; u0 < nu; u0 += 32) {
        int u = u0 + lane;
        double W = 0.0;
        if (u < nu) {
            float s = 0.f;
#pragma unroll
            for (int j = 0; j < kBpMix; j++) {
                float wj = bs.prj_w[j];
                if (wj == 0.f) continue;
                s += wj * __ldg(prj + bs.prj_off[j] + (long long)u * bs.su + (long long)vl * bs.sview);
            }
            if (type != RN_TYPE_FBP) {
                float2 cs = cell[u];
                float L = vg.xcls ? lenA / fabsf(vg.cosd * cs.x + vg.sind * cs.y)
                                  : lenA / fabsf(vg.sind * cs.x - vg.cosd * cs.y);
                s *= L;
            }
            // matched tables carry the sign and the 1/2 of the two-line average
            W = type == RN_TYPE_MATCHED ? (double)(s * (0.5f * vg.sigma)) : (double)s;
        }
        double incl = warp_incl_scan(W);
        double excl = carry + incl - W;
        if (u < nu) {
            float2 q = split_double(excl);
            if (type == RN_TYPE_MATCHED) {
                double dr = ed[u + 1] - ed[u];
                out[u] = make_float4(q.x, q.y, (float)(W / dr), (float)ed[u]);
            } else {
                out[u] = make_float4(q.x, q.y, (float)W, 0.f);
            }
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        float2 q = split_double(carry);
        out[nu] = make_float4(q.x, q.y, 0.f, type == RN_TYPE_MATCHED ? (float)ed[nu] : 0.f);
    }
}

// ---------------------------------------------------------------------------
// BP kernels.
// ---------------------------------------------------------------------------
struct BpParams {
    const ViewGeo* views;
    const GeoSet* sets;
    const BpSlice* bps;
    const float4* tab;
    long long tab_base;
    int s_begin;
    float* img;
    int* err;
    FanDims d;
    int accumulate;
    int type;
    int tiles_x, tiles_y;
    long long spin;    // polls of a chunk wait before it gives up (the plan's spin limit)
    int win;           // staged table entries per view
    // view split for small batches: CTA part k of a tile takes the k-th
    // share of the views and writes its partial image to parts + k *
    // part_stride (summed afterwards by bp_parts_sum_kernel)
    int nparts;
    long long part_stride;
    float* parts;
};

// out[i] = (accumulate ? out[i] : 0) + sum over k of parts[k * stride + i],
// the parts summed first, in a fixed order (deterministic; accumulating adds
// exactly the value a non-accumulating call writes).
__global__ void bp_parts_sum_kernel(float* __restrict__ out, const float* __restrict__ parts, int nparts,
                                    long long stride, long long n, int accumulate) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = 0.f;
        for (int k = 0; k < nparts; k++) v += parts[k * stride + i];
        out[i] = accumulate ? out[i] + v : v;
    }
}


// Per-view parameters the BP inner loop reads, staged in shared memory.
// Siddon BP table: per view, entry e holds the slope of ray e - 1 as hi / lo
// floats and the prefix C_e = sum_{u < e} c_u as hi / lo floats (FP64 scan),
// c_u = w_u * (ray length per band), w_u the sinogram value mixed over the
// slice's detector rows; entry 0 is a guard (C = 0) and entry nu + 1 holds
// the total.  c_u is C_(u+1) - C_u of two neighbouring entries.
__global__ void siddon_table_kernel(const float* __restrict__ prj, const BpSlice* __restrict__ bps, int s_begin,
                                    int ns, const GeoSet* __restrict__ sets, const ViewGeo* __restrict__ views,
                                    const double* __restrict__ cslopes, FanDims d, float4* __restrict__ tab,
                                    long long tab_base) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int si = blockIdx.y;
    if (si >= ns) return;
    const BpSlice bs = bps[s_begin + si];
    const GeoSet gs = sets[bs.set];
    const int vl = blockIdx.x * 8 + warp;
    if (vl >= gs.nview) return;
    const int gv = gs.view_off + vl;
    const int nu = d.nu;
    const double along = views[gv].xcls ? d.dx : d.dy, across = views[gv].xcls ? d.dy : d.dx;
    float4* out = tab + (bs.table_off - tab_base) + (long long)vl * (nu + 2);
    double carry = 0.0;
    for (int u0 = 0; u0 < nu; u0 += 32) {
        const int u = u0 + lane;
        double c = 0.0, r = 0.0;
        if (u < nu) {
            float w = 0.f;
#pragma unroll
            for (int k = 0; k < kBpMix; k++) {
                const float wk = bs.prj_w[k];
                if (wk == 0.f) continue;
                w += wk * __ldg(prj + bs.prj_off[k] + (long long)u * bs.su + (long long)vl * bs.sview);
            }
            r = cslopes[(long long)gv * (nu + 1) + u];
            c = (double)(w * (float)sqrt(r * r * along * along + across * across));
        }
        const double incl = carry + warp_incl_scan(c);
        if (u < nu) {
            const float rh = (float)r;
            const float2 q = split_double(incl);
            out[u + 1] = make_float4(rh, (float)(r - (double)rh), q.x, q.y);
        }
        carry = __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        const float2 q = split_double(carry);
        out[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        out[nu + 1] = make_float4(0.f, 0.f, q.x, q.y);
    }
}

// Pixel-driven BP table: per view, entry k = u + 1 (u = -1 .. nu) holds the
// slope r_u of the ray through the centre of cell u as hi / lo floats, dso^2
// P_u and dso^2 (P_{u+1} - P_u), P_u the sinogram value mixed over the slice's
// detector rows (P_{-1} = P_{nu} = 0: border addressing).  r_u for u = 0 .. nu
// comes from the cell-centre slope table; r_{-1} is r_0 turned by one cell
// pitch: with rho = kappa r = tan(psi), psi moving by +du (X class) or -du
// (Y class) per cell towards negative u.
__global__ void pd_table_kernel(const float* __restrict__ prj, const BpSlice* __restrict__ bps, int s_begin, int ns,
                                const GeoSet* __restrict__ sets, const ViewGeo* __restrict__ views,
                                const double* __restrict__ cslopes, FanDims d, float4* __restrict__ tab,
                                long long tab_base) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int si = blockIdx.y;
    if (si >= ns) return;
    const BpSlice bs = bps[s_begin + si];
    const GeoSet gs = sets[bs.set];
    const int vl = blockIdx.x * 8 + warp;
    if (vl >= gs.nview) return;
    const int gv = gs.view_off + vl;
    const int nu = d.nu;
    const int xcls = views[gv].xcls;
    const double dso2 = (double)d.dso * d.dso;
    float4* out = tab + (bs.table_off - tab_base) + (long long)vl * (nu + 2);
    auto value = [&](int u) -> float {
        if (u < 0 || u >= nu) return 0.f;
        float w = 0.f;
#pragma unroll
        for (int k = 0; k < kBpMix; k++) {
            const float wk = bs.prj_w[k];
            if (wk == 0.f) continue;
            w += wk * __ldg(prj + bs.prj_off[k] + (long long)u * bs.su + (long long)vl * bs.sview);
        }
        return w;
    };
    for (int k = lane; k < nu + 2; k += 32) {
        const int u = k - 1;
        double r;
        if (u >= 0) {
            r = cslopes[(long long)gv * (nu + 1) + u];
        } else {
            const double kap = xcls ? (double)d.dx / d.dy : (double)d.dy / d.dx;
            const double rho = kap * cslopes[(long long)gv * (nu + 1)], tn = tan((double)d.du);
            r = (xcls ? (rho + tn) / (1.0 - rho * tn) : (rho - tn) / (1.0 + rho * tn)) / kap;
        }
        const float p0 = value(u), p1 = value(u + 1);
        const float rh = (float)r;
        out[k] = make_float4(rh, (float)(r - (double)rh), (float)(dso2 * p0), (float)(dso2 * ((double)p1 - p0)));
    }
}

struct BpView {
    double pard, perpd;   // source coordinates (Siddon band positions)
    float par, perp, kappa, tA, tB, sigma;
    int xcls;
};

struct BpShared {
    ViewGeo rec[2][kBpViews];   // view records staged for the next chunk
    uint64_t bars[2];
    int elo[3][kBpViews];       // first staged table entry per view
    BpView vw[3][kBpViews];
};

// Edge index t of the matched parametrisation for a slope r
// (r = (q - par) / (l - perp) at lattice point (line l, position q)).
__device__ __forceinline__ float matched_t(const ViewGeo& vg, float r) {
    return vg.tA + vg.tB * atanf(vg.kappa * r);
}

// Matched backprojection: lane i of a warp owns pixel column x = X0 + i and
// kBmRows pixel rows from y0; lane 31 owns no pixel and only supplies the
// right edge of lane 30's column.  The staged table window T starts at table
// index ilo; entries carry the prefix (hi, lo), the slope scaled by sigma / 2
// and the edge slope r_e.
//
// Edge index t(r) = tA + tB atan(kappa r) as a cubic around the slope r_t at
// the lane's middle lattice point: along one lane the lattice points differ
// in one coordinate only, and the truncation stays below 4e-5 cells over 17
// points (it only selects the cell; the value inside it is exact).
struct TCubic {
    float rt, c0, c1, c2, c3;
};
__device__ __forceinline__ TCubic t_cubic(const BpView& vg, float rt) {
    const float ut = vg.kappa * rt;
    const float iw = __fdividef(1.0f, fmaf(ut, ut, 1.0f));
    const float k1 = vg.tB * vg.kappa * iw;
    TCubic c;
    c.rt = rt;
    c.c0 = fmaf(vg.tB, atanf(ut), vg.tA);
    c.c1 = k1;
    c.c2 = -k1 * vg.kappa * ut * iw;
    c.c3 = k1 * vg.kappa * vg.kappa * (fmaf(3.0f * ut, ut, -1.0f) * (1.0f / 3.0f)) * iw * iw;
    return c;
}

// H at slope r: prefix (hi) and the rest (lo + slope * (r - r_e)) of the
// table entry of the cell that contains r.
__device__ __forceinline__ void bp_h(const TCubic& c, float r, const float4* T, int ilo, int imax, float& hi,
                                     float& rest) {
    const float h = r - c.rt;
    const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
    // table index floor(t) + 1 for |t| < 2^22 via a round-down add; beyond
    // the detector it reaches a zero-slope guard entry
    int i = __float_as_int(__fadd_rd(t, 12582912.0f)) - (0x4B400000 - 1);
    i = min(max(i, ilo), imax);
    const float4 E = T[i - ilo];
    hi = E.x;
    rest = fmaf(E.z, r - E.w, E.y);
}

// X-class view (lattice lines are rows): the lane's lattice column q = x,
// lines y0 .. y0 + kBmRows.  Pixel (x, y) receives the footprint difference
// with the next lane's column on line y and, if line y + 1 exists, on line
// y + 1.
__device__ __forceinline__ void bp_matched_x(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                             int imax, int x, int y0, int ny) {
    const float A = (float)x - vg.par;
    // (approximate reciprocals: a relative error in 1 / (l - perp) scales all
    // slopes of a line alike)
    const TCubic c = t_cubic(vg, A * __fdividef(1.0f, (float)(y0 + kBmRows / 2) - vg.perp));
    float dprev = 0.f;
#pragma unroll
    for (int j = 0; j <= kBmRows; j++) {
        const float r = A * __fdividef(1.0f, (float)(y0 + j) - vg.perp);
        float hi, rest;
        bp_h(c, r, T, ilo, imax, hi, rest);
        const float nhi = __shfl_down_sync(0xffffffffu, hi, 1);
        const float nrest = __shfl_down_sync(0xffffffffu, rest, 1);
        const float d = (nhi - hi) + (nrest - rest);
        if (j > 0) acc[j - 1] += fmaf((y0 + j < ny) ? 1.f : 0.f, d, dprev);
        dprev = d;
    }
}

// Y-class view (lattice lines are columns): the lane's line l = x, lattice
// points q = y0 .. y0 + kBmRows.  Pixel (x, y) receives the difference along
// line x and, if line x + 1 exists, the next lane's difference along it.
__device__ __forceinline__ void bp_matched_y(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                             int imax, int x, int y0, int nx) {
    const float g = __fdividef(1.0f, (float)x - vg.perp);
    const float r0 = ((float)y0 - vg.par) * g;
    const TCubic c = t_cubic(vg, fmaf((float)(kBmRows / 2), g, r0));
    const float m = (x + 1 < nx) ? 1.f : 0.f;
    float hprev = 0.f, rprev = 0.f;
#pragma unroll
    for (int j = 0; j <= kBmRows; j++) {
        const float r = fmaf((float)j, g, r0);
        float hi, rest;
        bp_h(c, r, T, ilo, imax, hi, rest);
        if (j > 0) {
            const float d = (hi - hprev) + (rest - rprev);
            const float nd = __shfl_down_sync(0xffffffffu, d, 1);
            acc[j - 1] += fmaf(m, nd, d);
        }
        hprev = hi;
        rprev = rest;
    }
}

// Siddon backprojection (kMode 2), the exact transpose of the Siddon forward
// projection: pixel column q-range [q, q + 1] on the band between lattice
// lines l and l + 1 receives, from every ray u, c_u (its sinogram value times
// its length per band) times the fraction of the ray's band interval
// [pos_u(l), pos_u(l + 1)] inside [q, q + 1], where pos_u(l) = par +
// r_u (l - perp).  Written as F(q + 1) - F(q), with F(q) = sum_u c_u b_u(q)
// and b_u(q) the fraction of ray u's band interval below q: rays wholly below
// q give the table prefix C (hi / lo), so F needs the exact fraction only for
// the rays whose centre index u + 1/2 lies between the edge indices t of the
// lattice points (q, l) and (q, l + 1) (widened by 1e-3 against the cubic's
// truncation: a ray taken in that is wholly below or above q gets the
// fraction 1 or 0 exactly), usually one.  Positions increase with u where
// sigma > 0: the rays below q are then u < ua, else u > ub, whose sum is the
// total minus C_(ub+1); the total cancels in F(q + 1) - F(q).  X class: lane
// column q = x on lines y0 + j (F(x + 1) from the next lane); Y class: line l
// = x, positions q = y0 + j (the band's second line x + 1 from the next lane).
// The fraction of ray u below q: its position at line l relative to q, x_a =
// (par - q) + r (l - perp), from hi / lo parts (A = par - q and D = l - perp
// as hi / lo floats, r from the table) to ~1e-7 cells, x_b = x_a + r; the
// fraction is min(max(-min(x_a, x_b) / |r|, 0), 1), and a ray within 1e-6 of
// the line normal takes the point test x_a < 0.
__device__ __forceinline__ float siddon_below(const float4 E, float Ah, float Al, float Dh, float Dl) {
    const float xa = fmaf(E.x, Dh, Ah) + fmaf(E.y, Dh, fmaf(E.x, Dl, Al));
    const float ar = fabsf(E.x);
    const float lo = fminf(xa, xa + E.x);
    const float fr = fminf(fmaxf(__fdividef(-lo, ar), 0.f), 1.f);
    return ar > 1e-6f ? fr : (xa < 0.f ? 1.f : 0.f);
}

// floor(x) for |x| < 2^22 on the FMA / ALU pipes (round-down add of 1.5 * 2^23).
__device__ __forceinline__ int floor_small(float x) {
    return __float_as_int(__fadd_rd(x, 12582912.0f)) - 0x4B400000;
}

// F(q) = sum_u c_u b_u(q) (up to the total, for sigma < 0) as hi + rest, for
// the band between the lattice points with edge indices ta and tb.  Table
// indices clamp into the staged window [ilo, imax].  Kept out of line: the
// kernel's two unrolled 17-point loops with it inlined overflow the
// instruction cache (59.0 against 52.6 ms on the bench batch).
__device__ __noinline__ void siddon_F(const float4* T, int ilo, int imax, int nu, float sigma, float ta, float tb,
                                         float Ah, float Al, float Dh, float Dl, float& fhi, float& frest) {
    const float tmin = fminf(ta, tb), tmax = fmaxf(ta, tb);
    // first and last ray taken in (the staged window covers the tile's rays;
    // the clamps to it only keep the reads inside it)
    const int ua = max(max(-floor_small(0.5f + 1e-3f - tmin), 0), ilo - 1);
    const int ub = min(min(floor_small(tmax - 0.5f + 1e-3f), nu - 1), imax - 1);
    const float4 E0 = T[min(max(min(ua, nu), ilo), imax) - ilo];  // C_ua
    float ch = E0.z, cl = E0.w, part = 0.f;
    {   // the first ray taken in, without a branch: read at an index clamped
        // into the window, kept only when taken in
        const float4 E = T[min(ua + 1, imax) - ilo];
        const bool in = ua <= ub;
        const float c = (E.z - ch) + (E.w - cl);
        part = in ? c * siddon_below(E, Ah, Al, Dh, Dl) : 0.f;
        ch = in ? E.z : ch;
        cl = in ? E.w : cl;
    }
    for (int u = ua + 1; u <= ub; u++) {   // the rare further ones
        const float4 E = T[min(u + 1, imax) - ilo];
        const float c = (E.z - ch) + (E.w - cl);
        part = fmaf(c, siddon_below(E, Ah, Al, Dh, Dl), part);
        ch = E.z;
        cl = E.w;
    }
    // C_(ub+1) is the last entry read (C_ua when no ray was taken in)
    if (sigma > 0.f) {
        fhi = E0.z;
        frest = E0.w + part;
    } else {
        fhi = -ch;
        frest = part - cl;
    }
}

__device__ __forceinline__ void split_hilo(double v, float& h, float& l) {
    h = (float)v;
    l = (float)(v - (double)h);
}

// s + e = a + b exactly (TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ void bp_siddon_x(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                            int imax, int x, int y0, int nu) {
    const float A = (float)x - vg.par;
    const TCubic c = t_cubic(vg, A * __fdividef(1.0f, (float)(y0 + kBmRows / 2) - vg.perp));
    float Ah, Al, Dh0, Dl0;
    split_hilo(vg.pard - (double)x, Ah, Al);
    split_hilo((double)y0 - vg.perpd, Dh0, Dl0);
    float tp = 0.f;
#pragma unroll
    for (int j = 0; j <= kBmRows; j++) {
        const float h = A * __fdividef(1.0f, (float)(y0 + j) - vg.perp) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        if (j > 0) {
            // band y0 + j - 1: line y0 + j - 1 minus perp, stepped exactly from the first line
            float Dh, e, fhi, frest;
            two_sum(Dh0, (float)(j - 1), Dh, e);
            siddon_F(T, ilo, imax, nu, vg.sigma, tp, t, Ah, Al, Dh, Dl0 + e, fhi, frest);
            const float nhi = __shfl_down_sync(0xffffffffu, fhi, 1);
            const float nrest = __shfl_down_sync(0xffffffffu, frest, 1);
            acc[j - 1] += (nhi - fhi) + (nrest - frest);
        }
        tp = t;
    }
}

__device__ __forceinline__ void bp_siddon_y(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                            int imax, int x, int y0, int nu) {
    const float g = __fdividef(1.0f, (float)x - vg.perp);
    const float r0 = ((float)y0 - vg.par) * g;
    const TCubic c = t_cubic(vg, fmaf((float)(kBmRows / 2), g, r0));
    float Dh, Dl, Ah0, Al0;
    split_hilo((double)x - vg.perpd, Dh, Dl);
    split_hilo(vg.pard - (double)y0, Ah0, Al0);
    float hp = 0.f, rp = 0.f;
#pragma unroll
    for (int j = 0; j <= kBmRows; j++) {
        const float h = fmaf((float)j, g, r0) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        const float tn = __shfl_down_sync(0xffffffffu, t, 1);   // the band's second line, x + 1
        // position y0 + j: par minus it, stepped exactly from the first
        float Ah, e, fhi, frest;
        two_sum(Ah0, -(float)j, Ah, e);
        siddon_F(T, ilo, imax, nu, vg.sigma, t, tn, Ah, Al0 + e, Dh, Dl, fhi, frest);
        if (j > 0) acc[j - 1] += (fhi - hp) + (frest - rp);
        hp = fhi;
        rp = frest;
    }
}

// Reference-mode backprojection (kMode 0; DDBPFanKernelX/Y,
// DistanceDriven.cu:500-614): pixel (x, y) receives, per view, the mean of the
// pre-weighted detector prefix U over the interval between the detector
// coordinates t of its two edges taken on its centre line,
// (U(t2) - U(t1)) / (t2 - t1), U clamped to [0, nu] and the interval not
// (typeProjector 1 also weights it dso^2 / L^2 at the pixel centre).  On the
// column-warp tiles the edge coordinates come from the per-lane cubic: X
// class, lane column x evaluates its left edge (lattice column x) on the 16
// centre rows and takes the right edge from the next lane; Y class, lane
// column x (centre line x + 1/2) evaluates the 17 lattice points along it.
// A rounding of t moves both the prefix difference and the interval, so the
// ratio is insensitive to it (exactly so when both edges fall in one cell).
// Table entry e + 1 holds U at edge e as (hi, lo) and the value of cell e.
__device__ __forceinline__ void ref_u(float t, const float4* T, int ilo, int imax, int nu, float& hi, float& rest) {
    const float tc = fminf(fmaxf(t, 0.f), (float)nu);
    float fr;
    int i = floor_frac(tc, fr) + 1;
    i = min(max(i, ilo), imax);
    fr = tc - (float)(i - 1);
    const float4 E = T[i - ilo];
    hi = E.x;
    rest = fmaf(fr, E.z, E.y);
}

__device__ __forceinline__ void bp_ref_x(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                         int imax, int x, int y0, int nu, bool fbp, float dq, float dl, float dso2) {
    const float A = (float)x - vg.par;
    const TCubic c = t_cubic(vg, A * __fdividef(1.0f, (float)(y0 + kBmRows / 2) - vg.perp));
    const float aq = (A + 0.5f) * dq;
#pragma unroll
    for (int j = 0; j < kBmRows; j++) {
        const float D = (float)(y0 + j) + 0.5f - vg.perp;
        const float h = A * __fdividef(1.0f, D) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        float hi, rest;
        ref_u(t, T, ilo, imax, nu, hi, rest);
        const float nhi = __shfl_down_sync(0xffffffffu, hi, 1);
        const float nrest = __shfl_down_sync(0xffffffffu, rest, 1);
        const float nt = __shfl_down_sync(0xffffffffu, t, 1);
        float v = __fdividef((nhi - hi) + (nrest - rest), nt - t);
        if (fbp) {
            const float b = D * dl;
            v *= __fdividef(dso2, fmaf(aq, aq, b * b));
        }
        acc[j] += v;
    }
}

__device__ __forceinline__ void bp_ref_y(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                         int imax, int x, int y0, int nu, bool fbp, float dq, float dl, float dso2) {
    const float D = (float)x + 0.5f - vg.perp;
    const float g = __fdividef(1.0f, D);
    const float r0 = ((float)y0 - vg.par) * g;
    const TCubic c = t_cubic(vg, fmaf((float)(kBmRows / 2), g, r0));
    const float b = D * dl;
    float hprev = 0.f, rprev = 0.f, tprev = 0.f;
#pragma unroll
    for (int j = 0; j <= kBmRows; j++) {
        const float h = fmaf((float)j, g, r0) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        float hi, rest;
        ref_u(t, T, ilo, imax, nu, hi, rest);
        if (j > 0) {
            float v = __fdividef((hi - hprev) + (rest - rprev), t - tprev);
            if (fbp) {
                const float a = ((float)(y0 + j) - 0.5f - vg.par) * dq;
                v *= __fdividef(dso2, fmaf(a, a, b * b));
            }
            acc[j - 1] += v;
        }
        hprev = hi;
        rprev = rest;
        tprev = t;
    }
}

// Pixel-driven backprojection (kMode 3; bpFanKernel3D with the FBP weight,
// PixelDriven.cu:11-62): pixel (x, y) receives, per view, the sinogram value
// at the detector coordinate pu of the ray through its centre, interpolated
// linearly between cell centres (zero beyond the detector), times dso^2 / L^2,
// L the source-to-centre distance.  The edge-index cubic picks a cell u0 near
// pu; the rest is exact: with A = par - q_c and D = l_c - perp the centre's
// offsets from the source along / across the lines, x_u = A + r_u D is the
// offset of ray u0 from the centre along its line, r - r_u = -x_u / D, and
//   pu - u0 = tB atan(kappa (r - r_u) / (1 + kappa^2 r r_u))
//           = -tB dq dl x_u D / L^2 (1 + dq^2 A x_u / L^2)
// to second order in (r - r_u) (dq, dl the pixel pitches along / across the
// lines; L^2 = (A dq)^2 + (D dl)^2).  A, D and x_u are carried as hi / lo
// floats, so pu is good to ~1e-6 cells.  A pixel whose cell estimate is a
// hair off lands at a fraction just outside [0, 1] of the neighbouring
// interval, which is its exact linear extension.
__device__ __forceinline__ float pd_sample(const float4* T, int ilo, int imax, float t, float Ah, float Al, float Dh,
                                           float Dl, float cfrac, float dq, float dl) {
    // table index floor(pu) + 1 = floor(t - 1/2) + 1 (round-down add, |t| < 2^22)
    int k = __float_as_int(__fadd_rd(t - 0.5f, 12582912.0f)) - (0x4B400000 - 1);
    k = min(max(k, ilo), imax);
    const float4 E = T[k - ilo];
    const float xu = fmaf(E.x, Dh, Ah) + fmaf(E.y, Dh, fmaf(E.x, Dl, Al));
    const float a = Ah * dq, b = Dh * dl;
    const float il2 = __fdividef(1.0f, fmaf(a, a, b * b));
    const float xl = xu * il2;
    const float frac = cfrac * Dh * xl * fmaf(dq * a, xl, 1.0f);
    const float val = (k == 0 && frac < 0.f) ? 0.f : fmaf(frac, E.w, E.z);
    return val * il2;
}


// X-class view: lane column q = x, pixel rows y0 + j (centres l = y0 + j + 1/2).
__device__ __forceinline__ void bp_pixel_x(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                           int imax, int x, int y0, float dq, float dl) {
    const float A = (float)x + 0.5f - vg.par;
    const TCubic c = t_cubic(vg, A * __fdividef(1.0f, (float)(y0 + kBmRows / 2) - vg.perp));
    float Ah, Al, Dh0, Dl0;
    split_hilo(vg.pard - ((double)x + 0.5), Ah, Al);
    split_hilo(((double)y0 + 0.5) - vg.perpd, Dh0, Dl0);
    const float cfrac = -vg.tB * dq * dl;
#pragma unroll
    for (int j = 0; j < kBmRows; j++) {
        const float h = A * __fdividef(1.0f, (float)(y0 + j) + 0.5f - vg.perp) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        float Dh, e;
        two_sum(Dh0, (float)j, Dh, e);
        acc[j] += pd_sample(T, ilo, imax, t, Ah, Al, Dh, Dl0 + e, cfrac, dq, dl);
    }
}

// Y-class view: lane line l = x (centre x + 1/2), positions q = y0 + j + 1/2.
__device__ __forceinline__ void bp_pixel_y(float (&acc)[kBmRows], const BpView& vg, const float4* T, int ilo,
                                           int imax, int x, int y0, float dq, float dl) {
    const float g = __fdividef(1.0f, (float)x + 0.5f - vg.perp);
    const float r0 = ((float)y0 + 0.5f - vg.par) * g;
    const TCubic c = t_cubic(vg, fmaf((float)(kBmRows / 2) - 0.5f, g, r0));
    float Ah0, Al0, Dh, Dl;
    split_hilo(vg.pard - ((double)y0 + 0.5), Ah0, Al0);
    split_hilo(((double)x + 0.5) - vg.perpd, Dh, Dl);
    const float cfrac = -vg.tB * dq * dl;
#pragma unroll
    for (int j = 0; j < kBmRows; j++) {
        const float h = fmaf((float)j, g, r0) - c.rt;
        const float t = fmaf(h, fmaf(h, fmaf(h, c.c3, c.c2), c.c1), c.c0);
        float Ah, e;
        two_sum(Ah0, -(float)j, Ah, e);
        acc[j] += pd_sample(T, ilo, imax, t, Ah, Al0 + e, Dh, Dl, cfrac, dq, dl);
    }
}

// Warp 0 of a backprojection CTA prepares chunk c (views c*kBpViews ...) of
// its tile at (X0, Y0): lane = view * 4 + tile corner evaluates the edge index
// at its corner, a 4-lane min gives the first staged table entry, and the
// view's parameters go to slot c % 3.  Kept out of line: it runs once per
// chunk in one warp, and inlined its temporaries would raise the register
// count of the whole accumulation loop.
template <int kMode>
__device__ __noinline__ void bp_prep(BpShared* sh, const ViewGeo* src, int c, int nview, int X0, int Y0,
                                     int tabn, int win, const FanDims d) {
    const int lane = threadIdx.x & 31, v = lane >> 2, corner = lane & 3;
    const bool valid = c * kBpViews + v < nview;
    const ViewGeo& vg = src[valid ? v : 0];
    const int cx = corner & 1, cy = corner >> 1;
    const int xcls = vg.xcls;
    const float X = (float)(X0 + cx * kBmCols), Y = (float)(Y0 + cy * kBmTileY);
    const float l = xcls ? Y : X, q = xcls ? X : Y;
    float t = matched_t(vg, (q - (float)vg.par) / (l - (float)vg.perp));
    t = fminf(t, __shfl_xor_sync(0xffffffffu, t, 1));
    t = fminf(t, __shfl_xor_sync(0xffffffffu, t, 2));
    if (valid && corner == 0) {
        const int slot = c % 3;
        const int lo = (int)floorf(t) + 1 - 2;   // table index = edge/cell index + 1
        sh->elo[slot][v] = max(0, min(lo, tabn - win));
        BpView& w = sh->vw[slot][v];
        w.pard = vg.par;
        w.perpd = vg.perp;
        w.par = (float)vg.par;
        w.perp = (float)vg.perp;
        w.kappa = vg.kappa;
        w.tA = vg.tA;
        w.tB = vg.tB;
        w.sigma = vg.sigma;
        w.xcls = vg.xcls;
    }
}

// kMode: 0 reference-mode (typeProjector 0 / 1), 1 matched, 2 Siddon, 3 pixel-driven.
// Siddon tiles run three CTAs per SM (80 registers, 180 vs 174 Gupd/s at two
// CTAs); the DD modes keep the compiler's register choice (71 / 80).
template <int kMode>
__global__ void __launch_bounds__(kBpThreads, (kMode == 2 || kMode == 0) ? 3 : 0) fan_bp_kernel(BpParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    BpShared* sh = reinterpret_cast<BpShared*>(smem);
    size_t off = (sizeof(BpShared) + 127) & ~size_t(127);
    float4* const buf0 = reinterpret_cast<float4*>(smem + off);   // buffer b at buf0 + b * kBpViews * win

    const int tiles_per_slice = p.tiles_x * p.tiles_y;
    const int part = blockIdx.x % p.nparts;
    const int bid = blockIdx.x / p.nparts;
    const int si = bid / tiles_per_slice;
    const int ti = bid - si * tiles_per_slice;
    const int tyi = ti / p.tiles_x;
    const int txi = ti - tyi * p.tiles_x;
    const BpSlice bs = p.bps[p.s_begin + si];
    GeoSet gs = p.sets[bs.set];
    const int nu = p.d.nu, nx = p.d.nx, ny = p.d.ny;
    const float4* gtab = p.tab + (bs.table_off - p.tab_base);
    if (p.nparts > 1) {
        // this part's share of the views, in whole chunks
        const int nch = (gs.nview + kBpViews - 1) / kBpViews;
        const int cpp = (nch + p.nparts - 1) / p.nparts;
        const int vb = min(gs.nview, part * cpp * kBpViews), ve = min(gs.nview, (part + 1) * cpp * kBpViews);
        gs.view_off += vb;
        gs.nview = ve - vb;
        gtab += (long long)vb * (nu + 2);
    }
    const int tid = threadIdx.x;
    // Column-warp tiles: lane i of warp w owns pixel column X0 + i and rows
    // Y0 + 16 w .. + 15 (lane 31's column belongs to the next tile: it only
    // supplies edges).
    const int X0 = txi * kBmCols, Y0 = tyi * kBmTileY;
    const int lane = tid & 31, warp = tid >> 5;
    const int x0 = X0 + lane;
    const int y0 = Y0 + warp * kBmRows;
    const int tabn = nu + 2;   // table entries per view (guard + nu + total)

    if (tid == 0) {
        mbar_init(&sh->bars[0], 1);
        mbar_init(&sh->bars[1], 1);
        fence_mbar_init();
    }

    const int nchunks = (gs.nview + kBpViews - 1) / kBpViews;
    auto prep = [&](int c, const ViewGeo* src) {
        bp_prep<kMode>(sh, src, c, gs.nview, X0, Y0, tabn, p.win, p.d);
    };
    // tid 0: stage chunk c's table windows into buffer c & 1 and the view
    // records of chunk c + 1 into record slot (c + 1) & 1, on barrier c & 1.
    auto issue = [&](int c) {
        const int b = c & 1;
        const int vc = min(kBpViews, gs.nview - c * kBpViews);
        const int cnt = min(p.win, tabn);
        const int vn = c + 1 < nchunks ? min(kBpViews, gs.nview - (c + 1) * kBpViews) : 0;
        fence_proxy_async();
        mbar_arrive_expect_tx(&sh->bars[b], (uint32_t)(vc * cnt * sizeof(float4) + vn * sizeof(ViewGeo)));
        for (int v = 0; v < vc; v++) {
            const int vl = c * kBpViews + v;
            bulk_g2s(buf0 + (b * kBpViews + v) * p.win, gtab + (long long)vl * tabn + sh->elo[c % 3][v],
                     (uint32_t)(cnt * sizeof(float4)), &sh->bars[b]);
        }
        if (vn > 0)
            bulk_g2s(sh->rec[(c + 1) & 1], p.views + gs.view_off + (c + 1) * kBpViews,
                     (uint32_t)(vn * sizeof(ViewGeo)), &sh->bars[b]);
    };

    if (tid < 32) prep(0, p.views + gs.view_off);
    __syncthreads();
    if (tid == 0) issue(0);

    // accumulators: acc[j] = pixel (x0, y0 + j)
    float acc[kBmRows];
#pragma unroll
    for (int a = 0; a < kBmRows; a++) acc[a] = 0.f;

    // One barrier per chunk: after it every warp has finished chunk c - 1, so
    // buffer (c + 1) & 1 and record slot c & 1 may be refilled; window and
    // parameter slots rotate over three chunks because warp 0 prepares chunk
    // c + 1 while other warps may still compute chunk c - 1.
    bool ok = true;
    for (int c = 0; c < nchunks; c++) {
        const int b = c & 1;
        if (!mbar_wait(&sh->bars[b], (uint32_t)((c >> 1) & 1), p.spin)) ok = false;
        if (tid < 32 && c + 1 < nchunks) prep(c + 1, sh->rec[(c + 1) & 1]);
        if (!__syncthreads_and(ok)) {
            // chunk c's copies are the only ones in flight: wait for them
            // (bounded) before the CTA gives its shared memory back
            if (tid == 0) {
                atomicExch(p.err, RN_ERR_TIMEOUT);
                mbar_wait(&sh->bars[b], (uint32_t)((c >> 1) & 1));
            }
            ok = false;
            break;
        }
        if (tid == 0 && c + 1 < nchunks) issue(c + 1);
        const int slot = c % 3;
        const int vc = min(kBpViews, gs.nview - c * kBpViews);
        for (int v = 0; v < vc; v++) {
            const BpView vg = sh->vw[slot][v];
            const float4* T = buf0 + (b * kBpViews + v) * p.win;
            const int ilo = sh->elo[slot][v];
            const int cnt = min(p.win, tabn);
            const int imax = ilo + cnt - 1;   // <= nu + 1
            if (kMode == 3) {
                if (vg.xcls) bp_pixel_x(acc, vg, T, ilo, imax, x0, y0, p.d.dx, p.d.dy);
                else bp_pixel_y(acc, vg, T, ilo, imax, x0, y0, p.d.dy, p.d.dx);
            } else if (kMode == 2) {
                if (vg.xcls) bp_siddon_x(acc, vg, T, ilo, imax, x0, y0, nu);
                else bp_siddon_y(acc, vg, T, ilo, imax, x0, y0, nu);
            } else if (kMode == 1) {
                if (vg.xcls) bp_matched_x(acc, vg, T, ilo, imax, x0, y0, ny);
                else bp_matched_y(acc, vg, T, ilo, imax, x0, y0, nx);
            } else {
                const bool fbp = p.type == RN_TYPE_FBP;
                const float dso2 = p.d.dso * p.d.dso;
                if (vg.xcls) bp_ref_x(acc, vg, T, ilo, imax, x0, y0, nu, fbp, p.d.dx, p.d.dy, dso2);
                else bp_ref_y(acc, vg, T, ilo, imax, x0, y0, nu, fbp, p.d.dy, p.d.dx, dso2);
            }
        }
    }
    if (!ok) return;

    float* out = (p.nparts > 1 ? p.parts + part * p.part_stride : p.img) + bs.img_off;
    const bool add = p.nparts == 1 && p.accumulate;
    if (lane < kBmCols && x0 < nx) {
#pragma unroll
        for (int j = 0; j < kBmRows; j++) {
            const int iy = y0 + j;
            if (iy < ny) {
                float* q = out + (long long)x0 * p.d.isx + (long long)iy * p.d.isy;
                *q = add ? (*q + acc[j]) : acc[j];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
int fan_fp_views(int nu) {
    const int ngpv = (std::max(nu, 1) + 30) / 31;   // groups of 31 rays per view
    // the group slots of the smaller of the two CTA shapes (work items serve both modes)
    constexpr int slots = std::min(FpCfg<false>::groups * FpCfg<false>::warps, FpCfg<true>::groups * FpCfg<true>::warps);
    return std::min(kFpViews, slots / ngpv);
}

// DD lines are packed (P, a) float2 entries; Siddon lines add a value array
static size_t fp_smem_bytes(int nu, int sp, int R, bool siddon) {
    size_t off = kFpHeader + sizeof(float4) * (size_t)fan_fp_views(nu) * (nu + 1);
    off = (off + 127) & ~size_t(127);
    return off + 2 * (size_t)R * sp * (sizeof(float2) + (siddon ? sizeof(float) : 0));
}

static size_t bp_smem_bytes(int win) {
    return ((sizeof(BpShared) + 127) & ~size_t(127)) + 2 * (size_t)kBpViews * win * sizeof(float4);
}

// Padding (entries per side) of the FP line arrays needed by one view: the
// widest footprint along a line anywhere in the image (distance dmax_mm from
// the source at most, stretched by 1/cos of the steepest ray) plus one line's
// advance of the steepest ray (visited line ranges are widened by one line)
// and two entries of slack.  Visited positions then stay inside the array.
static double fp_margin_view(double rmax_abs, double kappa, double pix_along, double dmax_mm, double du) {
    double kr = kappa * rmax_abs;
    double foot = dmax_mm * du * std::sqrt(1.0 + kr * kr) / pix_along;
    return foot + rmax_abs + 2.0;
}

// Opt the large-shared-memory kernels in to the full per-CTA budget once per
// device (at plan creation), so that projection calls themselves only launch.
static std::mutex g_attr_mu;
static std::vector<char> g_attr_done;

int fan_kernel_attributes() {
    int dev = 0;
    RN_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if ((int)g_attr_done.size() <= dev) g_attr_done.resize(dev + 1, 0);
    if (g_attr_done[dev]) return RN_OK;
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_fp_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_fp_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_bp_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_bp_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_bp_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    RN_CUDA_TRY(cudaFuncSetAttribute(fan_bp_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
    g_attr_done[dev] = 1;
    return RN_OK;
}

int fan_build_geometry(rn_fan_plan* p, const float* host_deg, FanGeoHost& gh) {
    const RnFanGeom& g = p->g;
    const int nu = g.nu;
    const int64_t V = p->total_views;
    const double du = g.du, off_u = g.off_u;

    // per-edge (sin, cos) of the fan angle gamma_e; edge e sits at
    // a_e + du/2 of cell e (DistanceDriven.cu:83,90)
    std::vector<double2>& esc = gh.esc;
    esc.resize(nu + 1);
    for (int e = 0; e <= nu; e++) {
        double gam = (-((double)e - 0.5 - (nu - 1) / 2.0) - off_u) * du;
        esc[e] = make_double2(std::sin(gam), std::cos(gam));
    }
    std::vector<float2>& cell = gh.cell;
    cell.resize(nu);
    for (int u = 0; u < nu; u++) {
        double a = (-((double)u - (nu - 1) / 2.0) - off_u) * du;
        cell[u] = make_float2((float)std::cos(a), (float)std::sin(a));
    }

    std::vector<ViewGeo>& vg = gh.views;
    std::vector<double2>& vcs = gh.vcs;
    std::vector<int>& vx = gh.vx;
    std::vector<int>& perm = gh.perm;
    vg.resize(V);
    vcs.resize(V);
    vx.resize(V);
    perm.resize(V);
    const double dmax_mm = g.dso + std::sqrt(std::pow(g.nx * (double)g.dx / 2 + std::fabs(g.cx), 2) +
                                             std::pow(g.ny * (double)g.dy / 2 + std::fabs(g.cy), 2));
    double margin = 0.0;
    auto slope = [&](int xc, double c, double s, int e) {
        double sn = esc[e].x * c - esc[e].y * s;
        double cn = esc[e].y * c + esc[e].x * s;
        return xc ? (sn * g.dy) / (cn * g.dx) : (cn * g.dx) / (sn * g.dy);
    };
    for (size_t si = 0; si < p->h_sets.size(); si++) {
        GeoSet& gs = p->h_sets[si];
        int nxv = 0;
        for (int k = 0; k < gs.nview; k++) {
            int v = gs.view_off + k;
            double th = (double)host_deg[v];
            double c = std::cos(th), s = std::sin(th);
            // class rule of the reference host code (DistanceDriven.cu:302), in
            // float: ties of the rounded values go to the Y class
            const float degf = host_deg[v];
            int xc = std::fabs(std::cos(degf)) > std::fabs(std::sin(degf)) ? 1 : 0;
            double sx = (g.dso * s - g.cx) / g.dx + g.nx / 2.0;
            double sy = (-g.dso * c - g.cy) / g.dy + g.ny / 2.0;
            ViewGeo& q = vg[v];
            q.xcls = xc;
            q.par = xc ? sx : sy;
            q.perp = xc ? sy : sx;
            q.cosd = (float)c;
            q.sind = (float)s;
            double kap = xc ? g.dx / g.dy : g.dy / g.dx;
            q.kappa = (float)kap;
            double tB = xc ? -1.0 / du : 1.0 / du;
            int em = nu / 2;
            double rm = slope(xc, c, s, em);
            q.tB = (float)tB;
            q.tA = (float)((double)em - tB * std::atan(kap * rm));
            double r0 = slope(xc, c, s, 0), r1 = slope(xc, c, s, nu);
            q.rmin = (float)std::min(r0, r1);
            q.rmax = (float)std::max(r0, r1);
            margin = std::max(margin, fp_margin_view(std::max(std::fabs(r0), std::fabs(r1)), kap,
                                                     xc ? g.dx : g.dy, dmax_mm, du));
            int nl = xc ? g.ny : g.nx;
            double side = (nl / 2.0 - q.perp) > 0 ? 1.0 : -1.0;
            q.sigma = (float)((r1 > r0 ? 1.0 : -1.0) * side);
            q.pad[0] = q.pad[1] = q.pad[2] = 0;
            vcs[v] = make_double2(c, s);
            vx[v] = xc;
            if (xc) nxv++;
            // the source must lie outside the image across the lines
            if (std::fabs(q.perp - nl / 2.0) <= nl / 2.0 + 1.0)
                return set_error(RN_ERR_ARG, "fan geometry: source inside the image footprint");
        }
        gs.nxv = nxv;
        int a = 0, b = nxv;
        for (int k = 0; k < gs.nview; k++) {
            int v = gs.view_off + k;
            if (vx[v]) perm[gs.view_off + a++] = k;
            else perm[gs.view_off + b++] = k;
        }
    }
    if (std::fabs(nu * du / 2.0) >= M_PI / 4)
        return set_error(RN_ERR_ARG, "fan geometry: fan half-angle must be below 45 degrees");
    if (margin > 4096) return set_error(RN_ERR_ARG, "fan geometry: footprints too wide for the line arrays");
    p->dims.margin = (int)std::ceil(margin);
    p->dims.lpx = (g.nx + 1 + 2 * p->dims.margin + 3) & ~3;
    p->dims.lpy = (g.ny + 1 + 2 * p->dims.margin + 3) & ~3;
    p->dims.spx = line_stride(p->dims.lpx);
    p->dims.spy = line_stride(p->dims.lpy);

    // slopes of the rays through the cell centres (the Siddon pair): the same
    // table with the fan angle of cell u itself (entry nu repeats a spacing on)
    gh.csc.resize(nu + 1);
    for (int e = 0; e <= nu; e++) {
        double gam = (-((double)e - (nu - 1) / 2.0) - off_u) * du;
        gh.csc[e] = make_double2(std::sin(gam), std::cos(gam));
    }
    p->h_sets.shrink_to_fit();
    return RN_OK;
}

int fan_slope_tables(rn_fan_plan* p, const double2* d_vcs, const int* d_vx, const double2* d_esc,
                     const double2* d_csc, cudaStream_t st) {
    const RnFanGeom& g = p->g;
    const long long n = (long long)p->total_views * (g.nu + 1);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    edge_slope_kernel<<<blocks, 256, 0, st>>>(p->d_edges, d_vcs, d_vx, d_esc, (int)p->total_views, g.nu, g.dx, g.dy);
    RN_CUDA_TRY(cudaGetLastError());
    edge_slope_kernel<<<blocks, 256, 0, st>>>(p->d_cslopes, d_vcs, d_vx, d_csc, (int)p->total_views, g.nu, g.dx,
                                              g.dy);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

static int fp_lines_for_smem(int nu, int sp, bool siddon) {
    int R = kFpMaxLines;
    while (R > 1 && fp_smem_bytes(nu, sp, R, siddon) > (size_t)kSmemBudget) R--;
    return R;
}

static int fp_lines_max(const rn_fan_plan* p, bool siddon) {
    return std::min(fp_lines_for_smem(p->dims.nu, p->dims.spx, siddon),
                    fp_lines_for_smem(p->dims.nu, p->dims.spy, siddon));
}

int fan_fp_lines_max(const rn_fan_plan* p) { return fp_lines_max(p, false); }

int fan_project(rn_fan_plan* p, float* d_prj, const float* d_img, cudaStream_t st, bool siddon) {
    const FanDims& d = p->dims;
    const int nfp = (int)p->h_fp.size();
    const int Rmax = fp_lines_max(p, siddon);
    const int R = p->fp_R > 0 ? std::min(p->fp_R, Rmax) : Rmax;
    if (fp_smem_bytes(d.nu, std::max(d.spx, d.spy), R, siddon) > (size_t)kSmemBudget)
        return set_error(RN_ERR_ARG, "fan projection: image lines too long for shared memory");
    const size_t smem = fp_smem_bytes(d.nu, std::max(d.spx, d.spy), R, siddon);
    // slices are processed in waves of at most `slots` line buffers
    const long long slot = p->line_slot_elems;
    const int slots = (int)std::max<long long>(1, std::min<long long>(nfp, p->fp_slots));
    int wbeg = 0;
    for (int s0 = 0; s0 < nfp; s0 += slots) {
        int ns = std::min(slots, nfp - s0);
        long long warps = (long long)ns * (d.nx + d.ny);
        {
            LaunchScope ls0(p, st, 0);
            fan_lines_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(
                d_img, siddon ? p->d_fps : p->d_fp, s0, ns, d, p->d_hl, p->d_la, slot, siddon ? 1 : 0);
        }
        RN_CUDA_TRY(cudaGetLastError());
        int wend = wbeg;
        while (wend < p->n_fp_work && p->h_fp_work[4 * wend] < s0 + ns) wend++;
        if (wend > wbeg) {
            FpParams fp;
            fp.views = p->d_views;
            fp.edges = siddon ? p->d_cslopes : p->d_edges;
            fp.cell = p->d_cell;
            fp.perm = p->d_perm;
            fp.sets = p->d_sets;
            fp.fps = siddon ? p->d_fps : p->d_fp;
            fp.work = p->d_fp_work + wbeg;
            fp.hl = p->d_hl;
            fp.la = p->d_la;
            fp.slot_elems = slot;
            fp.slot_base = s0;
            fp.prj = d_prj;
            fp.err = p->d_err;
            fp.d = d;
            fp.R = R;
            fp.vt = fan_fp_views(d.nu);
            fp.spin = p->spin_limit;
            LaunchScope ls1(p, st, 1);
            if (siddon) fan_fp_kernel<true><<<wend - wbeg, FpCfg<true>::threads, smem, st>>>(fp);
            else fan_fp_kernel<false><<<wend - wbeg, FpCfg<false>::threads, smem, st>>>(fp);
            RN_CUDA_TRY(cudaGetLastError());
        }
        wbeg = wend;
    }
    return RN_OK;
}

// Backprojection slices of `type`: Siddon rows per image slice; matched: the
// transpose of the FP z mixing; reference modes and pixel-driven: rows mixed
// at the slice's v.
static const std::vector<BpSlice>& bp_slices(const rn_fan_plan* p, int type) {
    return type == RN_TYPE_SIDDON ? p->h_bps : (type == RN_TYPE_MATCHED) ? p->h_bp : p->h_bpr;
}

// End of the launch that starts at slice s0: as many slices as fit in the
// table scratch (at least one).
static int bp_wave_end(const rn_fan_plan* p, const std::vector<BpSlice>& bps, int s0) {
    const int nbp = (int)bps.size();
    const long long base = bps[s0].table_off;
    int s1 = s0;
    while (s1 < nbp) {
        const GeoSet& gs = p->h_sets[bps[s1].set];
        long long end = bps[s1].table_off + (long long)gs.nview * (p->dims.nu + 2);
        if (end - base > p->tab_elems && s1 > s0) break;
        s1++;
    }
    return s1;
}

static int bp_max_views(const rn_fan_plan* p, const std::vector<BpSlice>& bps, int s0, int s1) {
    int maxv = 0;
    for (int s = s0; s < s1; s++) maxv = std::max(maxv, p->h_sets[bps[s].set].nview);
    return maxv;
}

// A batch too small to fill the GPU (one launch, fewer than two CTAs per
// resident slot) splits every tile's views over several CTAs.
static int bp_parts(const rn_fan_plan* p, const std::vector<BpSlice>& bps, int s0, int s1) {
    if (s0 != 0 || s1 != (int)bps.size()) return 1;
    if (p->bp_nparts > 0) {   // tuned
        const int nch = (bp_max_views(p, bps, s0, s1) + kBpViews - 1) / kBpViews;
        return std::max(1, std::min(std::min(p->bp_nparts, kBpMaxParts), nch));
    }
    const FanDims& d = p->dims;
    const long long tiles = (long long)((d.nx + kBmCols - 1) / kBmCols) * ((d.ny + kBmTileY - 1) / kBmTileY);
    const long long ctas = (long long)(s1 - s0) * tiles;
    const long long target = 2LL * 148 * 3;
    if (ctas >= target) return 1;
    const int nch = (bp_max_views(p, bps, s0, s1) + kBpViews - 1) / kBpViews;
    const int want = (int)std::min<long long>(std::min<long long>(kBpMaxParts, (target + ctas - 1) / ctas), nch);
    return std::max(1, want);
}

int fan_bp_split(const rn_fan_plan* p, int type, int* first_wave_slices) {
    const std::vector<BpSlice>& bps = bp_slices(p, type);
    if (bps.empty()) {
        if (first_wave_slices) *first_wave_slices = 0;
        return 1;
    }
    const int s1 = bp_wave_end(p, bps, 0);
    if (first_wave_slices) *first_wave_slices = s1;
    return bp_parts(p, bps, 0, s1);
}

int fan_backproject(rn_fan_plan* p, float* d_img, const float* d_prj, int type, int accumulate, cudaStream_t st) {
    const FanDims& d = p->dims;
    const bool siddon = type == RN_TYPE_SIDDON, pixel = type == RN_TYPE_PIXEL;
    const std::vector<BpSlice>& bps = bp_slices(p, type);
    const BpSlice* dbp = siddon ? p->d_bps : (type == RN_TYPE_MATCHED) ? p->d_bp : p->d_bpr;
    const int nbp = (int)bps.size();
    const int win = p->table_win_m;
    const size_t smem = bp_smem_bytes(win);
    const int tiles_x = (d.nx + kBmCols - 1) / kBmCols, tiles_y = (d.ny + kBmTileY - 1) / kBmTileY;
    int s0 = 0;
    while (s0 < nbp) {
        const int s1 = bp_wave_end(p, bps, s0);
        const long long base = bps[s0].table_off;
        const int ns = s1 - s0;
        const int maxv = bp_max_views(p, bps, s0, s1);
        dim3 tg((maxv + 7) / 8, ns);
        {
            LaunchScope ls2(p, st, 2);
            if (siddon)
                siddon_table_kernel<<<tg, 256, 0, st>>>(d_prj, dbp, s0, ns, p->d_sets, p->d_views, p->d_cslopes, d,
                                                        p->d_tab, base);
            else if (pixel)
                pd_table_kernel<<<tg, 256, 0, st>>>(d_prj, dbp, s0, ns, p->d_sets, p->d_views, p->d_cslopes, d,
                                                    p->d_tab, base);
            else
                fan_table_kernel<<<tg, 256, 0, st>>>(d_prj, dbp, s0, ns, p->d_sets, p->d_views, p->d_edges, p->d_cell,
                                                     d, type, p->d_tab, base);
        }
        RN_CUDA_TRY(cudaGetLastError());
        BpParams bp;
        bp.views = p->d_views;
        bp.sets = p->d_sets;
        bp.bps = dbp;
        bp.tab = p->d_tab;
        bp.tab_base = base;
        bp.s_begin = s0;
        bp.img = d_img;
        bp.err = p->d_err;
        bp.d = d;
        bp.accumulate = accumulate;
        bp.type = type;
        bp.spin = p->spin_limit;
        bp.tiles_x = tiles_x;
        bp.tiles_y = tiles_y;
        bp.win = win;
        // the plan sized d_bp_parts for the split of every type
        bp.nparts = 1;
        bp.part_stride = 0;
        bp.parts = nullptr;
        const int want = bp_parts(p, bps, s0, s1);
        if (want > 1 && (long long)want * p->img_elems <= p->bp_parts_cap) {
            bp.nparts = want;
            bp.part_stride = p->img_elems;
            bp.parts = p->d_bp_parts;
        }
        unsigned grid = (unsigned)(ns * tiles_x * tiles_y * bp.nparts);
        LaunchScope ls3(p, st, 3);
        if (pixel) fan_bp_kernel<3><<<grid, kBpThreads, smem, st>>>(bp);
        else if (siddon) fan_bp_kernel<2><<<grid, kBpThreads, smem, st>>>(bp);
        else if (type == RN_TYPE_MATCHED) fan_bp_kernel<1><<<grid, kBpThreads, smem, st>>>(bp);
        else fan_bp_kernel<0><<<grid, kBpThreads, smem, st>>>(bp);
        RN_CUDA_TRY(cudaGetLastError());
        if (bp.nparts > 1) {
            LaunchScope ls4(p, st, 4);
            const long long n = p->img_elems;
            bp_parts_sum_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 148LL * 8), 256, 0, st>>>(
                d_img, bp.parts, bp.nparts, bp.part_stride, n, accumulate);
            RN_CUDA_TRY(cudaGetLastError());
        }
        s0 = s1;
    }
    return RN_OK;
}

}  // namespace rn

// ===========================================================================
// Forward projection without any allocation.
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory pool or under a strict memory budget, real-time or
// embedded pipelines that must not call cudaMalloc after start-up, and
// plugins that are only handed device pointers.  rn_fan_project_noalloc
// serves them: it is the forward projector above (same kernels, same
// arithmetic) with every piece of its scratch -- geometry tables, slopes and
// the line prefix arrays -- placed in the fixed device array below instead of
// a plan.  The array is kNoAllocScratchBytes (16 MiB) and stays resident on
// every GPU that loads this library until the process exits.
// ===========================================================================
namespace rn {

constexpr size_t kNoAllocScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the symbol is
// only a host-side stand-in, so the address is looked up once per device
// (with that device current) and passed to the kernels.
static std::mutex g_noalloc_mu;
static std::vector<unsigned char*> g_noalloc_ptr;

static int noalloc_scratch(unsigned char** out) {
    int dev = 0;
    RN_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if ((int)g_noalloc_ptr.size() <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
    if (!g_noalloc_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(ptr);
    }
    *out = g_noalloc_ptr[dev];
    return RN_OK;
}

static size_t na_align(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace rn

extern "C" int rn_fan_project_noalloc(float* d_prj, const float* d_img, const float* host_deg, int nx, int ny,
                                      float dx, float dy, int nu, int nview, float da, float off_a, float dsd,
                                      float dso, void* stream) {
    using namespace rn;
    clear_error();
    if (!d_prj || !d_img || !host_deg) return set_error(RN_ERR_ARG, "null argument");
    if (nx <= 0 || ny <= 0 || nu <= 0 || nview <= 0 || !(dx > 0 && dy > 0 && da > 0 && dsd > 0 && dso > 0))
        return set_error(RN_ERR_ARG, "sizes, pitches and distances must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    FanDims d;
    d.nx = nx;
    d.ny = ny;
    d.nu = nu;
    d.dx = dx;
    d.dy = dy;
    d.du = da;
    d.off_u = off_a;
    d.dsd = dsd;
    d.dso = dso;
    d.isx = ny;
    d.isy = 1;
    const int VT = fan_fp_views(nu);
    if (VT < 1) return set_error(RN_ERR_ARG, "too many detector channels for the forward projector");
    if (nx >= (1 << 15) || ny >= (1 << 15)) return set_error(RN_ERR_ARG, "image too large");

    // line padding: same bound as the plan path (fan_build_geometry)
    const double dmax_mm = dso + std::sqrt(std::pow(nx * (double)dx / 2, 2) + std::pow(ny * (double)dy / 2, 2));
    double margin = 0.0;
    for (int v = 0; v < nview; v++) {
        const float degf = host_deg[v];
        double th = (double)degf;
        int xc = std::fabs(std::cos(degf)) > std::fabs(std::sin(degf)) ? 1 : 0;
        double kap = xc ? (double)dx / dy : (double)dy / dx;
        double rmax = 0.0;
        for (int e : {0, nu}) {
            double gam = (-((double)e - 0.5 - (nu - 1) / 2.0) - off_a) * (double)da;
            double sn = std::sin(gam - th), cn = std::cos(gam - th);
            rmax = std::max(rmax, std::fabs(xc ? (sn * dy) / (cn * dx) : (cn * dx) / (sn * dy)));
        }
        margin = std::max(margin, fp_margin_view(rmax, kap, xc ? dx : dy, dmax_mm, da));
    }
    if (margin > 4096) return set_error(RN_ERR_ARG, "fan geometry: footprints too wide for the line arrays");
    d.margin = (int)std::ceil(margin);
    d.lpx = (nx + 1 + 2 * d.margin + 3) & ~3;
    d.lpy = (ny + 1 + 2 * d.margin + 3) & ~3;
    d.spx = line_stride(d.lpx);
    d.spy = line_stride(d.lpy);

    // scratch layout (offsets in bytes, 256-aligned)
    const int nwork_max = (nview + VT - 1) / VT + 2;
    const long long slot = (long long)ny * d.spx + (long long)nx * d.spy;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = na_align(off + bytes);
        return o;
    };
    const size_t o_err = take(sizeof(int));
    const size_t o_set = take(sizeof(GeoSet));
    const size_t o_fp = take(sizeof(FpSlice));
    const size_t o_views = take(sizeof(ViewGeo) * nview);
    const size_t o_perm = take(sizeof(int) * nview);
    const size_t o_work = take(sizeof(int4) * nwork_max);
    const size_t o_cell = take(sizeof(float2) * nu);
    const size_t o_vcs = take(sizeof(double2) * nview);
    const size_t o_vx = take(sizeof(int) * nview);
    const size_t o_esc = take(sizeof(double2) * (nu + 1));
    const size_t host_bytes = off;   // everything above is staged from the host
    const size_t o_edges = take(sizeof(double) * (size_t)nview * (nu + 1));
    const size_t o_hl = take(sizeof(float2) * (size_t)slot);
    const size_t o_la = take(sizeof(float) * (size_t)slot);
    if (off > kNoAllocScratchBytes)
        return set_error(RN_ERR_ARG, "rn_fan_project_noalloc: this geometry needs " + std::to_string(off) +
                                         " bytes of scratch, more than its fixed " +
                                         std::to_string(kNoAllocScratchBytes) + " bytes");
    const int R = std::min(fp_lines_for_smem(nu, d.spx, false), fp_lines_for_smem(nu, d.spy, false));
    const size_t smem = fp_smem_bytes(nu, std::max(d.spx, d.spy), R, false);
    if (smem > (size_t)kSmemBudget) return set_error(RN_ERR_ARG, "image lines too long for shared memory");

    // host-side tables, same quantities as fan_build_geometry
    std::vector<unsigned char> h(host_bytes, 0);
    ViewGeo* vg = reinterpret_cast<ViewGeo*>(h.data() + o_views);
    int* perm = reinterpret_cast<int*>(h.data() + o_perm);
    int4* work = reinterpret_cast<int4*>(h.data() + o_work);
    float2* cell = reinterpret_cast<float2*>(h.data() + o_cell);
    double2* vcs = reinterpret_cast<double2*>(h.data() + o_vcs);
    int* vx = reinterpret_cast<int*>(h.data() + o_vx);
    double2* esc = reinterpret_cast<double2*>(h.data() + o_esc);
    for (int e = 0; e <= nu; e++) {
        double gam = (-((double)e - 0.5 - (nu - 1) / 2.0) - off_a) * (double)da;
        esc[e] = make_double2(std::sin(gam), std::cos(gam));
    }
    for (int u = 0; u < nu; u++) {
        double a = (-((double)u - (nu - 1) / 2.0) - off_a) * (double)da;
        cell[u] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    if (std::fabs(nu * (double)da / 2.0) >= M_PI / 4)
        return set_error(RN_ERR_ARG, "fan geometry: fan half-angle must be below 45 degrees");
    int nxv = 0;
    for (int v = 0; v < nview; v++) {
        double th = (double)host_deg[v];
        double c = std::cos(th), s = std::sin(th);
        const float degf = host_deg[v];
        int xc = std::fabs(std::cos(degf)) > std::fabs(std::sin(degf)) ? 1 : 0;
        double sx = dso * s / dx + nx / 2.0;
        double sy = -dso * c / dy + ny / 2.0;
        auto slope = [&](int e) {
            double sn = esc[e].x * c - esc[e].y * s;
            double cn = esc[e].y * c + esc[e].x * s;
            return xc ? (sn * dy) / (cn * dx) : (cn * dx) / (sn * dy);
        };
        ViewGeo& q = vg[v];
        q.xcls = xc;
        q.par = xc ? sx : sy;
        q.perp = xc ? sy : sx;
        q.cosd = (float)c;
        q.sind = (float)s;
        double kap = xc ? (double)dx / dy : (double)dy / dx;
        q.kappa = (float)kap;
        double tB = xc ? -1.0 / da : 1.0 / da;
        q.tB = (float)tB;
        q.tA = (float)((double)(nu / 2) - tB * std::atan(kap * slope(nu / 2)));
        double r0 = slope(0), r1 = slope(nu);
        q.rmin = (float)std::min(r0, r1);
        q.rmax = (float)std::max(r0, r1);
        int nl = xc ? ny : nx;
        q.sigma = (float)((r1 > r0 ? 1.0 : -1.0) * ((nl / 2.0 - q.perp) > 0 ? 1.0 : -1.0));
        q.pad[0] = q.pad[1] = q.pad[2] = 0;
        if (std::fabs(q.perp - nl / 2.0) <= nl / 2.0 + 1.0)
            return set_error(RN_ERR_ARG, "fan geometry: source inside the image footprint");
        vcs[v] = make_double2(c, s);
        vx[v] = xc;
        nxv += xc;
    }
    {
        int a = 0, b = nxv;
        for (int v = 0; v < nview; v++) perm[vx[v] ? a++ : b++] = v;
    }
    int nwork = 0;
    for (int k = 0; k < nxv; k += VT) work[nwork++] = make_int4(0, 1, k, std::min(VT, nxv - k));
    for (int k = 0; k < nview - nxv; k += VT) work[nwork++] = make_int4(0, 0, nxv + k, std::min(VT, nview - nxv - k));
    *reinterpret_cast<GeoSet*>(h.data() + o_set) = GeoSet{0, nview, nxv};
    FpSlice* fs = reinterpret_cast<FpSlice*>(h.data() + o_fp);
    memset(fs, 0, sizeof(FpSlice));
    fs->img_w[0] = 1.f;
    fs->su = nview;
    fs->sview = 1;
    // o_err stays 0: the error word starts cleared on every call

    unsigned char* base = nullptr;
    RN_TRY(noalloc_scratch(&base));
    RN_CUDA_TRY(cudaMemcpyAsync(base, h.data(), host_bytes, cudaMemcpyHostToDevice, st));
    double* edges = reinterpret_cast<double*>(base + o_edges);
    long long ne = (long long)nview * (nu + 1);
    edge_slope_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(
        edges, reinterpret_cast<const double2*>(base + o_vcs), reinterpret_cast<const int*>(base + o_vx),
        reinterpret_cast<const double2*>(base + o_esc), nview, nu, dx, dy);
    RN_CUDA_TRY(cudaGetLastError());
    float2* hl = reinterpret_cast<float2*>(base + o_hl);
    float* la = reinterpret_cast<float*>(base + o_la);
    const FpSlice* dfs = reinterpret_cast<const FpSlice*>(base + o_fp);
    fan_lines_kernel<<<(unsigned)(((long long)(nx + ny) * 32 + 255) / 256), 256, 0, st>>>(d_img, dfs, 0, 1, d, hl,
                                                                                          la, slot, 0);
    RN_CUDA_TRY(cudaGetLastError());
    RN_TRY(fan_kernel_attributes());
    FpParams fp;
    fp.views = reinterpret_cast<const ViewGeo*>(base + o_views);
    fp.edges = edges;
    fp.cell = reinterpret_cast<const float2*>(base + o_cell);
    fp.perm = reinterpret_cast<const int*>(base + o_perm);
    fp.sets = reinterpret_cast<const GeoSet*>(base + o_set);
    fp.fps = dfs;
    fp.work = reinterpret_cast<const int4*>(base + o_work);
    fp.hl = hl;
    fp.la = la;
    fp.slot_elems = slot;
    fp.slot_base = 0;
    fp.prj = d_prj;
    fp.err = reinterpret_cast<int*>(base + o_err);
    fp.d = d;
    fp.R = R;
    fp.vt = VT;
    fp.spin = kSpinLimit;
    fan_fp_kernel<false><<<nwork, FpCfg<false>::threads, smem, st>>>(fp);
    RN_CUDA_TRY(cudaGetLastError());
    int herr = 0;
    RN_CUDA_TRY(cudaMemcpyAsync(&herr, base + o_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    RN_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr != 0) return set_error(RN_ERR_TIMEOUT, "a device-side wait exceeded its spin limit");
    return RN_OK;
}
