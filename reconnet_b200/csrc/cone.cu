// Siddon cone-beam projector pair with arbitrary per-view geometry
// (SiddonCone.cu): ray (iu, iview, iv) runs from src[iview] to
// detCenter + u detU + v detV, u = (iu - off_u - (nu-1)/2) du,
// v = (iv - off_v - (nv-1)/2) dv, and each voxel of the grid centred at
// (cx, cy, cz) receives the length (mm) of the ray inside it.
//
// Voxel coordinates put the origin at the corner of voxel 0
// (PhysicsToImg, Siddon.cu:14-21).  Every view has a main axis m (the axis
// along which its central ray advances most, in voxels) and lateral axes a,
// b; a ray's lateral positions are affine in its main coordinate:
// a(k) = S_a + (k - S_m) r_a, r_a = D_a / D_m.
//
// Forward projection: one thread per ray steps through the unit slabs
// [k, k + 1] along m.  Inside a slab the ray crosses at most ceil|r_a| +
// ceil|r_b| lateral grid lines (the host rejects views with |r| > 4), so the
// slab splits into a few pieces of known voxel; each piece adds
// (its share of the slab) x seg x the voxel value, seg being the ray's length
// per slab.  Lateral positions are 64-bit fixed point (32 fractional bits,
// stepped by an integer add), so the split points are exact to ~1e-7 slabs
// however far the source is.  With every slope at most 1 the block's voxels
// are staged in shared memory chunk by chunk (cone_fp_staged_kernel);
// otherwise the pieces are read from global memory (cone_fp_kernel).
//
// Backprojection, the exact transpose as a gather (the reference scatters
// with atomics): per voxel and view, the candidate rays are the detector
// cells inside the voxel's shadow (its 8 corners projected through the
// source, bounded by interval arithmetic); each candidate adds seg x its
// sinogram value x the part of the voxel's main-axis extent over which it
// lies inside the voxel laterally.  The ray's lateral offsets from the voxel
// at the voxel's low main-axis face, x_a = (S_a - a_v) + (m_v - S_m) r_a, come
// from hi / lo float parts with exact products, as in the fan Siddon
// backprojection, to ~1e-7 voxels (cone_bp_kernel).  When every view is
// separable the same way (detector perpendicular to the main axis, u and v
// along the two lateral axes: tomosynthesis) cone_bp_sep_kernel runs
// instead, on projections pre-multiplied by seg (cone_prj_seg_kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "rn_internal.h"

namespace rn {

struct ConeView {
    double S[3];              // source, voxel coordinates
    double C[3];              // end point of ray (iu, iv) = (0, 0), voxel coordinates
    double Eu[3], Ev[3];      // end-point step per detector index along u / v
    float Sh[3], Sl[3];       // source as hi / lo floats
    float au[4], av[4], ad[4];   // shadow: iu = (au . P + au[3]) / (ad . P + ad[3]), iv likewise
    float ulo, uhi, vlo, vhi, dlo, dhi;   // sums of min(0, a_k) / max(0, a_k) over the three axes
    // separable views (affine = 1 or 2): every ray advances by the same Dm0
    // along m, and r_a = rho[0] + iu rho[1] + iv rho[2], r_b = rho[3] +
    // iu rho[4] + iv rho[5] with rho[2] = rho[4] = 0 (affine = 1: a follows
    // iu, b follows iv) or rho[1] = rho[5] = 0 (affine = 2)
    double rho[6];
    double Dm0;
    int m, a, b, affine;
};

struct ConeDims {
    int n[3];
    float d[3];
    long long st[3];          // image strides (elements) along x, y, z
    int nc, nu, nv, nview, nb;
    long long img_b, prj_b;   // batch strides
};

// Per ray (view, iv, iu) geometry for the backprojection:
// {r_a hi, r_a lo, r_b hi, r_b lo}, {1 / r_a, 1 / r_b, seg, E_m}.
__global__ void cone_ray_kernel(float4* __restrict__ rays, const ConeView* __restrict__ views, ConeDims cd) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)cd.nview * cd.nv * cd.nu;
    if (i >= n) return;
    const int iu = (int)(i % cd.nu);
    const int iv = (int)((i / cd.nu) % cd.nv);
    const int view = (int)(i / ((long long)cd.nu * cd.nv));
    const ConeView& V = views[view];
    double D[3];
#pragma unroll
    for (int k = 0; k < 3; k++) D[k] = V.C[k] + iu * V.Eu[k] + iv * V.Ev[k] - V.S[k];
    const double Dm = D[V.m], ra = D[V.a] / Dm, rb = D[V.b] / Dm;
    const double dm = cd.d[V.m], da = cd.d[V.a], db = cd.d[V.b];
    const double seg = sqrt(dm * dm + ra * ra * da * da + rb * rb * db * db);
    const float rah = (float)ra, rbh = (float)rb;
    rays[2 * i] = make_float4(rah, (float)(ra - rah), rbh, (float)(rb - rbh));
    rays[2 * i + 1] = make_float4(fabs(ra) > 1e-30 ? (float)(1.0 / ra) : 1e30f,
                                  fabs(rb) > 1e-30 ? (float)(1.0 / rb) : 1e30f, (float)seg,
                                  (float)(V.S[V.m] + Dm));
}

__device__ __forceinline__ long long to_fixed(double v) { return llrint(v * 4294967296.0); }

// Fractional part of a fixed-point position as a float in [0, 1) (its top 23
// bits: exact to 1.2e-7).
__device__ __forceinline__ float fixed_frac(long long p) {
    return __uint_as_float(0x3f800000u | ((unsigned)p >> 9)) - 1.0f;
}

// Per-ray stepping state: lateral positions at the start of slab k0 and
// their step per slab (fixed point, 32 fractional bits), slope signs and
// |1 / r|, the ray's length per slab, the segment's own ends along m relative
// to slab k0, and the slabs [k0, k0 + ns).
struct RayStep {
    long long A, RA, B, RB;
    float seg, ira, irb, slo, shi;
    int k0, ns;
    bool pa, pb;
};

__device__ __forceinline__ RayStep cone_ray_step(const ConeView& V, int iu, int iv, const ConeDims& cd, int m, int a,
                                                 int b) {
    RayStep R;
    R.ns = 0;
    double D[3], S[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        S[k] = V.S[k];
        D[k] = V.C[k] + iu * V.Eu[k] + iv * V.Ev[k] - S[k];
    }
    // parameter range of the segment inside the grid
    double t0 = 0.0, t1 = 1.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (fabs(D[k]) > 1e-12) {
            const double ta = -S[k] / D[k], tb = (cd.n[k] - S[k]) / D[k];
            t0 = fmax(t0, fmin(ta, tb));
            t1 = fmin(t1, fmax(ta, tb));
        } else if (S[k] < 0.0 || S[k] > cd.n[k]) {
            t1 = -1.0;
        }
    }
    if (t1 <= t0) return R;
    const double Dm = m == 0 ? D[0] : m == 1 ? D[1] : D[2];
    const double Da = a == 0 ? D[0] : a == 1 ? D[1] : D[2];
    const double Db = b == 0 ? D[0] : b == 1 ? D[1] : D[2];
    const double Sm = m == 0 ? S[0] : m == 1 ? S[1] : S[2];
    const double Sa = a == 0 ? S[0] : a == 1 ? S[1] : S[2];
    const double Sb = b == 0 ? S[0] : b == 1 ? S[1] : S[2];
    const int nm = m == 0 ? cd.n[0] : m == 1 ? cd.n[1] : cd.n[2];
    const double ra = Da / Dm, rb = Db / Dm;
    const double mlo = Sm + fmin(t0 * Dm, t1 * Dm), mhi = Sm + fmax(t0 * Dm, t1 * Dm);
    const int k0 = max(0, (int)floor(mlo)), k1 = min(nm - 1, (int)ceil(mhi) - 1);
    if (k1 < k0) return R;
    const double dm = m == 0 ? cd.d[0] : m == 1 ? cd.d[1] : cd.d[2];
    const double da = a == 0 ? cd.d[0] : a == 1 ? cd.d[1] : cd.d[2];
    const double db = b == 0 ? cd.d[0] : b == 1 ? cd.d[1] : cd.d[2];
    R.seg = (float)sqrt(dm * dm + ra * ra * da * da + rb * rb * db * db);
    // the segment's own ends along m (the grid faces are handled by the
    // voxel bounds), relative to slab k0
    R.slo = (float)fmax(fmin(Sm, Sm + Dm) - k0, -1.0);
    R.shi = (float)fmin(fmax(Sm, Sm + Dm) - k0, (double)(k1 - k0) + 2.0);
    R.A = to_fixed(Sa + (k0 - Sm) * ra);
    R.B = to_fixed(Sb + (k0 - Sm) * rb);
    R.RA = to_fixed(ra);
    R.RB = to_fixed(rb);
    R.pa = ra > 0;
    R.pb = rb > 0;
    R.ira = fabs(ra) > 1e-30 ? (float)(1.0 / fabs(ra)) : 1e30f;
    R.irb = fabs(rb) > 1e-30 ? (float)(1.0 / fabs(rb)) : 1e30f;
    R.k0 = k0;
    R.ns = k1 - k0 + 1;
    return R;
}

// The voxel values along one slab of a ray times the share of the slab
// spent in each voxel, for slab entry positions A, B (fixed point), steps
// RA, RB, and the segment clip [tlo, thi] in slab units; sl points at the
// slab's voxel (0, 0) and sta, stb are the lateral strides (32-bit: the plan
// keeps a batch below 2^31 elements).  kUnit: |r| <= 1, so at most one
// crossing per lateral axis and three pieces, without branches; otherwise
// the pieces are walked.
template <bool kUnit>
__device__ __forceinline__ float slab_sum(long long A, long long RA, long long B, long long RB, bool pa, bool pb,
                                          float ira, float irb, float tlo, float thi, const float* sl, int sta,
                                          int stb, int na, int nb) {
    const long long An = A + RA, Bn = B + RB;
    const int ca0 = (int)(A >> 32), cb0 = (int)(B >> 32);
    const int ca1 = (int)(An >> 32), cb1 = (int)(Bn >> 32);
    if (kUnit) {
        const float fa = fixed_frac(A), fb = fixed_frac(B);
        const float ta = ca1 != ca0 ? (pa ? 1.f - fa : fa) * ira : 2.f;
        const float tb = cb1 != cb0 ? (pb ? 1.f - fb : fb) * irb : 2.f;
        const float t1 = fminf(ta, tb), t2 = fmaxf(ta, tb);
        const bool afirst = ta < tb;
        const int cam = afirst ? ca1 : ca0, cbm = afirst ? cb0 : cb1;
        const float l0 = fminf(t1, thi) - tlo, lm = fminf(t2, thi) - fmaxf(t1, tlo), l1 = thi - fmaxf(t2, tlo);
        float s = 0.f;
        if (l0 > 0.f && (unsigned)ca0 < (unsigned)na && (unsigned)cb0 < (unsigned)nb)
            s = l0 * __ldg(sl + (ca0 * sta + cb0 * stb));
        if (lm > 0.f && (unsigned)cam < (unsigned)na && (unsigned)cbm < (unsigned)nb)
            s = fmaf(lm, __ldg(sl + (cam * sta + cbm * stb)), s);
        if (l1 > 0.f && (unsigned)ca1 < (unsigned)na && (unsigned)cb1 < (unsigned)nb)
            s = fmaf(l1, __ldg(sl + (ca1 * sta + cb1 * stb)), s);
        return s;
    } else {
        int ca = ca0, cb = cb0;
        int nxa = abs(ca1 - ca0), nxb = abs(cb1 - cb0);
        float ta = nxa ? (pa ? 1.f - fixed_frac(A) : fixed_frac(A)) * ira : 2.f;
        float tb = nxb ? (pb ? 1.f - fixed_frac(B) : fixed_frac(B)) * irb : 2.f;
        float tcur = 0.f, s = 0.f;
        for (;;) {
            const float tn = fminf(fminf(ta, tb), thi);
            const float len = tn - fmaxf(tcur, tlo);
            if (len > 0.f && (unsigned)ca < (unsigned)na && (unsigned)cb < (unsigned)nb)
                s = fmaf(len, __ldg(sl + (ca * sta + cb * stb)), s);
            if (tn >= thi) break;
            tcur = tn;
            if (ta <= tb) {
                ca += pa ? 1 : -1;
                ta = (--nxa > 0) ? ta + ira : 2.f;
            } else {
                cb += pb ? 1 : -1;
                tb = (--nxb > 0) ? tb + irb : 2.f;
            }
        }
        return s;
    }
}

// Forward projection, one thread per ray: a block holds 32 rays along iu x
// 8 along iv, or 32 along iv x 8 along iu when `lanes_v` (the detector's v
// running along z, the image's contiguous axis, so that a warp's loads of
// one slab lie close together).
template <bool kUnit>
__global__ void __launch_bounds__(256) cone_fp_kernel(float* __restrict__ prj, const float* __restrict__ img,
                                                       const ConeView* __restrict__ views, ConeDims cd,
                                                       int lanes_v) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int iu = lanes_v ? blockIdx.x * 8 + warp : blockIdx.x * 32 + lane;
    const int iv = lanes_v ? blockIdx.y * 32 + lane : blockIdx.y * 8 + warp;
    if (iu >= cd.nu || iv >= cd.nv) return;
    int zi = blockIdx.z;
    const int c = zi % cd.nc;
    zi /= cd.nc;
    const int view = zi % cd.nview;
    const int bt = zi / cd.nview;
    const ConeView& V = views[view];
    const int m = V.m, a = V.a, b = V.b;
    const RayStep R = cone_ray_step(V, iu, iv, cd, m, a, b);
    float acc = 0.f;
    if (R.ns > 0) {
        const int sta = (int)(a == 0 ? cd.st[0] : a == 1 ? cd.st[1] : cd.st[2]);
        const int stb = (int)(b == 0 ? cd.st[0] : b == 1 ? cd.st[1] : cd.st[2]);
        const int stm = (int)(m == 0 ? cd.st[0] : m == 1 ? cd.st[1] : cd.st[2]);
        const int na = a == 0 ? cd.n[0] : a == 1 ? cd.n[1] : cd.n[2];
        const int nb = b == 0 ? cd.n[0] : b == 1 ? cd.n[1] : cd.n[2];
        const float* sl = img + bt * cd.img_b + c + R.k0 * stm;
        long long A = R.A, B = R.B;
        for (int j = 0; j < R.ns; j++) {
            acc += slab_sum<kUnit>(A, R.RA, B, R.RB, R.pa, R.pb, R.ira, R.irb, fmaxf(0.f, R.slo - (float)j),
                                   fminf(1.f, R.shi - (float)j), sl, sta, stb, na, nb);
            A += R.RA;
            B += R.RB;
            sl += stm;
        }
        acc *= R.seg;
    }
    prj[bt * cd.prj_b + (((long long)iu * cd.nview + view) * cd.nv + iv) * cd.nc + c] = acc;
}

// Forward projection with the voxels staged in shared memory (|r| <= 1).
// The block's rays advance through chunks of kFpZ slabs along m.  For each
// chunk the block reduces the lateral voxel index range its rays touch (a
// ray's positions are monotone along m, so its range is spanned by its
// entry into the chunk and its exit), copies that brick into shared memory
// as one plane per slab (voxels outside the grid as 0), and the rays take
// their pieces from there with the arithmetic of slab_sum<true>, so the sums
// are the same to the bit.  A warp's gathers then hit shared memory instead
// of ~15 sectors of L1 per load.  A chunk whose brick is larger than a plane
// falls back to loads from global memory.  `vec`: the main axis is the
// image's contiguous axis and every group of 4 voxels along it starts
// 16-byte aligned, so the copy loads float4.
constexpr int kFpZ = 16;         // slabs per chunk
constexpr int kFpPlane = 640;    // floats per staged slab plane

// Fractional part of a fixed-point position plus 1, in [1, 2).
__device__ __forceinline__ float fixed_frac1(long long p) { return __uint_as_float(0x3f800000u | ((unsigned)p >> 9)); }

// Slabs [0, n) of one ray through a staged chunk: A, B are the ray's
// fixed-point positions at its first slab and advance past the last; `pl` is
// the plane of the first slab; jf = that slab's index from the ray's first.
// kClip: some slab of the chunk holds an end of the segment (otherwise every
// slab is whole: tlo = 0, thi = 1).
template <bool kClip>
__device__ __forceinline__ void staged_run(float& acc, long long& A, long long& B, const RayStep& R, int n, float jf,
                                           const float* pl, int P, int Na, int alo, int blo) {
    const long long oa = (long long)alo << 32, ob = (long long)blo << 32;
    long long Ar = A - oa, Br = B - ob;
    // (pa ? 1 - f : f) * ira as one FMA on f + 1 (the same rounding)
    const float sA = R.pa ? -R.ira : R.ira, oA = R.pa ? 2.f * R.ira : -R.ira;
    const float sB = R.pb ? -R.irb : R.irb, oB = R.pb ? 2.f * R.irb : -R.irb;
    int ca = (int)(Ar >> 32), cb = (int)(Br >> 32);
    int i0 = cb * Na + ca;
    for (int j = 0; j < n; j++) {
        const float fa1 = fixed_frac1(Ar), fb1 = fixed_frac1(Br);
        Ar += R.RA;
        Br += R.RB;
        const int ca1 = (int)(Ar >> 32), cb1 = (int)(Br >> 32);
        const float ta = ca1 != ca ? fmaf(sA, fa1, oA) : 2.f;
        const float tb = cb1 != cb ? fmaf(sB, fb1, oB) : 2.f;
        const float t1 = fminf(ta, tb), t2 = fmaxf(ta, tb);
        const bool afirst = ta < tb;
        const int i1 = cb1 * Na + ca1;
        const int im = afirst ? cb * Na + ca1 : cb1 * Na + ca;
        float l0, lm, l1;
        if (kClip) {
            const float tlo = fmaxf(0.f, R.slo - jf), thi = fminf(1.f, R.shi - jf);
            l0 = fminf(t1, thi) - tlo;
            lm = fminf(t2, thi) - fmaxf(t1, tlo);
            l1 = thi - fmaxf(t2, tlo);
            jf += 1.f;
        } else {
            l0 = fminf(t1, 1.f);
            lm = fminf(t2, 1.f) - t1;
            l1 = 1.f - t2;
        }
        // branch-free (every index lies in the brick): a piece of length <= 0
        // adds exactly 0
        float s = fmaxf(l0, 0.f) * pl[i0];
        s = fmaf(fmaxf(lm, 0.f), pl[im], s);
        s = fmaf(fmaxf(l1, 0.f), pl[i1], s);
        acc += s;
        ca = ca1;
        cb = cb1;
        i0 = i1;
        pl += P;
    }
    A = Ar + oa;
    B = Br + ob;
}

__global__ void __launch_bounds__(256) cone_fp_staged_kernel(float* __restrict__ prj, const float* __restrict__ img,
                                                              const ConeView* __restrict__ views, ConeDims cd,
                                                              int lanes_v, int vec) {
    extern __shared__ float brick[];   // kFpZ planes of stride P
    __shared__ int4 s_part[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int iu = lanes_v ? blockIdx.x * 8 + warp : blockIdx.x * 32 + lane;
    const int iv = lanes_v ? blockIdx.y * 32 + lane : blockIdx.y * 8 + warp;
    const bool valid = iu < cd.nu && iv < cd.nv;
    int zi = blockIdx.z;
    const int c = zi % cd.nc;
    zi /= cd.nc;
    const int view = zi % cd.nview;
    const int bt = zi / cd.nview;
    const ConeView& V = views[view];
    const int m = V.m, a = V.a, b = V.b;
    RayStep R = cone_ray_step(V, min(iu, cd.nu - 1), min(iv, cd.nv - 1), cd, m, a, b);
    if (!valid) R.ns = 0;
    const int sta = (int)(a == 0 ? cd.st[0] : a == 1 ? cd.st[1] : cd.st[2]);
    const int stb = (int)(b == 0 ? cd.st[0] : b == 1 ? cd.st[1] : cd.st[2]);
    const int stm = (int)(m == 0 ? cd.st[0] : m == 1 ? cd.st[1] : cd.st[2]);
    const int na = a == 0 ? cd.n[0] : a == 1 ? cd.n[1] : cd.n[2];
    const int nb = b == 0 ? cd.n[0] : b == 1 ? cd.n[1] : cd.n[2];
    const int nm = m == 0 ? cd.n[0] : m == 1 ? cd.n[1] : cd.n[2];
    const bool vec4 = vec && m == 2;
    const float* vol = img + bt * cd.img_b + c;
    // the block's slabs
    int klo = R.ns > 0 ? R.k0 : INT_MAX, khi = R.ns > 0 ? R.k0 + R.ns : INT_MIN;
    klo = __reduce_min_sync(0xffffffffu, klo);
    khi = __reduce_max_sync(0xffffffffu, khi);
    if (lane == 0) s_part[warp] = make_int4(klo, khi, 0, 0);
    __syncthreads();
    {
        const int4 q = s_part[lane & 7];
        klo = __reduce_min_sync(0xffffffffu, q.x);
        khi = __reduce_max_sync(0xffffffffu, q.y);
    }
    __syncthreads();
    long long A = R.A, B = R.B;
    int kk = R.k0;                       // this ray's next slab
    const int kend = R.k0 + R.ns;
    float acc = 0.f;
    for (int K = klo >= khi ? khi : (klo / kFpZ) * kFpZ; K < khi; K += kFpZ) {
        const int js = max(K, kk), je = min(K + kFpZ, kend);
        const bool act = js < je;
        int alo = INT_MAX, ahi = INT_MIN, blo = INT_MAX, bhi = INT_MIN;
        if (act) {
            const long long Ae = A + (long long)(je - js) * R.RA, Be = B + (long long)(je - js) * R.RB;
            const int a0 = (int)(A >> 32), a1 = (int)(Ae >> 32), b0 = (int)(B >> 32), b1 = (int)(Be >> 32);
            alo = min(a0, a1);
            ahi = max(a0, a1);
            blo = min(b0, b1);
            bhi = max(b0, b1);
        }
        alo = __reduce_min_sync(0xffffffffu, alo);
        ahi = __reduce_max_sync(0xffffffffu, ahi);
        blo = __reduce_min_sync(0xffffffffu, blo);
        bhi = __reduce_max_sync(0xffffffffu, bhi);
        if (lane == 0) s_part[warp] = make_int4(alo, ahi, blo, bhi);
        __syncthreads();
        {
            const int4 q = s_part[lane & 7];
            alo = __reduce_min_sync(0xffffffffu, q.x);
            ahi = __reduce_max_sync(0xffffffffu, q.y);
            blo = __reduce_min_sync(0xffffffffu, q.z);
            bhi = __reduce_max_sync(0xffffffffu, q.w);
        }
        // brick planes of stride P = 2 (mod 32): the copy's stores are free
        // of bank conflicts
        const long long Na_l = (long long)ahi - alo + 1, Nb_l = (long long)bhi - blo + 1;
        const bool any = ahi >= alo && bhi >= blo;
        const long long cols = any ? Na_l * Nb_l : 0;
        const long long P_l = cols <= 2 ? 2 : ((cols - 2 + 31) / 32) * 32 + 2;
        const bool staged = any && P_l <= kFpPlane;
        const float jf = (float)(js - R.k0);
        if (staged) {
            const int Na = (int)Na_l, Nb = (int)Nb_l, P = (int)P_l;
            if (vec4 && K + kFpZ <= nm) {
                // 4 lanes per column, one float4 each
                const int q = lane & 3;
                for (int ib = warp; ib < Nb; ib += 8) {
                    const int bb = blo + ib;
                    const bool inb = (unsigned)bb < (unsigned)nb;
                    for (int ia = lane >> 2; ia < Na; ia += 8) {
                        const int aa = alo + ia;
                        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (inb && (unsigned)aa < (unsigned)na)
                            v = __ldg(reinterpret_cast<const float4*>(vol + (aa * sta + bb * stb + K + 4 * q)));
                        float* d = brick + 4 * q * P + ib * Na + ia;
                        d[0] = v.x;
                        d[P] = v.y;
                        d[2 * P] = v.z;
                        d[3 * P] = v.w;
                    }
                }
            } else {
                // 16 lanes per column, one slab each
                const int zc = lane & 15, k = K + zc;
                for (int ib = warp; ib < Nb; ib += 8) {
                    const int bb = blo + ib;
                    const bool inb = (unsigned)bb < (unsigned)nb && k < nm;
                    for (int ia = lane >> 4; ia < Na; ia += 2) {
                        const int aa = alo + ia;
                        float v = 0.f;
                        if (inb && (unsigned)aa < (unsigned)na) v = __ldg(vol + (aa * sta + bb * stb + k * stm));
                        brick[zc * P + ib * Na + ia] = v;
                    }
                }
            }
            __syncthreads();
            if (act) {
                const float* pl = brick + (js - K) * P;
                if (R.slo <= jf && R.shi >= jf + (float)(je - js))
                    staged_run<false>(acc, A, B, R, je - js, jf, pl, P, Na, alo, blo);
                else
                    staged_run<true>(acc, A, B, R, je - js, jf, pl, P, Na, alo, blo);
            }
        } else {
            __syncthreads();   // every lane has read s_part before the next chunk writes it
            if (act) {
                const float* sl = vol + js * stm;
                float jg = jf;
                for (int k = js; k < je; k++) {
                    acc += slab_sum<true>(A, R.RA, B, R.RB, R.pa, R.pb, R.ira, R.irb, fmaxf(0.f, R.slo - jg),
                                          fminf(1.f, R.shi - jg), sl, sta, stb, na, nb);
                    A += R.RA;
                    B += R.RB;
                    sl += stm;
                    jg += 1.f;
                }
            }
        }
        if (act) kk = je;
    }
    if (!valid) return;
    if (R.ns > 0) acc *= R.seg;
    prj[bt * cd.prj_b + (((long long)iu * cd.nview + view) * cd.nv + iv) * cd.nc + c] = acc;
}

__device__ __forceinline__ void two_sum_f(float a, float b, float& s, float& e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Separable views: the lateral offsets of ray (iu, iv) from voxel (x, y, z)
// at its low main-axis face are x_a = A + M r_a(i) and x_b = B + M r_b(j),
// with (i, j) = (iu, iv) (affine = 1) or (iv, iu) (affine = 2), A = S_a -
// a_v, B = S_b - b_v, M = m_v - S_m.  The cells whose ray can meet the voxel
// along a satisfy x_a in (-max(r_a, 0), 1 - min(r_a, 0)): an index range
// (widened by 0.02), found in FP64; likewise along b.  Each pair (i, j) then
// adds seg x prj x |[0, 1] n T_a(i) n T_b(j)|, T being the parameter
// interval over which the ray lies inside the voxel along that axis.
// Returns false (adding nothing) when a range holds more than kSepMax cells.
constexpr int kSepMax = 6;

__device__ __forceinline__ bool bp_separable(float& acc, const ConeView& V, int x, int y, int z, const ConeDims& cd,
                                             const float* pb, int view) {
    const int m = V.m, a = V.a, b = V.b;
    const int pm = m == 0 ? x : m == 1 ? y : z, pa = a == 0 ? x : a == 1 ? y : z, pbv = b == 0 ? x : b == 1 ? y : z;
    const double Sm = m == 0 ? V.S[0] : m == 1 ? V.S[1] : V.S[2];
    const double Sa = a == 0 ? V.S[0] : a == 1 ? V.S[1] : V.S[2];
    const double Sb = b == 0 ? V.S[0] : b == 1 ? V.S[1] : V.S[2];
    const double M = (double)pm - Sm, A = Sa - pa, B = Sb - pbv;
    const bool swap = V.affine == 2;
    // r_a = ra0 + i ra1, r_b = rb0 + j rb1
    const double ra0 = V.rho[0], ra1 = swap ? V.rho[2] : V.rho[1];
    const double rb0 = V.rho[3], rb1 = swap ? V.rho[4] : V.rho[5];
    const int ni = swap ? cd.nv : cd.nu, nj = swap ? cd.nu : cd.nv;
    // x(i) = X0 + i G with X0 = A + M r0 and G = M r1 (FP64); the index
    // range where x(i) in (lo, hi) needs no more than FP32 (it is widened by
    // 0.02), with r ~ -A / M, the slope of the ray through the voxel corner
    const double XA0 = A + M * ra0, XB0 = B + M * rb0, GA = M * ra1, GB = M * rb1;
    const float rs_a = (float)(-A) / (float)M, rs_b = (float)(-B) / (float)M;
    auto range = [&](double X0, double G, float rs, int n, int& i0, int& i1) {
        const float lo = -fmaxf(rs, 0.f) - 0.02f, hi = 1.f - fminf(rs, 0.f) + 0.02f;
        const float x0 = (float)X0, ig = __fdividef(1.f, (float)G);
        const float q0 = (lo - x0) * ig, q1 = (hi - x0) * ig;
        i0 = max(0, (int)ceilf(fmaxf(fminf(q0, q1), -1e9f)));
        i1 = min(n - 1, (int)floorf(fminf(fmaxf(q0, q1), 1e9f)));
    };
    int i0, i1, j0, j1;
    range(XA0, GA, rs_a, ni, i0, i1);
    range(XB0, GB, rs_b, nj, j0, j1);
    if (i1 < i0 || j1 < j0) return true;
    if (i1 - i0 >= kSepMax || j1 - j0 >= kSepMax) return false;
    // the first candidate's offsets in FP64, then steps in FP32
    const float xa0 = (float)fma((double)i0, GA, XA0), xb0 = (float)fma((double)j0, GB, XB0);
    const float ga = (float)GA, gb = (float)GB;
    const float ra1f = (float)ra1, rb1f = (float)rb1;
    const float rai_f = (float)(ra0 + i0 * ra1), rbj_f = (float)(rb0 + j0 * rb1);
    // the segment's ends along m, relative to the voxel's low face
    const float e0 = (float)(-M), e1 = (float)(-M + V.Dm0);
    const float clo = fmaxf(0.f, fminf(e0, e1)), chi = fminf(1.f, fmaxf(e0, e1));
    const float dm = m == 0 ? cd.d[0] : m == 1 ? cd.d[1] : cd.d[2];
    const float da = a == 0 ? cd.d[0] : a == 1 ? cd.d[1] : cd.d[2];
    const float db = b == 0 ? cd.d[0] : b == 1 ? cd.d[1] : cd.d[2];
    const float dm2 = dm * dm, da2 = da * da, db2 = db * db;
    const int su = cd.nview * cd.nv * cd.nc, sv = cd.nc;
    const float* pview = pb + (long long)view * cd.nv * cd.nc;
    for (int j = j0; j <= j1; j++) {
        const float kj = (float)(j - j0);
        const float xb = fmaf(kj, gb, xb0), rb = fmaf(kj, rb1f, rbj_f);
        const float ib = fabsf(rb) > 1e-30f ? __fdividef(1.f, rb) : 1e30f;
        const float tb0 = -xb * ib, tb1 = (1.f - xb) * ib;
        const float lb = fmaxf(clo, fminf(tb0, tb1)), hb = fminf(chi, fmaxf(tb0, tb1));
        if (!(hb > lb)) continue;
        const float qb = fmaf(rb * rb, db2, dm2);
        for (int i = i0; i <= i1; i++) {
            const float ki = (float)(i - i0);
            const float xa = fmaf(ki, ga, xa0), ra = fmaf(ki, ra1f, rai_f);
            const float ia = fabsf(ra) > 1e-30f ? __fdividef(1.f, ra) : 1e30f;
            const float ta0 = -xa * ia, ta1 = (1.f - xa) * ia;
            const float tl = fmaxf(lb, fminf(ta0, ta1)), th = fminf(hb, fmaxf(ta0, ta1));
            if (th > tl) {
                const float q = fmaf(ra * ra, da2, qb);
                const int iu = swap ? j : i, iv = swap ? i : j;
                acc = fmaf((th - tl) * (q * rsqrtf(q)), __ldg(pview + ((long long)iu * su + iv * sv)), acc);
            }
        }
    }
    return true;
}

// Backprojection for plans whose views are all separable the same way.  Call
// U the lateral axis that follows the detector's u and V the one that follows
// v; the slopes are r_U(iu) = rU0 + iu rU1 and r_V(iv) = rV0 + iv rV1.  A
// warp holds two neighbouring voxels along U (pu, pu + 1) for each of 32
// voxels along V (lanes), at one main-axis index pm.  For a view, the rays
// that can meet those voxels along U and their parameter intervals inside
// [pu, pu + 1] and [pu + 1, pu + 2] are the same for every lane: lane k
// computes candidate k's two intervals, clipped to the slab [0, 1] and to the
// segment's ends along m, into shared memory.  Each lane then walks its own V
// candidates and, for each, the warp's U candidates: pair (iu, iv) adds
// prjw x |T_U(iu) n T_V(iv)| to each of its two voxels, with one load for
// both; prjw = seg x prj comes from cone_prj_seg_kernel.  This is the sum of
// bp_separable with every interval and segment length computed once instead
// of once per pair.
constexpr int kSepWarps = 8;

// prjw = prj x seg for a separable plan: seg = sqrt(dM^2 + (r_U dU)^2 +
// (r_V dV)^2), the length per unit slab of ray (iu, iv), so that the
// backprojector's pairs need no square root.  Grid: x over the (iv, c) run,
// y = view, z = iu; batches in a loop.
__global__ void cone_prj_seg_kernel(float* __restrict__ prjw, const float* __restrict__ prj,
                                    const ConeView* __restrict__ views, ConeDims cd) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cd.nv * cd.nc) return;
    const int view = blockIdx.y, iu = blockIdx.z;
    const int iv = j / cd.nc;
    const ConeView& V = views[view];
    const bool a_is_u = views[0].affine == 1;
    const int m = views[0].m;
    const int ax_u = a_is_u ? views[0].a : views[0].b, ax_v = a_is_u ? views[0].b : views[0].a;
    const float dU = ax_u == 0 ? cd.d[0] : ax_u == 1 ? cd.d[1] : cd.d[2];
    const float dV = ax_v == 0 ? cd.d[0] : ax_v == 1 ? cd.d[1] : cd.d[2];
    const float dM = m == 0 ? cd.d[0] : m == 1 ? cd.d[1] : cd.d[2];
    const double rU0 = a_is_u ? V.rho[0] : V.rho[3], rU1 = a_is_u ? V.rho[1] : V.rho[4];
    const double rV0 = a_is_u ? V.rho[3] : V.rho[0], rV1 = a_is_u ? V.rho[5] : V.rho[2];
    const float ru = (float)fma((double)iu, rU1, rU0), rv = (float)fma((double)iv, rV1, rV0);
    const float seg = sqrtf(fmaf(ru * ru, dU * dU, fmaf(rv * rv, dV * dV, dM * dM)));
    const long long e = ((long long)iu * cd.nview + view) * cd.nv * cd.nc + j;
    for (int b = 0; b < cd.nb; b++) prjw[b * cd.prj_b + e] = prj[b * cd.prj_b + e] * seg;
}

__device__ __forceinline__ void sep_range(double X0, double G, float lo, float hi, int n, int& i0, int& i1) {
    const float x0 = (float)X0, ig = __fdividef(1.f, (float)G);
    const float q0 = (lo - x0) * ig, q1 = (hi - x0) * ig;
    i0 = max(0, (int)ceilf(fmaxf(fminf(q0, q1), -1e9f)));
    i1 = min(n - 1, (int)floorf(fminf(fmaxf(q0, q1), 1e9f)));
}

__global__ void __launch_bounds__(256) cone_bp_sep_kernel(float* __restrict__ img, const float* __restrict__ prj,
                                                           const ConeView* __restrict__ views, ConeDims cd,
                                                           int accumulate) {
    __shared__ float4 s_t[kSepWarps][32];   // {T lo, T hi} for voxel pu, then for pu + 1
    __shared__ int s_i[kSepWarps][32];      // iu
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = views[0].m;
    const bool a_is_u = views[0].affine == 1;
    const int ax_u = a_is_u ? views[0].a : views[0].b, ax_v = a_is_u ? views[0].b : views[0].a;
    const int nU = ax_u == 0 ? cd.n[0] : ax_u == 1 ? cd.n[1] : cd.n[2];
    const int nV = ax_v == 0 ? cd.n[0] : ax_v == 1 ? cd.n[1] : cd.n[2];
    const int nM = m == 0 ? cd.n[0] : m == 1 ? cd.n[1] : cd.n[2];
    const int nU2 = (nU + 1) / 2;
    const long long w = (long long)blockIdx.x * kSepWarps + warp;
    if (w >= (long long)nU2 * nM) return;   // the whole warp
    const int pu = 2 * (int)(w % nU2), pm = (int)(w / nU2);
    const int pv = blockIdx.y * 32 + lane;
    const bool live = pv < nV, live1 = live && pu + 1 < nU;
    const int bc = blockIdx.z;
    const int c = bc % cd.nc, bt = bc / cd.nc;
    const long long su = (long long)cd.nview * cd.nv * cd.nc;
    const int sv = cd.nc;
    const float* pb = prj + bt * cd.prj_b + c;
    float acc0 = 0.f, acc1 = 0.f;
    for (int view = 0; view < cd.nview; view++) {
        const ConeView& V = views[view];
        const double M = (double)pm - V.S[m];
        // the segment's ends along m, relative to the voxel's low face
        const float e0 = (float)(-M), e1 = (float)(-M + V.Dm0);
        const float clo = fmaxf(0.f, fminf(e0, e1)), chi = fminf(1.f, fmaxf(e0, e1));
        if (!(chi > clo)) continue;
        const double rU0 = a_is_u ? V.rho[0] : V.rho[3], rU1 = a_is_u ? V.rho[1] : V.rho[4];
        const double rV0 = a_is_u ? V.rho[3] : V.rho[0], rV1 = a_is_u ? V.rho[5] : V.rho[2];
        const double AU = V.S[ax_u] - (double)pu, AV = V.S[ax_v] - (double)pv;
        const float iM = __fdividef(1.f, (float)M);
        const double XU0 = AU + M * rU0, GU = M * rU1, XV0 = AV + M * rV0, GV = M * rV1;
        // candidates: x in (-max(r, 0), 1 - min(r, 0)) from voxel pu (and
        // x - 1 likewise from pu + 1), with r ~ the slope through the voxel
        // corner, widened by 0.02
        const float rs = (float)(-AU) * iM, rs1 = rs + iM, rv_s = (float)(-AV) * iM;
        int i0, i1, j0, j1;
        sep_range(XU0, GU, -fmaxf(fmaxf(rs, rs1), 0.f) - 0.02f, 2.f - fminf(fminf(rs, rs1), 0.f) + 0.02f, cd.nu, i0,
                  i1);
        sep_range(XV0, GV, -fmaxf(rv_s, 0.f) - 0.02f, 1.f - fminf(rv_s, 0.f) + 0.02f, cd.nv, j0, j1);
        if (!live) j1 = j0 - 1;
        // this lane's V candidates: offsets from FP64 for the first, then
        // FP32 steps
        const float xv0 = (float)fma((double)j0, GV, XV0), gv = (float)GV;
        const float rvj = (float)(rV0 + j0 * rV1), rv1f = (float)rV1;
        const float* pview = pb + (long long)view * cd.nv * cd.nc;
        for (int base = i0; base <= i1; base += 32) {
            const int nk = min(32, i1 - base + 1);
            __syncwarp();
            if (lane < nk) {
                const int i = base + lane;
                const float xu = (float)fma((double)i, GU, XU0);
                const float ru = (float)fma((double)i, rU1, rU0);
                const float iru = fabsf(ru) > 1e-30f ? __fdividef(1.f, ru) : 1e30f;
                const float t0 = -xu * iru, t1 = (1.f - xu) * iru, t2 = (2.f - xu) * iru;
                s_t[warp][lane] = make_float4(fmaxf(clo, fminf(t0, t1)), fminf(chi, fmaxf(t0, t1)),
                                              fmaxf(clo, fminf(t1, t2)), fminf(chi, fmaxf(t1, t2)));
                s_i[warp][lane] = i;
            }
            __syncwarp();
            float kj = 0.f;
            for (int j = j0; j <= j1; j++, kj += 1.f) {
                const float xv = fmaf(kj, gv, xv0), rv = fmaf(kj, rv1f, rvj);
                const float irv = fabsf(rv) > 1e-30f ? __fdividef(1.f, rv) : 1e30f;
                const float tv0 = -xv * irv, tv1 = (1.f - xv) * irv;
                const float lv = fminf(tv0, tv1), hv = fmaxf(tv0, tv1);
                const float* pcol = pview + j * sv;
                // branch-free: a pair that misses both voxels adds exactly 0
#pragma unroll 2
                for (int k = 0; k < nk; k++) {
                    const float4 E = s_t[warp][k];
                    const float l0 = fminf(hv, E.y) - fmaxf(lv, E.x), l1 = fminf(hv, E.w) - fmaxf(lv, E.z);
                    const float p = __ldg(pcol + (long long)s_i[warp][k] * su);
                    acc0 = fmaf(fmaxf(l0, 0.f), p, acc0);
                    acc1 = fmaf(fmaxf(l1, 0.f), p, acc1);
                }
            }
        }
    }
    if (!live) return;
    auto out = [&](int qu, float v) {
        const int x = ax_u == 0 ? qu : ax_v == 0 ? pv : pm;
        const int y = ax_u == 1 ? qu : ax_v == 1 ? pv : pm;
        const int z = ax_u == 2 ? qu : ax_v == 2 ? pv : pm;
        float* o = img + bt * cd.img_b + ((long long)x * cd.st[0] + (long long)y * cd.st[1] + (long long)z * cd.st[2]) + c;
        *o = accumulate ? *o + v : v;
    };
    out(pu, acc0);
    if (live1) out(pu + 1, acc1);
}

// One thread per voxel (z fastest) of slice `bc` = b * nc + c.
// `fast` is the grid axis that runs along the lanes of a warp: z (the
// image's contiguous axis) by default, or the lateral axis that follows the
// detector's v (the projections' contiguous axis) for separable views, so
// that a warp's candidate rays are neighbours in memory.
__global__ void __launch_bounds__(256) cone_bp_kernel(float* __restrict__ img, const float* __restrict__ prj,
                                                       const float4* __restrict__ rays,
                                                       const ConeView* __restrict__ views, ConeDims cd,
                                                       int accumulate, int fast) {
    const long long nvox = (long long)cd.n[0] * cd.n[1] * cd.n[2];
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nvox) return;
    const int bc = blockIdx.y;
    const int c = bc % cd.nc, bt = bc / cd.nc;
    // q -> (fast axis, then the other two in x, y, z order, the last slowest)
    const int s1 = fast == 0 ? 1 : 0, s2 = fast == 2 ? 1 : 2;
    const int nf = fast == 0 ? cd.n[0] : fast == 1 ? cd.n[1] : cd.n[2];
    const int n1 = s1 == 0 ? cd.n[0] : cd.n[1];
    const int i_f = (int)(q % nf);
    const long long r = q / nf;
    const int i_1 = (int)(r % n1), i_2 = (int)(r / n1);
    const int x = fast == 0 ? i_f : i_1;
    const int y = fast == 1 ? i_f : (s1 == 1 ? i_1 : i_2);
    const int z = fast == 2 ? i_f : i_2;
    (void)s2;
    const float P[3] = {(float)x, (float)y, (float)z};
    const float* pb = prj + bt * cd.prj_b + c;
    float acc = 0.f;
    for (int view = 0; view < cd.nview; view++) {
        const ConeView& V = views[view];
        if (V.affine && bp_separable(acc, V, x, y, z, cd, pb, view)) continue;
        // shadow of the voxel [P, P + 1]^3 on the detector, in cell indices
        const float nu0 = fmaf(V.au[0], P[0], fmaf(V.au[1], P[1], fmaf(V.au[2], P[2], V.au[3])));
        const float nv0 = fmaf(V.av[0], P[0], fmaf(V.av[1], P[1], fmaf(V.av[2], P[2], V.av[3])));
        const float nd0 = fmaf(V.ad[0], P[0], fmaf(V.ad[1], P[1], fmaf(V.ad[2], P[2], V.ad[3])));
        const float dmin = nd0 + V.dlo, dmax = nd0 + V.dhi;
        if (!(dmin > 0.f)) continue;
        const float id0 = __fdividef(1.f, dmin), id1 = __fdividef(1.f, dmax);
        const float ulo = nu0 + V.ulo, uhi = nu0 + V.uhi, vlo = nv0 + V.vlo, vhi = nv0 + V.vhi;
        const int u0 = max(0, (int)ceilf(fminf(ulo * id0, ulo * id1) - 1e-3f));
        const int u1 = min(cd.nu - 1, (int)floorf(fmaxf(uhi * id0, uhi * id1) + 1e-3f));
        const int v0 = max(0, (int)ceilf(fminf(vlo * id0, vlo * id1) - 1e-3f));
        const int v1 = min(cd.nv - 1, (int)floorf(fmaxf(vhi * id0, vhi * id1) + 1e-3f));
        if (u0 > u1 || v0 > v1) continue;
        // voxel offsets from the source as hi / lo: A = S - lateral index,
        // M = main index - S_m
        const int m = V.m, a = V.a, b = V.b;
        const int pm = m == 0 ? x : m == 1 ? y : z, pa_ = a == 0 ? x : a == 1 ? y : z, pb_ = b == 0 ? x : b == 1 ? y : z;
        const float Shm = m == 0 ? V.Sh[0] : m == 1 ? V.Sh[1] : V.Sh[2];
        const float Sha = a == 0 ? V.Sh[0] : a == 1 ? V.Sh[1] : V.Sh[2];
        const float Shb = b == 0 ? V.Sh[0] : b == 1 ? V.Sh[1] : V.Sh[2];
        const float Slm = m == 0 ? V.Sl[0] : m == 1 ? V.Sl[1] : V.Sl[2];
        const float Sla = a == 0 ? V.Sl[0] : a == 1 ? V.Sl[1] : V.Sl[2];
        const float Slb = b == 0 ? V.Sl[0] : b == 1 ? V.Sl[1] : V.Sl[2];
        float Ah, Al, Bh, Bl, Mh, Ml, e;
        two_sum_f(Sha, -(float)pa_, Ah, e);
        Al = e + Sla;
        two_sum_f(Shb, -(float)pb_, Bh, e);
        Bl = e + Slb;
        two_sum_f((float)pm, -Shm, Mh, e);
        Ml = e - Slm;
        const float sm = (float)pm - Shm - Slm;   // main index - S_m (segment clipping only)
        const long long su = (long long)cd.nview * cd.nv * cd.nc;
        for (int iv = v0; iv <= v1; iv++) {
            const long long rrow = ((long long)view * cd.nv + iv) * cd.nu;
            const float* prow = pb + ((long long)view * cd.nv + iv) * cd.nc;
            for (int iu = u0; iu <= u1; iu++) {
                const float4 g0 = __ldg(rays + 2 * (rrow + iu));
                const float4 g1 = __ldg(rays + 2 * (rrow + iu) + 1);
                const float xa = fmaf(g0.x, Mh, Ah) + fmaf(g0.y, Mh, fmaf(g0.x, Ml, Al));
                const float xb = fmaf(g0.z, Mh, Bh) + fmaf(g0.w, Mh, fmaf(g0.z, Ml, Bl));
                const float ta0 = -xa * g1.x, ta1 = (1.f - xa) * g1.x;
                const float tb0 = -xb * g1.y, tb1 = (1.f - xb) * g1.y;
                // the segment's ends along m: source (at -sm from the voxel's
                // low face) and end point E_m
                const float e0 = -sm, e1 = g1.w - (float)pm;
                const float tl = fmaxf(fmaxf(fmaxf(0.f, fminf(ta0, ta1)), fminf(tb0, tb1)), fminf(e0, e1));
                const float th = fminf(fminf(fminf(1.f, fmaxf(ta0, ta1)), fmaxf(tb0, tb1)), fmaxf(e0, e1));
                // branch-free: a candidate that misses the voxel adds exactly 0
                acc = fmaf(fmaxf(th - tl, 0.f) * g1.z, __ldg(prow + (long long)iu * su), acc);
            }
        }
    }
    float* o = img + bt * cd.img_b + ((long long)x * cd.st[0] + (long long)y * cd.st[1] + (long long)z * cd.st[2]) + c;
    *o = accumulate ? *o + acc : acc;
}

}  // namespace rn

using namespace rn;

struct rn_cone_plan {
    ConeDims cd;
    int device = 0;
    ConeView* d_views = nullptr;
    float4* d_rays = nullptr;
    int lanes_v = 0;           // forward projection: warps along the detector's v
    int bp_fast = 2;           // backprojection: grid axis along the lanes
    bool bp_sep = false;       // every view separable the same way (cone_bp_sep_kernel)
    ConeView h_view0;          // host copy of view 0 (axes of a separable plan)
    bool unit = true;          // every ray's lateral slopes are at most 1
    float* d_prjw = nullptr;   // separable backprojection: projections times segment lengths (lazily allocated)
    long long launches = 0;
};

namespace {

int cone_views(rn_cone_plan* p, const RnConeGeom& g, const float* dc, const float* du_, const float* dv_,
               const float* src, std::vector<ConeView>& out, double& max_slope) {
    max_slope = 0.0;
    const int n[3] = {g.nx, g.ny, g.nz};
    const double d[3] = {g.dx, g.dy, g.dz}, cen[3] = {g.cx, g.cy, g.cz};
    const double u0 = g.off_u + (g.nu - 1) / 2.0, v0 = g.off_v + (g.nv - 1) / 2.0;
    out.resize(g.nview);
    for (int iv = 0; iv < g.nview; iv++) {
        ConeView V;
        memset(&V, 0, sizeof(V));
        for (int k = 0; k < 3; k++) {
            V.S[k] = ((double)src[3 * iv + k] - cen[k]) / d[k] + n[k] / 2.0;
            V.Eu[k] = (double)du_[3 * iv + k] * g.du / d[k];
            V.Ev[k] = (double)dv_[3 * iv + k] * g.dv / d[k];
            V.C[k] = ((double)dc[3 * iv + k] - u0 * g.du * du_[3 * iv + k] - v0 * g.dv * dv_[3 * iv + k] - cen[k]) / d[k] +
                     n[k] / 2.0;
            V.Sh[k] = (float)V.S[k];
            V.Sl[k] = (float)(V.S[k] - (double)V.Sh[k]);
        }
        // main axis: the largest advance of the central ray, in voxels
        double Dc[3];
        for (int k = 0; k < 3; k++) Dc[k] = V.C[k] + (g.nu - 1) / 2.0 * V.Eu[k] + (g.nv - 1) / 2.0 * V.Ev[k] - V.S[k];
        int m = 0;
        for (int k = 1; k < 3; k++)
            if (std::fabs(Dc[k]) > std::fabs(Dc[m])) m = k;
        V.m = m;
        V.a = (m + 1) % 3;
        V.b = (m + 2) % 3;
        if (V.a > V.b) std::swap(V.a, V.b);
        // every ray must advance along m, with lateral slopes of at most 4
        for (int corner = 0; corner < 4; corner++) {
            const double iu = (corner & 1) ? g.nu - 1 : 0, ivv = (corner & 2) ? g.nv - 1 : 0;
            double D[3];
            for (int k = 0; k < 3; k++) D[k] = V.C[k] + iu * V.Eu[k] + ivv * V.Ev[k] - V.S[k];
            if (D[m] * Dc[m] <= 0.0 || std::fabs(D[V.a]) > 4.0 * std::fabs(D[m]) ||
                std::fabs(D[V.b]) > 4.0 * std::fabs(D[m]))
                return set_error(RN_ERR_ARG, "cone geometry: rays of one view too oblique to a common main axis");
            max_slope = std::max(max_slope, std::max(std::fabs(D[V.a]), std::fabs(D[V.b])) / std::fabs(D[m]));
        }
        // shadow: the ray from S through P meets the detector plane at
        // index (iu, iv); with W = P - S and the plane normal nrm (oriented
        // so that K = nrm . (C - S) > 0), iu = (alpha_u . W) / (nrm . W)
        double nrm[3] = {V.Eu[1] * V.Ev[2] - V.Eu[2] * V.Ev[1], V.Eu[2] * V.Ev[0] - V.Eu[0] * V.Ev[2],
                         V.Eu[0] * V.Ev[1] - V.Eu[1] * V.Ev[0]};
        double K = 0;
        for (int k = 0; k < 3; k++) K += nrm[k] * (V.C[k] - V.S[k]);
        if (std::fabs(K) < 1e-12) return set_error(RN_ERR_ARG, "cone geometry: source in the detector plane");
        if (K < 0) {
            for (int k = 0; k < 3; k++) nrm[k] = -nrm[k];
            K = -K;
        }
        auto cross = [](const double* x, const double* y, double* r) {
            r[0] = x[1] * y[2] - x[2] * y[1];
            r[1] = x[2] * y[0] - x[0] * y[2];
            r[2] = x[0] * y[1] - x[1] * y[0];
        };
        double gu[3], gv[3];
        cross(V.Ev, nrm, gu);
        double su = 0;
        for (int k = 0; k < 3; k++) su += V.Eu[k] * gu[k];
        for (int k = 0; k < 3; k++) gu[k] /= su;
        cross(nrm, V.Eu, gv);
        double sv = 0;
        for (int k = 0; k < 3; k++) sv += V.Ev[k] * gv[k];
        for (int k = 0; k < 3; k++) gv[k] /= sv;
        double scu = 0, scv = 0;   // (S - C) . g
        for (int k = 0; k < 3; k++) {
            scu += (V.S[k] - V.C[k]) * gu[k];
            scv += (V.S[k] - V.C[k]) * gv[k];
        }
        double au[3], av[3], bu = 0, bv = 0, bd = 0;
        for (int k = 0; k < 3; k++) {
            au[k] = scu * nrm[k] + K * gu[k];
            av[k] = scv * nrm[k] + K * gv[k];
            bu -= au[k] * V.S[k];
            bv -= av[k] * V.S[k];
            bd -= nrm[k] * V.S[k];
        }
        for (int k = 0; k < 3; k++) {
            V.au[k] = (float)au[k];
            V.av[k] = (float)av[k];
            V.ad[k] = (float)nrm[k];
            V.ulo += (float)std::min(0.0, au[k]);
            V.uhi += (float)std::max(0.0, au[k]);
            V.vlo += (float)std::min(0.0, av[k]);
            V.vhi += (float)std::max(0.0, av[k]);
            V.dlo += (float)std::min(0.0, nrm[k]);
            V.dhi += (float)std::max(0.0, nrm[k]);
        }
        V.au[3] = (float)bu;
        V.av[3] = (float)bv;
        V.ad[3] = (float)bd;
        // separable views: the detector is perpendicular to the main axis and
        // its u / v steps each move along one lateral axis only
        const double tiny = 1e-9 * std::fabs(Dc[m]);
        const bool perp = std::fabs(V.Eu[m]) * g.nu + std::fabs(V.Ev[m]) * g.nv <= tiny;
        const bool a_u = std::fabs(V.Ev[V.a]) * g.nv <= tiny && std::fabs(V.Eu[V.b]) * g.nu <= tiny;
        const bool a_v = std::fabs(V.Eu[V.a]) * g.nu <= tiny && std::fabs(V.Ev[V.b]) * g.nv <= tiny;
        if (perp && (a_u || a_v)) {
            const double Dm0 = V.C[m] - V.S[m];
            V.affine = a_u ? 1 : 2;
            V.Dm0 = Dm0;
            V.rho[0] = (V.C[V.a] - V.S[V.a]) / Dm0;
            V.rho[1] = V.Eu[V.a] / Dm0;
            V.rho[2] = V.Ev[V.a] / Dm0;
            V.rho[3] = (V.C[V.b] - V.S[V.b]) / Dm0;
            V.rho[4] = V.Eu[V.b] / Dm0;
            V.rho[5] = V.Ev[V.b] / Dm0;
        }
        out[iv] = V;
    }
    (void)p;
    return RN_OK;
}

}  // namespace

extern "C" {

int rn_cone_plan_create(rn_cone_plan** out, const RnConeGeom* g, const float* host_detCenter, const float* host_detU,
                        const float* host_detV, const float* host_src, void* stream) {
    clear_error();
    if (!out || !g || !host_detCenter || !host_detU || !host_detV || !host_src)
        return set_error(RN_ERR_ARG, "null argument");
    *out = nullptr;
    if (g->nBatches <= 0 || g->nChannels <= 0 || g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->nu <= 0 ||
        g->nview <= 0 || g->nv <= 0)
        return set_error(RN_ERR_ARG, "cone geometry: sizes must be positive");
    if (!(g->dx > 0) || !(g->dy > 0) || !(g->dz > 0) || !(g->du > 0) || !(g->dv > 0))
        return set_error(RN_ERR_ARG, "cone geometry: pixel sizes must be positive");
    if ((long long)g->nx * g->ny * g->nz * g->nChannels >= (1LL << 31))
        return set_error(RN_ERR_ARG, "cone geometry: more than 2^31 voxels x channels per batch");
    rn_cone_plan* p = new rn_cone_plan();
    cudaGetDevice(&p->device);
    ConeDims& cd = p->cd;
    cd.n[0] = g->nx;
    cd.n[1] = g->ny;
    cd.n[2] = g->nz;
    cd.d[0] = g->dx;
    cd.d[1] = g->dy;
    cd.d[2] = g->dz;
    cd.nc = g->nChannels;
    cd.st[2] = cd.nc;
    cd.st[1] = (long long)g->nz * cd.nc;
    cd.st[0] = (long long)g->ny * cd.st[1];
    cd.nu = g->nu;
    cd.nv = g->nv;
    cd.nview = g->nview;
    cd.nb = g->nBatches;
    cd.img_b = (long long)g->nx * cd.st[0];
    cd.prj_b = (long long)g->nu * g->nview * g->nv * cd.nc;
    std::vector<ConeView> views;
    double max_slope = 0.0;
    int s = cone_views(p, *g, host_detCenter, host_detU, host_detV, host_src, views, max_slope);
    if (s != RN_OK) {
        delete p;
        return s;
    }
    p->unit = max_slope <= 1.0;
    // warps along iv when the detector's v step of view 0 runs mostly along z
    // and z is not the main axis
    {
        const double* e = views[0].Ev;
        p->lanes_v = (views[0].m != 2 && std::fabs(e[2]) >= std::max(std::fabs(e[0]), std::fabs(e[1]))) ? 1 : 0;
        // backprojection lanes along the lateral axis that follows the
        // detector's v when every view is separable the same way
        bool same = true;
        for (const ConeView& v : views)
            same = same && v.affine != 0 && v.affine == views[0].affine && v.a == views[0].a && v.b == views[0].b;
        if (same) p->bp_fast = views[0].affine == 1 ? views[0].b : views[0].a;
        p->bp_sep = same;
        p->h_view0 = views[0];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const long long nrays = (long long)g->nview * g->nv * g->nu;
    cudaError_t e = cudaMalloc(&p->d_views, sizeof(ConeView) * views.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->d_rays, sizeof(float4) * 2 * nrays);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_views, views.data(), sizeof(ConeView) * views.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        cone_ray_kernel<<<(unsigned)((nrays + 255) / 256), 256, 0, st>>>(p->d_rays, p->d_views, cd);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // `views` goes out of scope
    if (e != cudaSuccess) {
        rn_cone_plan_destroy(p);
        return set_cuda_error(e, "rn_cone_plan_create");
    }
    *out = p;
    return RN_OK;
}

int rn_cone_plan_destroy(rn_cone_plan* p) {
    if (!p) return RN_OK;
    cudaFree(p->d_views);
    cudaFree(p->d_rays);
    cudaFree(p->d_prjw);
    delete p;
    return RN_OK;
}

int rn_cone_project(rn_cone_plan* p, float* d_prj, const float* d_img, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    const ConeDims& cd = p->cd;
    const long long nz = (long long)cd.nb * cd.nview * cd.nc;
    if (nz > 65535) return set_error(RN_ERR_ARG, "cone projection: more than 65535 views x batches x channels");
    const int gx = p->lanes_v ? (cd.nu + 7) / 8 : (cd.nu + 31) / 32;
    const int gy = p->lanes_v ? (cd.nv + 31) / 32 : (cd.nv + 7) / 8;
    dim3 grid(gx, gy, (unsigned)nz);
    if (p->unit) {
        // float4 copies when the voxels along z come in aligned groups of 4
        const int vec = cd.nc == 1 && cd.n[2] % 4 == 0 && ((uintptr_t)d_img & 15) == 0;
        cone_fp_staged_kernel<<<grid, 256, kFpZ * kFpPlane * sizeof(float), (cudaStream_t)stream>>>(
            d_prj, d_img, p->d_views, cd, p->lanes_v, vec);
    } else {
        cone_fp_kernel<false><<<grid, 256, 0, (cudaStream_t)stream>>>(d_prj, d_img, p->d_views, cd, p->lanes_v);
    }
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

int rn_cone_backproject(rn_cone_plan* p, float* d_img, const float* d_prj, int accumulate, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    const ConeDims& cd = p->cd;
    const long long nvox = (long long)cd.n[0] * cd.n[1] * cd.n[2];
    const int slices = cd.nb * cd.nc;
    if (slices > 65535) return set_error(RN_ERR_ARG, "cone backprojection: too many batches x channels");
    if (p->bp_sep) {
        // one warp per 2 (U) x 32 (V) voxels at one m
        const ConeView& v0 = p->h_view0;
        const int ax_u = v0.affine == 1 ? v0.a : v0.b;
        const int nv_axis = cd.n[p->bp_fast];
        const long long warps = (long long)((cd.n[ax_u] + 1) / 2) * cd.n[v0.m];
        if (!p->d_prjw) RN_CUDA_TRY(cudaMalloc(&p->d_prjw, sizeof(float) * cd.nb * cd.prj_b));
        if (cd.nu > 65535 || cd.nview > 65535)
            return set_error(RN_ERR_ARG, "cone backprojection: more than 65535 detector columns or views");
        cone_prj_seg_kernel<<<dim3((unsigned)((cd.nv * cd.nc + 255) / 256), (unsigned)cd.nview, (unsigned)cd.nu), 256,
                              0, (cudaStream_t)stream>>>(p->d_prjw, d_prj, p->d_views, cd);
        RN_CUDA_TRY(cudaGetLastError());
        p->launches++;
        dim3 grid((unsigned)((warps + kSepWarps - 1) / kSepWarps), (unsigned)((nv_axis + 31) / 32), slices);
        cone_bp_sep_kernel<<<grid, 32 * kSepWarps, 0, (cudaStream_t)stream>>>(d_img, p->d_prjw, p->d_views, cd,
                                                                             accumulate);
    } else {
        dim3 grid((unsigned)((nvox + 255) / 256), slices);
        cone_bp_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(d_img, d_prj, p->d_rays, p->d_views, cd, accumulate,
                                                                p->bp_fast);
    }
    p->launches++;
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

long long rn_cone_plan_launches(const rn_cone_plan* p) { return p ? p->launches : 0; }

}  // extern "C"

namespace rn {

// r = a - b (cone OS-SQS residual, no weights: ossqs.cu:281-287).
__global__ void cone_residual_kernel(float* __restrict__ r, const float* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r[i] -= b[i];
}

// x = clamp(mask (x - lm bp / (norm + 1e-6)), lb, ub): Divide2D, Minus2D,
// Multiply2D and ValueCrop2D of ossqs.cu:299-316 in one pass.
__global__ void cone_sqs_kernel(float* __restrict__ x, const float* __restrict__ bp, const float* __restrict__ norm,
                                const float* __restrict__ mask, float lm, float lb, float ub, int clamp, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = (x[i] - lm * (bp[i] / (norm[i] + 1e-6f))) * mask[i];
        if (clamp) v = fminf(fmaxf(v, lb), ub);
        x[i] = v;
    }
}

static RnConeGeom cone_geom(int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, float cx,
                            float cy, float cz, int nu, int nview, int nv, float du, float dv, float off_u,
                            float off_v) {
    RnConeGeom g;
    g.nBatches = nBatches;
    g.nChannels = nChannels;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    g.cx = cx;
    g.cy = cy;
    g.cz = cz;
    g.nu = nu;
    g.nview = nview;
    g.nv = nv;
    g.du = du;
    g.dv = dv;
    g.off_u = off_u;
    g.off_v = off_v;
    return g;
}

// Device buffers of one host call, freed on every path.
struct HostBufs {
    std::vector<void*> ptrs;
    template <class T>
    int get(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, count * sizeof(T));
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc");
        ptrs.push_back(q);
        *p = reinterpret_cast<T*>(q);
        return RN_OK;
    }
    ~HostBufs() {
        for (void* q : ptrs) cudaFree(q);
    }
};

static int cone_host(bool forward, float* out, const float* in, const float* dc, const float* du_, const float* dv_,
                     const float* src, const RnConeGeom& g) {
    const size_t ni = (size_t)g.nBatches * g.nx * g.ny * g.nz * g.nChannels;
    const size_t np = (size_t)g.nBatches * g.nu * g.nview * g.nv * g.nChannels;
    rn_cone_plan* p = nullptr;
    RN_TRY(rn_cone_plan_create(&p, &g, dc, du_, dv_, src, nullptr));
    HostBufs hb;
    float *dimg = nullptr, *dprj = nullptr;
    int s = hb.get(&dimg, ni);
    if (s == RN_OK) s = hb.get(&dprj, np);
    if (s == RN_OK) {
        cudaError_t e = forward ? cudaMemcpy(dimg, in, ni * 4, cudaMemcpyHostToDevice)
                                : cudaMemcpy(dprj, in, np * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) s = set_cuda_error(e, "copy to device");
    }
    if (s == RN_OK) s = forward ? rn_cone_project(p, dprj, dimg, nullptr) : rn_cone_backproject(p, dimg, dprj, 0, nullptr);
    if (s == RN_OK) {
        cudaError_t e = forward ? cudaMemcpy(out, dprj, np * 4, cudaMemcpyDeviceToHost)
                                : cudaMemcpy(out, dimg, ni * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) s = set_cuda_error(e, "copy to host");
    }
    rn_cone_plan_destroy(p);
    return s;
}

}  // namespace rn

extern "C" {

void cSiddonConeProjectionAbitrary(float* prj, const float* img, const float* detCenter, const float* detU,
                                   const float* detV, const float* src, int nBatches, int nChannels, int nx, int ny,
                                   int nz, float dx, float dy, float dz, float cx, float cy, float cz, int nu,
                                   int nview, int nv, float du, float dv, float off_u, float off_v) {
    clear_error();
    if (!prj || !img) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    cone_host(true, prj, img, detCenter, detU, detV, src,
              cone_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v));
}

void cSiddonConeBackprojectionAbitrary(float* img, const float* prj, const float* detCenter, const float* detU,
                                       const float* detV, const float* src, int nBatches, int nChannels, int nx,
                                       int ny, int nz, float dx, float dy, float dz, float cx, float cy, float cz,
                                       int nu, int nview, int nv, float du, float dv, float off_u, float off_v) {
    clear_error();
    if (!prj || !img) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    cone_host(false, img, prj, detCenter, detU, detV, src,
              cone_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v));
}

void cOSSQSConeAbitrary(float* res, const float* img, const float* prj, const float* normImg, const float* mask,
                        const float* detCenter, const float* detU, const float* detV, const float* src, float lb,
                        float ub, int nviewPerSubset, int nSubsets, int nBatches, int nChannels, int nx, int ny,
                        int nz, float dx, float dy, float dz, float cx, float cy, float cz, int nu, int nview, int nv,
                        float du, float dv, float off_u, float off_v, int typeProjector, float lambda) {
    (void)typeProjector;
    clear_error();
    if (!res || !img || !prj || !normImg || !mask || !detCenter || !detU || !detV || !src || nviewPerSubset <= 0 ||
        nSubsets <= 0) {
        set_error(RN_ERR_ARG, "cOSSQSConeAbitrary: bad argument");
        return;
    }
    const size_t ni = (size_t)nBatches * nx * ny * nz * nChannels;
    const size_t rowC = (size_t)nv * nChannels;
    HostBufs hb;
    float *x = nullptr, *dn = nullptr, *dm = nullptr, *bp = nullptr, *fp = nullptr, *ps = nullptr;
    const size_t nsmax = (size_t)nBatches * nu * nviewPerSubset * rowC;
    if (hb.get(&x, ni) || hb.get(&dn, ni) || hb.get(&dm, ni) || hb.get(&bp, ni) || hb.get(&fp, nsmax) ||
        hb.get(&ps, nsmax))
        return;
    if (cudaMemcpy(x, img, ni * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dn, normImg, ni * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dm, mask, ni * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error(RN_ERR_CUDA, "cOSSQSConeAbitrary: copy failed");
        return;
    }
    std::vector<float> hs;
    int start = 0;
    for (int k = 0; k < nSubsets && start < nview; k++) {
        const int cnt = std::min(nviewPerSubset, nview - start);
        RnConeGeom g = cone_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, cnt, nv, du, dv, off_u,
                                 off_v);
        rn_cone_plan* p = nullptr;
        if (rn_cone_plan_create(&p, &g, detCenter + 3 * start, detU + 3 * start, detV + 3 * start, src + 3 * start,
                                nullptr) != RN_OK)
            return;
        const size_t ns = (size_t)nBatches * nu * cnt * rowC;
        hs.resize(ns);
        for (int b = 0; b < nBatches; b++)
            for (int u = 0; u < nu; u++)
                memcpy(&hs[((size_t)b * nu + u) * cnt * rowC], prj + (((size_t)b * nu + u) * nview + start) * rowC,
                       sizeof(float) * cnt * rowC);
        int s = RN_OK;
        if (cudaMemcpy(ps, hs.data(), ns * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            s = set_error(RN_ERR_CUDA, "cOSSQSConeAbitrary: copy failed");
        if (s == RN_OK) s = rn_cone_project(p, fp, x, nullptr);
        if (s == RN_OK) {
            cone_residual_kernel<<<(unsigned)std::min<size_t>((ns + 255) / 256, 148 * 16), 256>>>(fp, ps, (long long)ns);
            s = rn_cone_backproject(p, bp, fp, 0, nullptr);
        }
        if (s == RN_OK) {
            cone_sqs_kernel<<<(unsigned)std::min<size_t>((ni + 255) / 256, 148 * 16), 256>>>(
                x, bp, dn, dm, lambda * nSubsets, lb, ub, lb < ub ? 1 : 0, (long long)ni);
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) s = set_cuda_error(e, "cOSSQSConeAbitrary");
        }
        rn_cone_plan_destroy(p);
        if (s != RN_OK) return;
        start += cnt;
    }
    if (cudaMemcpy(res, x, ni * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        set_error(RN_ERR_CUDA, "cOSSQSConeAbitrary: copy failed");
}

}  // extern "C"
