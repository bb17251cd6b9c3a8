/*
 * reconnet_b200 -- B200-native (sm_100a) distance-driven CT projector library.
 *
 * C ABI only: plain pointers, sizes and scalars; no C++ or torch types.
 *
 * Two layers:
 *   1. Drop-in entry points with the reference's names and signatures
 *      (host pointers, synchronous).  Each replaces the reference function
 *      cited beside it (paths are relative to the wudufan/ReconNet tree).
 *   2. A native device API: device pointers, caller-chosen CUDA stream, no
 *      implicit device synchronisation, int status codes, and a plan object
 *      that owns geometry tables and scratch so repeated calls allocate
 *      nothing.
 *
 * Conventions (same as the reference):
 *   image    [nBatches][nx][ny][nz][nChannels]   float32, C order
 *   sinogram [nBatches][nu][nview][nv][nChannels] float32, C order
 *   angles in radians; da (angular detector pitch) = du_mm / dsd.
 *
 * typeProjector for the fan backprojector:
 *   0  iterative backprojection of the reference (length pre-weight),
 *   1  FBP backprojection of the reference (distance weight),
 *   2  matched backprojection: the exact transpose of the forward projector
 *      (not in the reference; used by OS-SQS and the autograd backward).
 *
 * Errors: native functions return RN_OK (0) or an RN_ERR_* code and set a
 * thread-local message readable with rn_last_error().  The reference-named
 * functions keep their void/float returns and also set rn_last_error();
 * rn_last_status() returns the code of the most recent call on the thread.
 */
#ifndef RECONNET_B200_H
#define RECONNET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RN_OK 0
#define RN_ERR_ARG 1         /* invalid argument or unsupported geometry */
#define RN_ERR_CUDA 2        /* CUDA runtime error */
#define RN_ERR_ALLOC 3       /* device allocation failed */
#define RN_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define RN_ERR_NOT_READY 5   /* library not initialised for this device */

#define RN_TYPE_ITERATIVE 0
#define RN_TYPE_FBP 1
#define RN_TYPE_MATCHED 2
#define RN_TYPE_SIDDON 3     /* Siddon ray lengths (rn_fan_project_siddon / rn_fan_backproject) */
#define RN_TYPE_PIXEL 4      /* pixel-driven FBP backprojection (rn_fan_backproject) */

const char* rn_last_error(void);
int rn_last_status(void);
int rn_version(void);

/* ------------------------------------------------------------------------
 * Reference-named drop-in entry points (host pointers, synchronous).
 * ------------------------------------------------------------------------ */

/* replaces ReconNet4D/Projector.cu:12 */
int SetDevice(int device);

/* replaces ReconNet4D/DistanceDriven.cu:386-439 (prj is overwritten) */
void cDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, int nBatches, int nChannels,
                                  int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv,
                                  float da, float dv, float off_a, float off_v, float dsd, float dso,
                                  int typeProjector);

/* replaces ReconNet4D/DistanceDriven.cu:793-846 (img is overwritten, as the
 * reference zeroes its device copy before accumulating) */
void cDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels,
                                      int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview,
                                      int nv, float da, float dv, float off_a, float off_v, float dsd, float dso,
                                      int typeProjector);

/* replaces ReconNet4D/Siddon.cu:424-479 (prj is overwritten) */
void cSiddonFanProjection(float* prj, const float* img, const float* deg, int nBatches, int nChannels, int nx, int ny,
                          int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da, float dv,
                          float off_a, float off_v, float dsd, float dso, int typeProjector);

/* replaces ReconNet4D/Siddon.cu:481-536 (img is overwritten, as the reference
 * zeroes its device copy before scattering) */
void cSiddonFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels, int nx,
                              int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da,
                              float dv, float off_a, float off_v, float dsd, float dso, int typeProjector);

/* replaces ReconNet4D/DistanceDriven3D.cu:346-407 */
void cDistanceDrivenTomoProjection(float* prj, const float* img, const float* detCenter, const float* src,
                                   int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz,
                                   float cx, float cy, float cz, int nu, int nview, int nv, float du, float dv,
                                   float off_u, float off_v);

/* replaces ReconNet4D/DistanceDriven3D.cu:666-727 */
void cDistanceDrivenTomoBackprojection(float* img, const float* prj, const float* detCenter, const float* src,
                                       int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy,
                                       float dz, float cx, float cy, float cz, int nu, int nview, int nv, float du,
                                       float dv, float off_u, float off_v);

/* replaces ReconNet4D/Filter.cu:432-474 (equiangular fan ramp filter) */
void cFilterFanFilter(float* pFPrj, const float* pPrj, int nBatches, int nChannels, int nu, int nview, int nv,
                      float da, float dv, float off_a, float off_v, float dsd, float dso, int typeFilter,
                      int typeProjector);

/* replaces ReconNet4D/Filter.cu:476-518 (equispaced parallel ramp filter) */
void cFilterParallelFilter(float* pFPrj, const float* pPrj, int nBatches, int nChannels, int nu, int nview, int nv,
                           float da, float dv, float off_a, float off_v, float dsd, float dso, int typeFilter,
                           int typeProjector);

/* replaces ReconNet4D/PixelDriven.cu:100-141 (pixel-driven backprojection
 * with the FBP weight dso^2 / L^2, bilinear in (u, v), zero beyond the
 * detector).  Same signature; typeProjector is ignored as in the reference;
 * img is overwritten.  Channels are read with their stride (the reference's
 * texture copy is only right for nChannels = 1). */
void cPixelDrivenFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels,
                                   int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv,
                                   float da, float dv, float off_a, float off_v, float dsd, float dso,
                                   int typeProjector);

/* replaces ReconNet4D/ossqs.cu:12-161.  Same arguments and the same projector:
 * the Siddon fan pair (cSiddonFanProjection and its transpose), typeProjector
 * ignored as the reference's SiddonFan ignores it.  The last subset holds
 * views [startView, nview) instead of the reference's nview - nviewPerSubset. */
void cOSSQS(float* res, const float* img, const float* prj, const float* normImg, const float* wprj,
            const float* degs, float lb, float ub, int nviewPerSubset, int nSubsets, int nBatches, int nChannels,
            int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da, float dv,
            float off_a, float off_v, float dsd, float dso, int typeProjector, float lambda);

/* cOSSQS with the DD fan pair: cDistanceDrivenFanProjection and the
 * backprojector selected by typeProjector (0 / 1 reference modes, 2 matched
 * transpose).  No reference counterpart. */
void cDDFanOSSQS(float* res, const float* img, const float* prj, const float* normImg, const float* wprj,
                 const float* degs, float lb, float ub, int nviewPerSubset, int nSubsets, int nBatches,
                 int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv,
                 float da, float dv, float off_a, float off_v, float dsd, float dso, int typeProjector,
                 float lambda);

/* replaces ReconNet4D/TotalVariation.cu:70-142; the TV value is summed in FP64 */
float cTVSQS2D(float* grad, float* norm, const float* img, int nx, int ny);

/* ------------------------------------------------------------------------
 * Native device API.
 * ------------------------------------------------------------------------ */

/* Geometry; field names and meaning follow Projector (ReconNet4D/Projector.h:10-37).
 * du is the angular pitch (da) for the fan projector. */
typedef struct RnFanGeom {
    int nBatches, nChannels;
    int nx, ny, nz;
    float dx, dy, dz;
    float cx, cy, cz;
    int nu, nview, nv;
    float du, dv, off_u, off_v;
    float dsd, dso;
} RnFanGeom;

typedef struct rn_fan_plan rn_fan_plan;

/* Plan for the reference layout: image [B][nx][ny][nz][C], sinogram
 * [B][nu][nview][nv][C], one angle list (host_deg, nview floats) shared by
 * all batches.  Builds device geometry tables and scratch on `stream`. */
int rn_fan_plan_create(rn_fan_plan** plan, const RnFanGeom* g, const float* host_deg, void* stream);

/* Plan for a ragged batch of independent 2D slices (the batched OS-SQS
 * workload): g->nBatches slices of [nx][ny] stored back to back; slice s has
 * nview_per_slice[s] views with angles host_deg[view_offset(s) + k], and its
 * sinogram [nu][nview_s] starts at float offset nu * view_offset(s) of a
 * packed sinogram buffer, where view_offset(s) = sum of nview over earlier
 * slices.  nz, nv, nChannels must be 1. */
int rn_fan_plan_create_ragged(rn_fan_plan** plan, const RnFanGeom* g, const int* nview_per_slice,
                              const float* host_deg, void* stream);

int rn_fan_plan_destroy(rn_fan_plan* plan);

/* Total number of views in the plan (sum over slices for ragged plans). */
int64_t rn_fan_plan_total_views(const rn_fan_plan* plan);

/* Forward projection, device pointers, stream-ordered; prj is overwritten. */
int rn_fan_project(rn_fan_plan* plan, float* d_prj, const float* d_img, void* stream);

/* Siddon forward projection (SiddonFanProjectionKernel,
 * ReconNet4D/Siddon.cu:240-266): each ray, from the source to the centre of
 * its detector cell at the height of its detector row, sums the voxels times
 * the length (mm) of the ray inside them.  prj is overwritten. */
int rn_fan_project_siddon(rn_fan_plan* plan, float* d_prj, const float* d_img, void* stream);

/* Backprojection; typeProjector as above (RN_TYPE_SIDDON: the exact transpose
 * of rn_fan_project_siddon, gathered per voxel; the reference scatters with
 * atomics, Siddon.cu:268-380; RN_TYPE_PIXEL: the pixel-driven FBP
 * backprojection of PixelDriven.cu:11-62).  accumulate = 0 overwrites img, 1
 * adds to it (the reference class-level Backprojection accumulates). */
int rn_fan_backproject(rn_fan_plan* plan, float* d_img, const float* d_prj, int typeProjector, int accumulate,
                       void* stream);

/* Device-side error word of the plan's kernels (bounded waits that gave up):
 * synchronises `stream`, returns RN_OK or RN_ERR_TIMEOUT, clears the word. */
int rn_fan_plan_check(rn_fan_plan* plan, void* stream);

/* Polls each chunk wait of the plan's projection and backprojection kernels
 * makes before it gives up (records RN_ERR_TIMEOUT, waits for its own bulk
 * copy in flight, and returns); -1 restores the default of 2^22.  A limit of
 * 0 makes every wait give up at once: the failure path runs, without any
 * fault, for tests. */
int rn_fan_plan_set_spin_limit(rn_fan_plan* plan, long long polls);

/* Instrumentation.  rn_fan_plan_set_timing(plan, 1) brackets every kernel
 * launch of the plan with CUDA events on its stream; rn_fan_plan_read_timing
 * synchronises on them and returns, per kernel kind (0 line prologue,
 * 1 forward projection, 2 edge tables, 3 backprojection, 4 other), the summed
 * milliseconds and launch counts since the last read, plus the total number of
 * kernels the plan has launched. */
int rn_fan_plan_set_timing(rn_fan_plan* plan, int enable);
int rn_fan_plan_read_timing(rn_fan_plan* plan, float* ms, int* counts, int nkinds, long long* launches);

/* Launch-parameter tuning (no counterpart in the reference, whose kernels
 * have fixed launch shapes).  Three parameters shape a plan's launches:
 *   fp_views  views per forward-projection CTA (1 .. 4 for up to ~990
 *             channels; fewer views give more, smaller CTAs),
 *   fp_lines  image lines per chunk staged into shared memory (1 .. the most
 *             that fit),
 *   bp_parts  CTAs over which each backprojection tile's views are split
 *             when the whole batch runs in one launch (1 .. 16, and at most
 *             what the plan's scratch holds; used only for batches too small
 *             to fill the GPU).
 * 0 selects the built-in choice; rn_fan_plan_set_tuning clamps fp_views and
 * fp_lines to their maxima.  Results do not depend on them beyond
 * FP32 rounding of the chunked positions.
 * rn_fan_plan_autotune times the candidates on the caller's buffers (prj is
 * overwritten; for typeProjector's backprojection the plan allocates an
 * image-sized scratch once) and keeps the fastest; choices are cached for the
 * process by geometry, per-slice view counts and type, so a second plan of
 * the same shape takes them without timing.  rn_fan_plan_set_tuning sets
 * them directly (a solver can tune one subset plan and apply its choice to
 * the others); rn_fan_plan_get_tuning returns the values in use (bp_parts 0 =
 * built-in).  Both re-upload the plan's work list on `stream`: the plan must
 * not be running on another stream meanwhile. */
int rn_fan_plan_autotune(rn_fan_plan* plan, float* d_prj, const float* d_img, int typeProjector, void* stream);
int rn_fan_plan_set_tuning(rn_fan_plan* plan, int fp_views, int fp_lines, int bp_parts, void* stream);
int rn_fan_plan_get_tuning(const rn_fan_plan* plan, int* fp_views, int* fp_lines, int* bp_parts);

/* Ramp filter on device pointers (fan = 1 equiangular / 0 parallel); same
 * parameters as cFilterFanFilter. */
int rn_filter(float* d_out, const float* d_prj, int nBatches, int nChannels, int nu, int nview, int nv, float da,
              float off_a, float dsd, float dso, int typeFilter, int fan, void* stream);

/* Which ramp-filter kernel rn_filter and the host filters run (process-wide):
 * 0 (default) the register four-step FFT where the transform length is 512,
 * 1024 or 2048 (nu <= 1024), else the shared-memory FFT; 1 the
 * shared-memory FFT; 2 the direct Toeplitz product.  All give the same
 * result to FP32 rounding; the choice exists for comparisons. */
int rn_filter_set_form(int form);

/* The same filter with short-scan weights d_w [nu][nview] (broadcast over
 * batches, detector rows and channels) multiplied into the sinogram as it is
 * loaded: the reference's FBP chain multiplies its Parker / Riess weights
 * into the projections before cFilterFanFilter (python/ReconNet_no_tf.py:
 * 640-693 with :396-440).  d_w comes from rn_fan_shortscan_weights. */
int rn_filter_weighted(float* d_out, const float* d_prj, const float* d_w, int nBatches, int nChannels, int nu,
                       int nview, int nv, float da, float off_a, float dsd, float dso, int typeFilter, int fan,
                       void* stream);

/* Short-scan redundancy weights [nu][nview] for fan-beam FBP over
 * [0, angles[nview-1]] (gamma = (angles[nview-1] - pi) / 2).  Replaces the
 * reference's Python ParkerWeighting / RiessWeighting
 * (python/ReconNet_no_tf.py:640-659 / 665-693), with the same channel angle
 * alpha = ((u - (nu-1)/2) - off_a) * da.  kind RN_WEIGHT_PARKER, or
 * RN_WEIGHT_RIESS with its Gaussian smoothing (sigma channels, reach
 * int(4 sigma + 0.5)) outside theta < beta < pi + 2 gamma - theta.  riessMask
 * 0 keeps only channel 0 of those middle views unsmoothed, as the reference's
 * np.where(np.all(...)) does; 1 keeps the whole view unsmoothed.  d_angles is
 * a device array; the _host variant takes and returns host arrays.  Pitch,
 * offset, sigma and theta are doubles, as the reference's Python holds them. */
#define RN_WEIGHT_PARKER 0
#define RN_WEIGHT_RIESS 1
int rn_fan_shortscan_weights(float* d_w, const float* d_angles, int nu, int nview, double da, double off_a, int kind,
                             double sigma, double theta, int riessMask, void* stream);
int rn_fan_shortscan_weights_host(float* w, const float* angles, int nu, int nview, double da, double off_a, int kind,
                                  double sigma, double theta, int riessMask);

/* TV surrogate on a batch of S slices [S][nx][ny]; grad/norm may be NULL;
 * d_tv (may be NULL) receives S FP64 TV values. */
int rn_tv_sqs(float* d_grad, float* d_norm, double* d_tv, const float* d_img, int nslices, int nx, int ny,
              void* stream);

/* ---------------------------------------------------------------------------
 * Siddon cone-beam pair with arbitrary per-view geometry (SiddonCone.cu).
 * Ray (iu, iview, iv) runs from src[iview] to detCenter[iview] + u detU[iview]
 * + v detV[iview], u = (iu - off_u - (nu-1)/2) du, v = (iv - off_v -
 * (nv-1)/2) dv; the grid of nx x ny x nz voxels (dx, dy, dz mm) is centred at
 * (cx, cy, cz).  Geometry arrays are [nview][3] floats (mm), images
 * [nBatches][nx][ny][nz][nChannels], projections [nBatches][nu][nview][nv]
 * [nChannels].  Every view needs a main axis along which all its rays advance,
 * with lateral slopes of at most 4 (RN_ERR_ARG otherwise).
 * ------------------------------------------------------------------------- */
typedef struct {
    int nBatches, nChannels, nx, ny, nz;
    float dx, dy, dz, cx, cy, cz;
    int nu, nview, nv;
    float du, dv, off_u, off_v;
} RnConeGeom;

typedef struct rn_cone_plan rn_cone_plan;

/* Plan: per-view geometry and the per-ray table (32 B per ray) on the device.
 * The geometry arrays are host pointers. */
int rn_cone_plan_create(rn_cone_plan** plan, const RnConeGeom* g, const float* detCenter, const float* detU,
                        const float* detV, const float* src, void* stream);
int rn_cone_plan_destroy(rn_cone_plan* plan);
/* Forward projection (prj overwritten) and its exact transpose (accumulate =
 * 0 overwrites img, 1 adds to it), device pointers, on `stream`. */
int rn_cone_project(rn_cone_plan* plan, float* d_prj, const float* d_img, void* stream);
int rn_cone_backproject(rn_cone_plan* plan, float* d_img, const float* d_prj, int accumulate, void* stream);
long long rn_cone_plan_launches(const rn_cone_plan* plan);

/* replaces ReconNet4D/SiddonCone.cu:126-201 (host pointers; prj overwritten) */
void cSiddonConeProjectionAbitrary(float* prj, const float* img, const float* detCenter, const float* detU,
                                   const float* detV, const float* src, int nBatches, int nChannels, int nx, int ny,
                                   int nz, float dx, float dy, float dz, float cx, float cy, float cz, int nu,
                                   int nview, int nv, float du, float dv, float off_u, float off_v);

/* replaces ReconNet4D/SiddonCone.cu:203-278 (host pointers; img overwritten;
 * the exact transpose, gathered per voxel: the reference scatters with
 * atomics) */
void cSiddonConeBackprojectionAbitrary(float* img, const float* prj, const float* detCenter, const float* detU,
                                       const float* detV, const float* src, int nBatches, int nChannels, int nx,
                                       int ny, int nz, float dx, float dy, float dz, float cx, float cy, float cz,
                                       int nu, int nview, int nv, float du, float dv, float off_u, float off_v);

/* replaces ReconNet4D/ossqs.cu:163-333: OS-SQS with the cone pair,
 *   x = clamp(mask * (x - lambda nSubsets A_s^T (A_s x - b_s) / (normImg + 1e-6)), lb, ub)
 * over contiguous subsets of nviewPerSubset views (the last one holds the
 * remaining views); typeProjector is ignored as in the reference. */
void cOSSQSConeAbitrary(float* res, const float* img, const float* prj, const float* normImg, const float* mask,
                        const float* detCenter, const float* detU, const float* detV, const float* src, float lb,
                        float ub, int nviewPerSubset, int nSubsets, int nBatches, int nChannels, int nx, int ny,
                        int nz, float dx, float dy, float dz, float cx, float cy, float cz, int nu, int nview, int nv,
                        float du, float dv, float off_u, float off_v, int typeProjector, float lambda);

/* Isotropic TV surrogate of the prior solver (PriorFunctionSolver/TVSQS.cu:8-93
 * 2D, :160-265 3D) on device pointers, one pass: with backward differences d_k
 * and forward differences f_k (0 on the borders),
 *   var = sqrt(sum_k d_k^2 + eps),
 *   s1  = sum_k d_k / var + sum_k f_k / var(p + e_k),
 *   s2  = ndim / var + sum_k 1 / var(p + e_k)   (var(p + e_k) = var on the high border).
 * Arrays [nb][nx][ny][nz][nc]; ndim 2 requires nz = 1; d_var may be NULL. */
int rn_tv_iso_sqs(float* d_s1, float* d_s2, float* d_var, const float* d_img, int nb, int nx, int ny, int nz, int nc,
                  float eps, int ndim, void* stream);

/* The same on host pointers (synchronous; the prior-solver shim's cTVSQS2D /
 * cTVSQS3D forward here). */
int rn_tv_iso_sqs_host(float* s1, float* s2, float* var, const float* img, int nb, int nx, int ny, int nz, int nc,
                       float eps, int ndim);

/* One OS-SQS subset update on all slices of a plan (device pointers):
 *   x_out = clamp(x_in - lambda * (nSubsets * A_s^T W_s (A_s x_in - b_s) + beta * grad_tv(x_in))
 *                  / (normImg + beta * norm_tv(x_in) + 1e-6), lb, ub)
 * `subset_plan` is a plan holding only the subset's views (same slice
 * layout); d_prj_s / d_w_s are the subset's measured and weight sinograms in
 * that plan's layout.  typeProjector 0 / 1 / 2 run the DD forward projector
 * with that backprojector, 3 the Siddon pair.  x_out must not alias x_in. */
int rn_fan_sqs_update(rn_fan_plan* subset_plan, float* d_x_out, const float* d_x_in, const float* d_prj_s,
                      const float* d_w_s, const float* d_norm_img, float lambda, float beta, int nSubsets, float lb,
                      float ub, int typeProjector, void* stream);

/* Forward projection of one 2D slice that allocates nothing (no counterpart
 * in the reference).  For callers that may not allocate device memory --
 * code running inside another framework's memory pool or under a fixed
 * memory budget, real-time pipelines that forbid cudaMalloc after start-up,
 * plugins handed only device pointers.  Same kernels and results as
 * rn_fan_project on a plan with nBatches = nChannels = nz = nv = 1: d_img is
 * [nx][ny], d_prj [nu][nview] (both device memory, caller-owned), host_deg
 * holds nview angles on the host.  All scratch (geometry tables, edge slopes,
 * line prefix arrays) lives in one fixed 16 MiB device array compiled into
 * the library, which every GPU that loads the library keeps until exit; a
 * geometry whose scratch exceeds it (bytes ~ 8*nview*(nu+1) +
 * 16*(ny*(nx+1+2m) + nx*(ny+1+2m)) + small tables, m ~ 12 line padding
 * entries, e.g. 512x512 with up to about 1000 views of 888 channels) is
 * rejected with RN_ERR_ARG and a message giving the bytes needed.  The
 * first call on a device sets up that device: it looks up the array's device
 * address (cudaGetSymbolAddress) with the device current, so make that first
 * call before any stream capture.  Every call shares the one array and
 * overwrites it (the device error word is cleared by each call), so calls
 * that overlap on the GPU -- from several host threads or streams -- race;
 * serialise them.  The call synchronises `stream` before returning. */
int rn_fan_project_noalloc(float* d_prj, const float* d_img, const float* host_deg, int nx, int ny, float dx,
                           float dy, int nu, int nview, float da, float off_a, float dsd, float dso, void* stream);

/* Tomosynthesis DD on device pointers (same arguments as the reference-named
 * host functions above plus a caller-provided FP64 scratch d_sat whose size
 * rn_tomo_sat_bytes reports: fp_bytes for projection, bp_bytes for
 * backprojection).  detCenter / src are [nview][3] device arrays.
 * weightAllViews = 0 reproduces cDistanceDrivenTomoBackprojection, whose
 * length pre-weight reaches view 0 only (its launch grid holds one row of
 * views, ReconNet4D/DistanceDriven3D.cu:612-621); 1 weights every view. */
int rn_tomo_sat_bytes(int nx, int ny, int nz, int nu, int nview, int nv, size_t* fp_bytes, size_t* bp_bytes);
int rn_tomo_project(float* d_prj, const float* d_img, const float* d_detCenter, const float* d_src, double* d_sat,
                    int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, float cx,
                    float cy, float cz, int nu, int nview, int nv, float du, float dv, float off_u, float off_v,
                    void* stream);
int rn_tomo_backproject(float* d_img, const float* d_prj, const float* d_detCenter, const float* d_src, double* d_sat,
                        int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, float cx,
                        float cy, float cz, int nu, int nview, int nv, float du, float dv, float off_u, float off_v,
                        int weightAllViews, void* stream);

/* ---------------------------------------------------------------------------
 * Cylindrical-detector cone-beam DD pair on a circular orbit (no counterpart
 * in the reference: its DistanceDriven3D.cu:139-227 / 519-559 is a flat,
 * axis-aligned tomosynthesis pair with z as the main axis; this generalises
 * that rectangle-footprint DD and the fan geometry of DistanceDriven.cu:64-196
 * to a 360-degree orbit).  Source (dso sin t, -dso cos t, 0); detector a
 * cylinder of radius dsd about the source, cell (u, v) at fan angle
 * a_u = (-(u - (nu-1)/2) - off_a) da and height v_c = (v - (nv-1)/2 + off_v) dv
 * at the detector; volume of nx x ny x nz voxels (dx, dy, dz mm) centred at
 * (cx, cy, cz).  Volumes are [nBatches][nx][ny][nz], projections
 * [nBatches][nu][nview][nv] (the reference's layouts without channels).  The
 * backprojection is the exact transpose and overwrites its output.  The plan
 * owns the view tables and the backprojection's row tables
 * (nBatches * nview * nu * (nv + 1) float2). */
typedef struct RnCylGeom {
    int nBatches;
    int nx, ny, nz;
    float dx, dy, dz, cx, cy, cz;
    int nu, nview, nv;
    float da, dv, off_a, off_v, dsd, dso;
} RnCylGeom;
typedef struct rn_cyl_plan rn_cyl_plan;
int rn_cyl_plan_create(rn_cyl_plan** plan, const RnCylGeom* geom, const float* host_deg, void* stream);
int rn_cyl_plan_destroy(rn_cyl_plan* plan);
int rn_cyl_project(rn_cyl_plan* plan, float* d_prj, const float* d_vol, void* stream);
int rn_cyl_backproject(rn_cyl_plan* plan, float* d_vol, const float* d_prj, void* stream);
long long rn_cyl_plan_launches(const rn_cyl_plan* plan);

/* ---------------------------------------------------------------------------
 * BF16 3x3 convolutions of the learned prior (no counterpart in the
 * reference, whose learned path is TensorFlow's: python/ReconNet.py:773-830).
 * tcgen05 tensor-core kernels with FP32 accumulation; activations are bf16
 * "blocked" [N][C/8][H][W][8], 16-byte aligned.  d_wpack is the weight
 * operand image: chunk kc of 8 input channels x NPAD output rows x 8 bf16
 * (NPAD = 32, or 16 for one output channel), kc = tap * (cin/8) + ci/8 for
 * cin = 32, kc = tap for cin = 8 (plus a zero tenth chunk).
 * mode 0: d_out blocked bf16 = relu(conv + bias), cout 32;
 * mode 1: d_out fp32 [N][H][W] = conv + bias + d_aux (fp32 residual), cout 1;
 * mode 2: d_out blocked bf16 = conv * (d_aux > 0), d_aux the blocked
 *         activation (the input gradient through a ReLU), cout 32;
 * mode 3: d_out fp32 [N][cout][H][W] = conv (+ bias if given).
 * A device wait that runs out records RN_ERR_TIMEOUT in *d_err. */
int rn_conv3x3(void* d_out, const void* d_in, const void* d_wpack, const float* d_bias, const void* d_aux, int N,
               int H, int W, int cin, int cout, int mode, int* d_err, void* stream);
/* Weight gradient: d_dw [32][ncols] fp32, ncols = rn_conv3x3_wgrad_cols(cin):
 * column tap * 32 + ci (cin 32) or (tap / 2) * 16 + (tap % 2) * 8 + ci (cin 8),
 * then 16 columns of the bias gradient sum_p dY[p][co]; rows >= cout are 0.
 * d_partial: scratch of at least (number of SMs) * 32 * ncols floats. */
int rn_conv3x3_wgrad_cols(int cin);
int rn_conv3x3_wgrad(float* d_dw, float* d_partial, size_t partial_bytes, const void* d_x, const void* d_dy, int N,
                     int H, int W, int cin, int cout, int* d_err, void* stream);
/* fp32 [N][H][W] -> blocked bf16 with 8 channels: channel 0 = (img - sub) * scale
 * (d_sub may be NULL), channels 1..7 zero. */
int rn_conv_pack_image(void* d_out, const float* d_img, const float* d_sub, float scale, int N, int H, int W,
                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RECONNET_B200_H */
