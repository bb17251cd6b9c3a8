// Internal definitions shared by the reconnet_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/reconnet_b200.h"

namespace rn {

// ---------------------------------------------------------------------------
// Error reporting (thread-local last error, int status codes).
// ---------------------------------------------------------------------------
int set_error(int code, const std::string& msg);
int set_cuda_error(cudaError_t e, const char* what);
void clear_error();

#define RN_CUDA_TRY(call)                                         \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return ::rn::set_cuda_error(_e, #call); \
    } while (0)

#define RN_TRY(call)                       \
    do {                                   \
        int _s = (call);                   \
        if (_s != RN_OK) return _s;        \
    } while (0)

// Spin limit of every device-side wait (mbarrier parity waits).  A wait that
// exceeds it records RN_ERR_TIMEOUT in the plan's error word and the kernel
// returns early instead of hanging the GPU.
constexpr long long kSpinLimit = 1ll << 22;

// ---------------------------------------------------------------------------
// Geometry tables (device).
// ---------------------------------------------------------------------------

// Per view, image coordinates with the origin at the corner of pixel 0
// (PhysicsToImg, ReconNet4D/DistanceDriven.cu:14-20).  "Lines" are image rows
// for X-class views (|cos| > |sin|, DistanceDriven.cu:299-312) and image
// columns for Y-class views; positions along a line are x (X) or y (Y).
struct ViewGeo {
    double par, perp;   // source coordinate along / across the lines
    float cosd, sind;   // cos/sin of the view angle
    float tA, tB;       // edge index of a slope r: t = tA + tB * atan(kappa * r)
    float kappa;        // physical / image slope factor
    float rmin, rmax;   // slope range covered by the detector
    float sigma;        // +-1: do edge indices increase along the line?
    int xcls;           // 1 = X-class
    int pad[3];         // 64-byte records: chunks of them are bulk-copyable
};
static_assert(sizeof(ViewGeo) == 64, "ViewGeo is staged by 16-byte bulk copies");

// A 2D forward problem: sinogram plane at prj_off (strides su, sview)
// projected from a mix of up to 2 image planes (z interpolation).
struct FpSlice {
    long long img_off[2];
    float img_w[2];
    long long prj_off;
    int su, sview;
    int set;            // geometry set (angle list)
    int line_slot;      // index of this slice's line buffers
};

// A 2D backward problem: image plane at img_off from a mix of up to 4
// sinogram planes.
constexpr int kBpMix = 4;
// Backprojection tiles (CTA of 256 threads, every mode): 31 pixel columns
// (one per lane; lane 31 only supplies an edge) by 8 warps x kBmRows rows.
constexpr int kBpThreads = 256;
constexpr int kBmCols = 31;
constexpr int kBmRows = 16;
constexpr int kBmTileY = kBmRows * (kBpThreads / 32);
constexpr int kBpMaxParts = 16;   // most view parts of a split backprojection

struct BpSlice {
    long long img_off;
    long long prj_off[kBpMix];
    float prj_w[kBpMix];
    int su, sview;
    int set;
    long long table_off;  // first float4 of this slice's edge tables
};

struct GeoSet {
    int view_off;   // first view in the view tables
    int nview;
    int nxv;        // number of X-class views; class-sorted order in perm
};

// Kernel launch parameters shared by the fan kernels.
// FP line arrays keep one unused slot after every 16 entries (entry j at
// j + j / 16), so that the lanes of a warp, whose entries are typically 1-1.4
// apart, do not meet in the same shared-memory bank 16 or 32 entries apart.
__host__ __device__ inline int line_pos(int j) { return j + (j >> 4); }
inline int line_stride(int lp) { return (line_pos(lp - 1) + 1 + 3) & ~3; }

struct FanDims {
    int nx, ny, nu;
    float dx, dy;
    float du, off_u, dsd, dso;
    int margin;     // padding entries on each side of an FP line array
    int lpx, lpy;   // FP line lengths: n + 1 + 2 * margin, rounded up to a multiple of 4
    int spx, spy;   // FP line strides in memory: entry j sits at line_pos(j)
    long long isx, isy;   // image strides (elements) along x and y
};

}  // namespace rn

// Plan object (opaque in the C API).
struct rn_fan_plan {
    RnFanGeom g;
    bool ragged;
    int device;
    rn::FanDims dims;

    // host copies
    std::vector<rn::GeoSet> h_sets;
    std::vector<rn::FpSlice> h_fp;
    std::vector<rn::BpSlice> h_bp;     // matched backprojection slices
    std::vector<rn::BpSlice> h_bpr;    // reference-mode backprojection slices
    std::vector<int> h_fp_work;    // packed FP work items
    int n_fp_work = 0;
    int64_t total_views = 0;
    long long prj_elems = 0, img_elems = 0;

    // device tables
    rn::ViewGeo* d_views = nullptr;
    double* d_edges = nullptr;      // [total_views][nu+1] slopes
    float2* d_cell = nullptr;       // [nu] (cos a_u, sin a_u)
    int* d_perm = nullptr;          // [total_views] class-sorted view order per set
    rn::GeoSet* d_sets = nullptr;
    rn::FpSlice* d_fp = nullptr;
    rn::BpSlice* d_bp = nullptr;
    rn::BpSlice* d_bpr = nullptr;
    int4* d_fp_work = nullptr;      // {slice, class, vbegin, vcount}
    // Siddon pair: FP slices (one image slice per detector row), BP slices
    // (the detector rows of each image slice) and ray slopes at cell centres
    std::vector<rn::FpSlice> h_fps;
    std::vector<rn::BpSlice> h_bps;
    rn::FpSlice* d_fps = nullptr;
    rn::BpSlice* d_bps = nullptr;
    double* d_cslopes = nullptr;    // [views][nu + 1], entry u = slope of the ray through cell u
    int* d_err = nullptr;           // device error word

    // scratch
    float2* d_hl = nullptr;         // FP line prefixes (hi, lo)
    float* d_la = nullptr;          // FP line values
    long long line_slot_elems = 0;  // per FP slice: ny*lpx + nx*lpy
    long long fp_slots = 0;         // FP slices whose lines fit in the scratch
    int table_win_m = 0;            // staged table entries per view (BP tiles of 31 x 128 pixels)
    float4* d_tab = nullptr;        // BP edge tables
    long long tab_elems = 0;
    float* d_tmp_img = nullptr;     // image-sized scratch (SQS update, autotuner)
    float* d_bp_parts = nullptr;    // partial images of a view-split backprojection
    long long bp_parts_cap = 0;     // elements
    // launch parameters (0 = the built-in choice); set by rn_fan_plan_set_tuning
    // or rn_fan_plan_autotune
    int fp_vt = 0;                  // views per forward-projection work item
    int fp_R = 0;                   // lines per staged chunk of the forward projection
    int bp_nparts = 0;              // view parts of a split backprojection (single-launch batches)
    int fp_vt_used = 0;             // views per work item of the current work list
    int fp_work_cap = 0;            // work items the device list holds (one view each)
    long long spin_limit = rn::kSpinLimit;   // polls of a chunk wait before it gives up
    float* d_tmp_prj = nullptr;     // sinogram-sized scratch (SQS update)
    // every device table and scratch above lives in this one allocation
    void* d_arena = nullptr;
    size_t arena_bytes = 0;

    // instrumentation: kernel launch count and optional per-kernel CUDA-event
    // timing (kinds: 0 line prologue, 1 forward projection, 2 edge tables,
    // 3 backprojection, 4 other)
    long long launches = 0;
    bool timing = false;
    struct TimedLaunch {
        int kind;
        cudaEvent_t start, stop;
    };
    std::vector<TimedLaunch> timed;
};

namespace rn {
// Views per forward-projection CTA for nu channels (0 if nu is too large).
int fan_fp_views(int nu);
// Sets the dynamic shared-memory limits of the fan kernels on the current
// device (once per device).
int fan_kernel_attributes();
constexpr int kTimedKinds = 5;
// Brackets one kernel launch of `plan` on stream `st`: counts it and, when
// timing is enabled, records a start/stop event pair around it.
struct LaunchScope {
    rn_fan_plan* p;
    cudaStream_t st;
    int idx = -1;
    LaunchScope(rn_fan_plan* plan, cudaStream_t s, int kind) : p(plan), st(s) {
        p->launches++;
        if (p->timing) {
            rn_fan_plan::TimedLaunch t{kind, nullptr, nullptr};
            cudaEventCreate(&t.start);
            cudaEventCreate(&t.stop);
            cudaEventRecord(t.start, st);
            p->timed.push_back(t);
            idx = (int)p->timed.size() - 1;
        }
    }
    ~LaunchScope() {
        if (idx >= 0) cudaEventRecord(p->timed[idx].stop, st);
    }
};
// Host-side geometry tables of a fan plan, built by fan_build_geometry and
// uploaded with the rest of the plan.
struct FanGeoHost {
    std::vector<ViewGeo> views;
    std::vector<double2> vcs;       // per view (cos theta, sin theta)
    std::vector<int> vx;            // per view: 1 for the X class
    std::vector<int> perm;          // class-sorted view order per set
    std::vector<double2> esc;       // per detector edge (sin, cos) of its fan angle
    std::vector<double2> csc;       // per cell centre (sin, cos); entry nu one spacing on
    std::vector<float2> cell;       // per cell (cos a_u, sin a_u)
};
// Fills the host tables and the line padding of p->dims (no device work).
int fan_build_geometry(rn_fan_plan* p, const float* host_deg, FanGeoHost& gh);
// Device slope tables d_edges / d_cslopes from the uploaded per-view and
// per-edge terms.
int fan_slope_tables(rn_fan_plan* p, const double2* d_vcs, const int* d_vx, const double2* d_esc,
                     const double2* d_csc, cudaStream_t st);
// Parts over which fan_backproject splits a backprojection of `type` (1 when
// it does not split), and the number of slices in its first launch.
int fan_bp_split(const rn_fan_plan* p, int type, int* first_wave_slices);
// Most lines per staged forward-projection chunk that shared memory holds.
int fan_fp_lines_max(const rn_fan_plan* p);
int fan_project(rn_fan_plan* p, float* d_prj, const float* d_img, cudaStream_t st, bool siddon = false);
int fan_backproject(rn_fan_plan* p, float* d_img, const float* d_prj, int type, int accumulate, cudaStream_t st);
}  // namespace rn
