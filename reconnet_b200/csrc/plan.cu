// Plan construction for the fan projector and the native device API.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "rn_internal.h"

namespace rn {

// ---------------------------------------------------------------------------
// Error state.
// ---------------------------------------------------------------------------
static thread_local std::string t_err;
static thread_local int t_status = RN_OK;

int set_error(int code, const std::string& msg) {
    t_status = code;
    t_err = msg;
    return code;
}

int set_cuda_error(cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? RN_ERR_ALLOC : RN_ERR_CUDA;
    return set_error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

void clear_error() {
    t_status = RN_OK;
    t_err.clear();
}

// Scratch budgets (bytes) for line buffers and edge tables; slices beyond the
// budget are processed in waves.
static const long long kLineBudget = 4ll << 30;
static const long long kTableBudget = 4ll << 30;

static int validate(const RnFanGeom* g) {
    if (!g) return set_error(RN_ERR_ARG, "null geometry");
    if (g->nBatches <= 0 || g->nChannels <= 0 || g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->nu <= 0 ||
        g->nview <= 0 || g->nv <= 0)
        return set_error(RN_ERR_ARG, "geometry sizes must be positive");
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0 && g->du > 0 && g->dv > 0 && g->dsd > 0 && g->dso > 0))
        return set_error(RN_ERR_ARG, "pixel sizes, detector pitch and distances must be positive");
    if (g->nx >= (1 << 15) || g->ny >= (1 << 15))
        return set_error(RN_ERR_ARG, "image too large (at most 32767 pixels per side)");
    if (fan_fp_views(g->nu) < 1)
        return set_error(RN_ERR_ARG, "too many detector channels for the forward projector");
    return RN_OK;
}

static void set_dims(rn_fan_plan* p, long long isx, long long isy) {
    const RnFanGeom& g = p->g;
    FanDims& d = p->dims;
    d.nx = g.nx;
    d.ny = g.ny;
    d.nu = g.nu;
    d.dx = g.dx;
    d.dy = g.dy;
    d.du = g.du;
    d.off_u = g.off_u;
    d.dsd = g.dsd;
    d.dso = g.dso;
    d.margin = 0;            // set with the geometry tables (fan_build_geometry)
    d.lpx = g.nx + 1;
    d.lpy = g.ny + 1;
    d.spx = line_stride(d.lpx);
    d.spy = line_stride(d.lpy);
    d.isx = isx;
    d.isy = isy;
}

static void build_fp_work(rn_fan_plan* p) {
    // views per work item: at most the kernel's table capacity, fewer when a
    // small batch would leave SMs idle (one CTA per SM; aim for two waves),
    // or the tuned count.  A ray's sum does not depend on which views share
    // its CTA.
    const int vmax = fan_fp_views(p->g.nu);
    int VT = vmax;
    auto items = [&](int vt) {
        long long n = 0;
        for (size_t s = 0; s < p->h_fp.size(); s++) {
            const GeoSet& gs = p->h_sets[p->h_fp[s].set];
            n += (gs.nxv + vt - 1) / vt + (gs.nview - gs.nxv + vt - 1) / vt;
        }
        return n;
    };
    if (p->fp_vt > 0) VT = std::min(p->fp_vt, vmax);
    else
        while (VT > 1 && items(VT) < 2LL * 148) VT--;
    p->fp_vt_used = VT;
    p->h_fp_work.clear();
    for (size_t s = 0; s < p->h_fp.size(); s++) {
        const GeoSet& gs = p->h_sets[p->h_fp[s].set];
        for (int k = 0; k < gs.nxv; k += VT) {
            int w[4] = {(int)s, 1, k, std::min(VT, gs.nxv - k)};
            p->h_fp_work.insert(p->h_fp_work.end(), w, w + 4);
        }
        int ny_ = gs.nview - gs.nxv;
        for (int k = 0; k < ny_; k += VT) {
            int w[4] = {(int)s, 0, gs.nxv + k, std::min(VT, ny_ - k)};
            p->h_fp_work.insert(p->h_fp_work.end(), w, w + 4);
        }
    }
    p->n_fp_work = (int)(p->h_fp_work.size() / 4);
    // Within each wave of slices that share the line scratch, items with more
    // views go first: the block scheduler hands out CTAs in index order, so
    // the short items fill the last wave instead of trailing it (a longest-
    // processing-time-first list schedule).  The order within equal view
    // counts stays by slice, so CTAs running together read the same slices'
    // lines.
    const int slots = (int)std::max<long long>(1, p->fp_slots);
    int* w = p->h_fp_work.data();
    for (int b = 0; b < p->n_fp_work;) {
        const int s_end = (w[4 * b] / slots + 1) * slots;   // the wave of fan_project holding item b
        int e = b;
        while (e < p->n_fp_work && w[4 * e] < s_end) e++;
        std::vector<int4> wave(e - b);
        for (int i = b; i < e; i++) wave[i - b] = make_int4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
        std::stable_sort(wave.begin(), wave.end(), [](const int4& x, const int4& y) { return x.w > y.w; });
        for (int i = b; i < e; i++) {
            w[4 * i] = wave[i - b].x;
            w[4 * i + 1] = wave[i - b].y;
            w[4 * i + 2] = wave[i - b].z;
            w[4 * i + 3] = wave[i - b].w;
        }
        b = e;
    }
}

// Table window (entries per view staged by the BP kernels): the detector
// extent, in cells, of a tw x th-pixel tile at the point closest to the source.
static int table_window(const RnFanGeom& g, int tw, int th) {
    double diag = std::sqrt((double)tw * tw * g.dx * g.dx + (double)th * th * g.dy * g.dy);
    double hx = g.nx * g.dx / 2.0 + std::fabs(g.cx), hy = g.ny * g.dy / 2.0 + std::fabs(g.cy);
    double dmin = g.dso - std::sqrt(hx * hx + hy * hy);
    if (dmin <= 0) return -1;
    double w = diag / (dmin * g.du) + 8;
    int win = (int)std::ceil(w);
    win = (win + 7) & ~7;
    return std::min(win, g.nu + 2);
}

// ---------------------------------------------------------------------------
// Plan memory.  All tables and scratch of a plan share one device allocation,
// filled by one upload.  A destroyed plan's allocation is kept for the next
// plan on that device (one per device, at most kArenaKeepBytes), so a plan
// rebuilt for new angles (the host entry points do this whenever the angles
// change) calls neither cudaMalloc nor cudaFree.
// ---------------------------------------------------------------------------
static const size_t kArenaKeepBytes = 256ull << 20;
struct KeptArena {
    void* ptr = nullptr;
    size_t bytes = 0;
};
static std::mutex g_arena_mu;
static std::vector<KeptArena> g_kept;   // indexed by device

static int arena_acquire(int dev, size_t bytes, void** out, size_t* got) {
    void* stale = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        if ((int)g_kept.size() > dev && g_kept[dev].ptr) {
            if (g_kept[dev].bytes >= bytes) {
                *out = g_kept[dev].ptr;
                *got = g_kept[dev].bytes;
                g_kept[dev] = KeptArena();
                return RN_OK;
            }
            stale = g_kept[dev].ptr;   // too small for this plan
            g_kept[dev] = KeptArena();
        }
    }
    if (stale) cudaFree(stale);
    RN_CUDA_TRY(cudaMalloc(out, bytes));
    *got = bytes;
    return RN_OK;
}

// The caller has synchronised the device: no launch still reads `ptr`.
static void arena_release(int dev, void* ptr, size_t bytes) {
    if (!ptr) return;
    if (bytes > kArenaKeepBytes || dev < 0) {
        cudaFree(ptr);
        return;
    }
    void* old = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        if ((int)g_kept.size() <= dev) g_kept.resize(dev + 1);
        old = g_kept[dev].ptr;
        g_kept[dev].ptr = ptr;
        g_kept[dev].bytes = bytes;
    }
    if (old) cudaFree(old);
}

// One region of the plan allocation; `src` (when set) is uploaded into it.
struct ArenaPart {
    void** dst;
    size_t bytes;
    const void* src;
    size_t src_bytes;
};

static int finish_plan(rn_fan_plan* p, const float* host_deg, cudaStream_t st) {
    const RnFanGeom& g = p->g;
    const int win_m = table_window(g, kBmCols, kBmTileY);
    if (win_m < 0) return set_error(RN_ERR_ARG, "fan geometry: the image reaches the source");
    if (win_m > 800) return set_error(RN_ERR_ARG, "fan geometry: backprojection tile window too large");
    p->table_win_m = win_m;
    RN_TRY(fan_kernel_attributes());
    FanGeoHost gh;
    RN_TRY(fan_build_geometry(p, host_deg, gh));
    // line scratch: slices whose lines fit the budget form one wave of FP work
    p->line_slot_elems = (long long)p->dims.ny * p->dims.spx + (long long)p->dims.nx * p->dims.spy;
    p->fp_slots = std::max(1ll, std::min((long long)p->h_fp.size(),
                                         kLineBudget / (p->line_slot_elems * (long long)(sizeof(float2) + sizeof(float)))));
    build_fp_work(p);
    {
        long long cap = 0;   // one view per item: room for any tuning
        for (size_t s = 0; s < p->h_fp.size(); s++) cap += p->h_sets[p->h_fp[s].set].nview;
        p->fp_work_cap = (int)std::max<long long>(cap, p->n_fp_work);
    }

    // table scratch: all slices if within budget, else at least the largest slice
    long long need = 0, largest = 0;
    for (const BpSlice& b : p->h_bp) {
        long long n = (long long)p->h_sets[b.set].nview * (g.nu + 2);
        need = std::max(need, b.table_off + n);
        largest = std::max(largest, n);
    }
    p->tab_elems = std::max(largest, std::min(need, kTableBudget / (long long)sizeof(float4)));
    // partial images of a split backprojection: the most any type asks for
    long long parts = 1;
    for (int type : {RN_TYPE_ITERATIVE, RN_TYPE_MATCHED, RN_TYPE_SIDDON})
        parts = std::max<long long>(parts, fan_bp_split(p, type, nullptr));
    p->bp_parts_cap = parts > 1 ? parts * p->img_elems : 0;

    const long long V = p->total_views, nu = g.nu;
    double2 *d_vcs = nullptr, *d_esc = nullptr, *d_csc = nullptr;
    int* d_vx = nullptr;
    std::vector<ArenaPart> up, dev;
    auto upload = [&](auto** dst, const auto& vec) {
        const size_t n = vec.size() * sizeof(vec[0]);
        up.push_back(ArenaPart{reinterpret_cast<void**>(dst), std::max<size_t>(n, 16), vec.data(), n});
    };
    auto device = [&](auto** dst, size_t bytes) {
        dev.push_back(ArenaPart{reinterpret_cast<void**>(dst), std::max<size_t>(bytes, 16), nullptr, 0});
    };
    upload(&p->d_views, gh.views);
    upload(&p->d_cell, gh.cell);
    upload(&p->d_perm, gh.perm);
    upload(&p->d_sets, p->h_sets);
    upload(&p->d_fp, p->h_fp);
    upload(&p->d_bp, p->h_bp);
    upload(&p->d_bpr, p->h_bpr);
    upload(&p->d_fps, p->h_fps);
    upload(&p->d_bps, p->h_bps);
    up.push_back(ArenaPart{reinterpret_cast<void**>(&p->d_fp_work), sizeof(int4) * (size_t)std::max(1, p->fp_work_cap),
                           p->h_fp_work.data(), sizeof(int) * p->h_fp_work.size()});
    upload(&d_vcs, gh.vcs);
    upload(&d_vx, gh.vx);
    upload(&d_esc, gh.esc);
    upload(&d_csc, gh.csc);
    device(&p->d_err, sizeof(int));
    device(&p->d_edges, sizeof(double) * V * (nu + 1));
    device(&p->d_cslopes, sizeof(double) * V * (nu + 1));
    device(&p->d_hl, sizeof(float2) * p->fp_slots * p->line_slot_elems);
    device(&p->d_la, sizeof(float) * p->fp_slots * p->line_slot_elems);
    device(&p->d_tab, sizeof(float4) * p->tab_elems);
    if (p->bp_parts_cap > 0) device(&p->d_bp_parts, sizeof(float) * p->bp_parts_cap);
    // residual and backprojection scratch of the SQS step and the autotuner:
    // part of the plan, so a step never allocates
    device(&p->d_tmp_prj, sizeof(float) * (size_t)p->prj_elems);
    device(&p->d_tmp_img, sizeof(float) * (size_t)p->img_elems);

    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t upload_bytes = 0;
    for (const ArenaPart& a : up) upload_bytes = align(upload_bytes + a.bytes);
    size_t total = upload_bytes;
    for (const ArenaPart& a : dev) total = align(total + a.bytes);
    RN_TRY(arena_acquire(p->device, total, &p->d_arena, &p->arena_bytes));
    std::vector<unsigned char> blob(upload_bytes, 0);
    size_t off = 0;
    for (const ArenaPart& a : up) {
        *a.dst = static_cast<unsigned char*>(p->d_arena) + off;
        if (a.src_bytes) memcpy(blob.data() + off, a.src, a.src_bytes);
        off = align(off + a.bytes);
    }
    for (const ArenaPart& a : dev) {
        *a.dst = static_cast<unsigned char*>(p->d_arena) + off;
        off = align(off + a.bytes);
    }
    RN_CUDA_TRY(cudaMemcpyAsync(p->d_arena, blob.data(), upload_bytes, cudaMemcpyHostToDevice, st));
    RN_CUDA_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
    RN_TRY(fan_slope_tables(p, d_vcs, d_vx, d_esc, d_csc, st));
    RN_CUDA_TRY(cudaStreamSynchronize(st));   // blob and gh go out of scope
    return RN_OK;
}

// ---------------------------------------------------------------------------
// Launch-parameter tuning: views per forward-projection work item, lines per
// staged chunk, and the view split of a single-launch backprojection.  Tuned
// choices are cached by a hash of the geometry, the per-slice view counts and
// classes, and the projector type.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::unordered_map<uint64_t, std::vector<int>> g_tuned;

static uint64_t tune_key(const rn_fan_plan* p, int type) {
    uint64_t h = 1469598103934665603ull;   // FNV-1a
    auto mix = [&](const void* d, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(d);
        for (size_t i = 0; i < n; i++) {
            h ^= c[i];
            h *= 1099511628211ull;
        }
    };
    const int ragged = p->ragged ? 1 : 0;
    mix(&p->g, sizeof(p->g));
    mix(&ragged, sizeof(ragged));
    mix(&type, sizeof(type));
    for (const GeoSet& gs : p->h_sets) {
        mix(&gs.nview, sizeof(gs.nview));
        mix(&gs.nxv, sizeof(gs.nxv));
    }
    return h;
}

// Sets the overrides and uploads the rebuilt work list (stream-ordered).
static int apply_tuning(rn_fan_plan* p, int fp_vt, int fp_R, int bp_nparts, cudaStream_t st) {
    p->fp_vt = fp_vt;
    p->fp_R = fp_R;
    p->bp_nparts = bp_nparts;
    build_fp_work(p);
    if (p->n_fp_work > p->fp_work_cap) return set_error(RN_ERR_ARG, "tuning: work list exceeds its capacity");
    if (p->n_fp_work > 0)
        RN_CUDA_TRY(cudaMemcpyAsync(p->d_fp_work, p->h_fp_work.data(), sizeof(int4) * p->n_fp_work,
                                    cudaMemcpyHostToDevice, st));
    return RN_OK;
}

}  // namespace rn

using namespace rn;

extern "C" {

const char* rn_last_error(void) { return rn::t_err.c_str(); }
int rn_last_status(void) { return rn::t_status; }
int rn_version(void) { return 1; }

int rn_fan_plan_destroy(rn_fan_plan* p) {
    if (!p) return RN_OK;
    if (p->d_arena) {
        // as cudaFree would, wait until no launch on the device still reads
        // the plan; after an error keep nothing
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != p->device) cudaSetDevice(p->device);
        if (cudaDeviceSynchronize() == cudaSuccess) arena_release(p->device, p->d_arena, p->arena_bytes);
        else cudaFree(p->d_arena);
        if (cur >= 0 && cur != p->device) cudaSetDevice(cur);
    }
    for (auto& t : p->timed) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    delete p;
    return RN_OK;
}

int rn_fan_plan_create(rn_fan_plan** out, const RnFanGeom* g, const float* host_deg, void* stream) {
    clear_error();
    if (!out || !host_deg) return set_error(RN_ERR_ARG, "null argument");
    *out = nullptr;
    RN_TRY(validate(g));
    cudaStream_t st = (cudaStream_t)stream;
    rn_fan_plan* p = new rn_fan_plan();
    p->g = *g;
    p->ragged = false;
    cudaGetDevice(&p->device);
    const int B = g->nBatches, C = g->nChannels, nx = g->nx, ny = g->ny, nz = g->nz, nu = g->nu, nview = g->nview,
              nv = g->nv;
    set_dims(p, (long long)ny * nz * C, (long long)nz * C);
    p->total_views = nview;
    p->h_sets.push_back(GeoSet{0, nview, 0});
    const long long img_b = (long long)nx * ny * nz * C, prj_b = (long long)nu * nview * nv * C;
    p->img_elems = img_b * B;
    p->prj_elems = prj_b * B;

    // FP slices (b, iv, c): image planes mixed at the z texture coordinate of
    // detector row iv (DistanceDriven.cu:86,99; texel-centre convention, border).
    std::vector<std::vector<std::pair<int, float>>> zmix(nv);
    for (int iv = 0; iv < nv; iv++) {
        double z = (iv - (nv - 1) / 2.0 + g->off_v) * g->dv;
        double zc = (z - g->cz) / g->dz + nz / 2.0;
        double zb = zc - 0.5;
        double z0 = std::floor(zb);
        double wz = zb - z0;
        for (int k = 0; k < 2; k++) {
            int zi = (int)z0 + k;
            float w = (float)(k ? wz : 1.0 - wz);
            if (zi >= 0 && zi < nz && w != 0.f) zmix[iv].push_back({zi, w});
        }
    }
    for (int b = 0; b < B; b++)
        for (int iv = 0; iv < nv; iv++)
            for (int c = 0; c < C; c++) {
                FpSlice f;
                memset(&f, 0, sizeof(f));
                for (size_t k = 0; k < zmix[iv].size(); k++) {
                    f.img_off[k] = b * img_b + (long long)zmix[iv][k].first * C + c;
                    f.img_w[k] = zmix[iv][k].second;
                }
                f.prj_off = b * prj_b + (long long)iv * C + c;
                f.su = nview * nv * C;
                f.sview = nv * C;
                f.set = 0;
                f.line_slot = 0;
                p->h_fp.push_back(f);
            }
    // matched BP slices (b, z, c): transpose of the z mixing above
    std::vector<std::vector<std::pair<int, float>>> zin(nz);
    for (int iv = 0; iv < nv; iv++)
        for (auto& t : zmix[iv]) zin[t.first].push_back({iv, t.second});
    // reference BP slices (b, iz, c): sinogram rows mixed at ivf + 0.5
    // (DistanceDriven.cu:518,543; border addressing along v)
    std::vector<std::vector<std::pair<int, float>>> vmix(nz);
    for (int iz = 0; iz < nz; iz++) {
        double ivf = (iz - (nz - 1) / 2.0) * g->dz / g->dv + g->off_v + (nv - 1.0) / 2.0;
        double v0 = std::floor(ivf);
        double wv = ivf - v0;
        for (int k = 0; k < 2; k++) {
            int vi = (int)v0 + k;
            float w = (float)(k ? wv : 1.0 - wv);
            if (vi >= 0 && vi < nv && w != 0.f) vmix[iz].push_back({vi, w});
        }
    }
    for (int iz = 0; iz < nz; iz++)
        if ((int)zin[iz].size() > kBpMix) {
            delete p;
            return set_error(RN_ERR_ARG, "fan geometry: more than 4 detector rows map onto one image slice");
        }
    long long toff = 0;
    for (int b = 0; b < B; b++)
        for (int z = 0; z < nz; z++)
            for (int c = 0; c < C; c++) {
                BpSlice m, r;
                memset(&m, 0, sizeof(m));
                memset(&r, 0, sizeof(r));
                m.img_off = r.img_off = b * img_b + (long long)z * C + c;
                for (size_t k = 0; k < zin[z].size(); k++) {
                    m.prj_off[k] = b * prj_b + (long long)zin[z][k].first * C + c;
                    m.prj_w[k] = zin[z][k].second;
                }
                for (size_t k = 0; k < vmix[z].size(); k++) {
                    r.prj_off[k] = b * prj_b + (long long)vmix[z][k].first * C + c;
                    r.prj_w[k] = vmix[z][k].second;
                }
                m.su = r.su = nview * nv * C;
                m.sview = r.sview = nv * C;
                m.set = r.set = 0;
                m.table_off = r.table_off = toff;
                toff += (long long)nview * (nu + 2);
                p->h_bp.push_back(m);
                p->h_bpr.push_back(r);
            }
    // Siddon slices: a ray at the height of detector row iv stays in image
    // slice floor(z) (it is parallel to the slices, Siddon.cu:22-60), none if
    // z falls outside [0, nz)
    std::vector<int> siz(nv, -1);
    std::vector<std::vector<int>> srows(nz);
    for (int iv = 0; iv < nv; iv++) {
        double z = (iv - (nv - 1) / 2.0 + g->off_v) * g->dv;
        double zc = (z - g->cz) / g->dz + nz / 2.0;
        if (zc >= 0 && zc < nz) {
            siz[iv] = std::min((int)std::floor(zc), nz - 1);
            srows[siz[iv]].push_back(iv);
        }
    }
    for (int iz = 0; iz < nz; iz++)
        if ((int)srows[iz].size() > kBpMix) {
            delete p;
            return set_error(RN_ERR_ARG, "fan geometry: more than 4 detector rows fall in one image slice (Siddon)");
        }
    for (int b = 0; b < B; b++)
        for (int iv = 0; iv < nv; iv++)
            for (int c = 0; c < C; c++) {
                FpSlice f = p->h_fp[((size_t)b * nv + iv) * C + c];
                memset(f.img_off, 0, sizeof(f.img_off));
                memset(f.img_w, 0, sizeof(f.img_w));
                if (siz[iv] >= 0) {
                    f.img_off[0] = b * img_b + (long long)siz[iv] * C + c;
                    f.img_w[0] = 1.f;
                }
                p->h_fps.push_back(f);
            }
    for (int b = 0; b < B; b++)
        for (int z = 0; z < nz; z++)
            for (int c = 0; c < C; c++) {
                BpSlice m = p->h_bp[((size_t)b * nz + z) * C + c];
                memset(m.prj_off, 0, sizeof(m.prj_off));
                memset(m.prj_w, 0, sizeof(m.prj_w));
                for (size_t k = 0; k < srows[z].size(); k++) {
                    m.prj_off[k] = b * prj_b + (long long)srows[z][k] * C + c;
                    m.prj_w[k] = 1.f;
                }
                p->h_bps.push_back(m);
            }
    int s = finish_plan(p, host_deg, st);
    if (s != RN_OK) {
        std::string msg = rn_last_error();
        rn_fan_plan_destroy(p);
        return set_error(s, msg);
    }
    *out = p;
    return RN_OK;
}

int rn_fan_plan_create_ragged(rn_fan_plan** out, const RnFanGeom* g, const int* nview_per_slice,
                              const float* host_deg, void* stream) {
    clear_error();
    if (!out || !host_deg || !nview_per_slice) return set_error(RN_ERR_ARG, "null argument");
    *out = nullptr;
    RnFanGeom gg = *g;
    gg.nz = gg.nv = gg.nChannels = 1;
    if (g->nz != 1 || g->nv != 1 || g->nChannels != 1)
        return set_error(RN_ERR_ARG, "ragged plans hold 2D slices: nz, nv and nChannels must be 1");
    long long total = 0;
    for (int s = 0; s < g->nBatches; s++) {
        if (nview_per_slice[s] <= 0) return set_error(RN_ERR_ARG, "every slice needs at least one view");
        total += nview_per_slice[s];
    }
    gg.nview = (int)std::min<long long>(total, 1 << 30);
    RN_TRY(validate(&gg));
    cudaStream_t st = (cudaStream_t)stream;
    rn_fan_plan* p = new rn_fan_plan();
    p->g = gg;
    p->ragged = true;
    cudaGetDevice(&p->device);
    const int S = g->nBatches, nx = g->nx, ny = g->ny, nu = g->nu;
    set_dims(p, ny, 1);
    p->total_views = total;
    p->img_elems = (long long)S * nx * ny;
    p->prj_elems = total * nu;
    int voff = 0;
    for (int s = 0; s < S; s++) {
        int nvs = nview_per_slice[s];
        p->h_sets.push_back(GeoSet{voff, nvs, 0});
        FpSlice f;
        memset(&f, 0, sizeof(f));
        f.img_off[0] = (long long)s * nx * ny;
        f.img_w[0] = 1.f;
        f.prj_off = (long long)nu * voff;
        f.su = nvs;
        f.sview = 1;
        f.set = s;
        p->h_fp.push_back(f);
        BpSlice b;
        memset(&b, 0, sizeof(b));
        b.img_off = (long long)s * nx * ny;
        b.prj_off[0] = (long long)nu * voff;
        b.prj_w[0] = 1.f;
        b.su = nvs;
        b.sview = 1;
        b.set = s;
        b.table_off = (long long)voff * (nu + 2);
        p->h_bp.push_back(b);
        p->h_bpr.push_back(b);
        p->h_fps.push_back(f);
        p->h_bps.push_back(b);
        voff += nvs;
    }
    int st2 = finish_plan(p, host_deg, st);
    if (st2 != RN_OK) {
        std::string msg = rn_last_error();
        rn_fan_plan_destroy(p);
        return set_error(st2, msg);
    }
    *out = p;
    return RN_OK;
}

int64_t rn_fan_plan_total_views(const rn_fan_plan* p) { return p ? p->total_views : 0; }

int rn_fan_project(rn_fan_plan* p, float* d_prj, const float* d_img, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    return rn::fan_project(p, d_prj, d_img, (cudaStream_t)stream);
}

int rn_fan_project_siddon(rn_fan_plan* p, float* d_prj, const float* d_img, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    return rn::fan_project(p, d_prj, d_img, (cudaStream_t)stream, true);
}

int rn_fan_backproject(rn_fan_plan* p, float* d_img, const float* d_prj, int type, int accumulate, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    if (type < 0 || type > 4) return set_error(RN_ERR_ARG, "typeProjector must be 0, 1, 2, 3 or 4");
    return rn::fan_backproject(p, d_img, d_prj, type, accumulate ? 1 : 0, (cudaStream_t)stream);
}

int rn_fan_plan_set_timing(rn_fan_plan* p, int enable) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    p->timing = enable != 0;
    return RN_OK;
}

int rn_fan_plan_read_timing(rn_fan_plan* p, float* ms, int* counts, int nkinds, long long* launches) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    for (int k = 0; k < nkinds; k++) {
        if (ms) ms[k] = 0.f;
        if (counts) counts[k] = 0;
    }
    if (launches) *launches = p->launches;
    if (nkinds <= 0) return RN_OK;   // launch count only; keep pending timings
    for (auto& t : p->timed) {
        float e = 0.f;
        if (cudaEventSynchronize(t.stop) == cudaSuccess && cudaEventElapsedTime(&e, t.start, t.stop) == cudaSuccess &&
            t.kind >= 0 && t.kind < nkinds) {
            if (ms) ms[t.kind] += e;
            if (counts) counts[t.kind] += 1;
        }
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    p->timed.clear();
    return RN_OK;
}

int rn_fan_plan_set_tuning(rn_fan_plan* p, int fp_views, int fp_lines, int bp_parts, void* stream) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    if (fp_views < 0 || fp_lines < 0 || bp_parts < 0 || bp_parts > kBpMaxParts)
        return set_error(RN_ERR_ARG, "tuning: negative value, or bp_parts above 16");
    // above their maxima the first two clamp (plans of one solver can differ
    // a little in how many lines fit)
    return apply_tuning(p, std::min(fp_views, fan_fp_views(p->g.nu)), std::min(fp_lines, fan_fp_lines_max(p)),
                        bp_parts, (cudaStream_t)stream);
}

int rn_fan_plan_get_tuning(const rn_fan_plan* p, int* fp_views, int* fp_lines, int* bp_parts) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    const int Rmax = fan_fp_lines_max(p);
    if (fp_views) *fp_views = p->fp_vt_used;
    if (fp_lines) *fp_lines = p->fp_R > 0 ? std::min(p->fp_R, Rmax) : Rmax;
    if (bp_parts) *bp_parts = p->bp_nparts;
    return RN_OK;
}

int rn_fan_plan_autotune(rn_fan_plan* p, float* d_prj, const float* d_img, int typeProjector, void* stream) {
    clear_error();
    if (!p || !d_prj || !d_img) return set_error(RN_ERR_ARG, "null argument");
    if (typeProjector < RN_TYPE_ITERATIVE || typeProjector > RN_TYPE_PIXEL)
        return set_error(RN_ERR_ARG, "autotune: unknown typeProjector");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t key = tune_key(p, typeProjector);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return apply_tuning(p, it->second[0], it->second[1], it->second[2], st);
    }
    const bool siddon = typeProjector == RN_TYPE_SIDDON;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RN_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_error(RN_ERR_CUDA, "autotune: cudaEventCreate");
    }
    // mean of two runs after one untimed run
    auto timed = [&](auto&& run, float& ms) -> int {
        RN_TRY(run());
        RN_CUDA_TRY(cudaEventRecord(e0, st));
        RN_TRY(run());
        RN_TRY(run());
        RN_CUDA_TRY(cudaEventRecord(e1, st));
        RN_CUDA_TRY(cudaEventSynchronize(e1));
        RN_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        ms *= 0.5f;
        return RN_OK;
    };
    int s = RN_OK;
    int best_vt = 0, best_R = 0, best_parts = 0;
    float best = 1e30f;
    const int vmax = fan_fp_views(p->g.nu), Rmax = fan_fp_lines_max(p);
    for (int vt = vmax; vt >= 1 && s == RN_OK; vt--) {
        for (int R : {Rmax, Rmax / 2}) {
            if (R < 1) continue;
            float ms = 0.f;
            s = apply_tuning(p, vt, R, 0, st);
            if (s == RN_OK) s = timed([&] { return fan_project(p, d_prj, d_img, st, siddon); }, ms);
            if (s != RN_OK) break;
            if (ms < best) {
                best = ms;
                best_vt = vt;
                best_R = R;
            }
        }
    }
    // the view split of the backprojection, where the plan can split it
    if (s == RN_OK && p->bp_parts_cap > 0) {
        best = 1e30f;
        for (int parts = 1; parts <= kBpMaxParts && s == RN_OK; parts *= 2) {
            if ((long long)parts * p->img_elems > p->bp_parts_cap && parts > 1) break;
            float ms = 0.f;
            s = apply_tuning(p, best_vt, best_R, parts, st);
            if (s == RN_OK)
                s = timed([&] { return fan_backproject(p, p->d_tmp_img, d_prj, typeProjector, 0, st); }, ms);
            if (s == RN_OK && ms < best) {
                best = ms;
                best_parts = parts;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != RN_OK) {
        const std::string msg = rn_last_error();
        apply_tuning(p, 0, 0, 0, st);
        return set_error(s, msg);
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = {best_vt, best_R, best_parts};
    }
    return apply_tuning(p, best_vt, best_R, best_parts, st);
}

int rn_fan_plan_set_spin_limit(rn_fan_plan* p, long long polls) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    if (polls < -1) return set_error(RN_ERR_ARG, "spin limit must be >= 0 (-1 restores the default)");
    p->spin_limit = polls == -1 ? kSpinLimit : polls;
    return RN_OK;
}

int rn_fan_plan_check(rn_fan_plan* p, void* stream) {
    clear_error();
    if (!p) return set_error(RN_ERR_ARG, "null plan");
    int h = 0;
    cudaStream_t st = (cudaStream_t)stream;
    RN_CUDA_TRY(cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    RN_CUDA_TRY(cudaStreamSynchronize(st));
    if (h != 0) {
        RN_CUDA_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
        return set_error(RN_ERR_TIMEOUT, "a device-side wait exceeded its spin limit");
    }
    return RN_OK;
}

}  // extern "C"
