// Checks the header-only projector classes (include/reconnet_b200_projector.hpp)
// against the plain C ABI on the GPU: DistanceDrivenFan::Projection must equal
// rn_fan_project, Backprojection must add rn_fan_backproject's result to the
// image (called twice: twice the result), a changed angle set must rebuild the
// tables, and DistanceDrivenTomo must equal rn_tomo_project / _backproject.
// Exit status 0 on success.
#include <cuda_runtime_api.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "reconnet_b200_projector.hpp"

static std::vector<float> seq(size_t n, unsigned seed) {
    std::vector<float> v(n);
    unsigned s = seed;
    for (auto& x : v) {
        s = s * 1664525u + 1013904223u;
        x = (float)((s >> 8) & 0xffff) / 65536.0f;
    }
    return v;
}

template <class T>
static T* dev(const std::vector<T>& h) {
    T* d = nullptr;
    cudaMalloc((void**)&d, sizeof(T) * h.size());
    cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return d;
}

static std::vector<float> host(const float* d, size_t n) {
    std::vector<float> h(n);
    cudaMemcpy(h.data(), d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    return h;
}

static double maxdiff(const std::vector<float>& a, const std::vector<float>& b, float scale_b = 1.f) {
    double m = 0;
    for (size_t i = 0; i < a.size(); i++) m = std::fmax(m, std::fabs((double)a[i] - (double)scale_b * b[i]));
    return m;
}

int main() {
    using namespace reconnet_b200;
    int fails = 0;
    // ---- fan ----
    const int B = 2, C = 1, nx = 48, ny = 40, nz = 1, nu = 64, nview = 36, nv = 1;
    const float dx = 1.f, dy = 1.1f, dz = 1.f, da = 0.0025f, dv = 1.f, dsd = 1085.6f, dso = 595.f;
    std::vector<float> deg(nview), deg2(nview);
    for (int i = 0; i < nview; i++) {
        deg[i] = (float)(2 * M_PI * i / nview);
        deg2[i] = deg[i] + 0.01f;
    }
    const size_t ni = (size_t)B * nx * ny * nz * C, np = (size_t)B * nu * nview * nv * C;
    float* d_img = dev(seq(ni, 1));
    float* d_prj = dev(seq(np, 2));
    float* d_deg = dev(deg);
    float* d_deg2 = dev(deg2);
    float *d_out, *d_ref;
    cudaMalloc((void**)&d_out, sizeof(float) * std::max(ni, np));
    cudaMalloc((void**)&d_ref, sizeof(float) * std::max(ni, np));

    RnFanGeom g = {B, C, nx, ny, nz, dx, dy, dz, 0, 0, 0, nu, nview, nv, da, dv, 0, 0, dsd, dso};
    for (int type = 0; type < 3; type++) {
        DistanceDrivenFan fan;
        fan.Setup(B, C, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, 0.f, 0.f, dsd, dso, type);
        cudaStream_t st;
        cudaStreamCreate(&st);
        fan.SetCudaStream(st);
        for (int pass = 0; pass < 2; pass++) {   // pass 1: other angles, tables rebuilt
            const float* dd = pass ? d_deg2 : d_deg;
            rn_fan_plan* plan = nullptr;
            throw_if(rn_fan_plan_create(&plan, &g, pass ? deg2.data() : deg.data(), st));
            fan.Projection(d_img, d_out, dd);
            throw_if(rn_fan_project(plan, d_ref, d_img, st));
            cudaStreamSynchronize(st);
            double e = maxdiff(host(d_out, np), host(d_ref, np));
            if (e != 0) {
                std::printf("fan type %d pass %d: Projection differs by %g\n", type, pass, e);
                fails++;
            }
            cudaMemsetAsync(d_out, 0, sizeof(float) * ni, st);
            fan.Backprojection(d_out, d_prj, dd);
            fan.Backprojection(d_out, d_prj, dd);
            throw_if(rn_fan_backproject(plan, d_ref, d_prj, type, 0, st));
            cudaStreamSynchronize(st);
            e = maxdiff(host(d_out, ni), host(d_ref, ni), 2.f);
            if (e > 1e-5) {
                std::printf("fan type %d pass %d: two Backprojections differ from 2x by %g\n", type, pass, e);
                fails++;
            }
            rn_fan_plan_destroy(plan);
        }
        cudaStreamDestroy(st);
    }

    // ---- tomosynthesis ----
    const int tnx = 24, tny = 20, tnz = 6, tnu = 32, tnv = 28, tview = 5;
    std::vector<float> det(3 * tview), src(3 * tview);
    for (int i = 0; i < tview; i++) {
        float a = (i - 2) * 0.15f;
        src[3 * i] = 600.f * std::sin(a);
        src[3 * i + 1] = 10.f;
        src[3 * i + 2] = 600.f * std::cos(a);
        det[3 * i] = 0.f;
        det[3 * i + 1] = 0.f;
        det[3 * i + 2] = -40.f;
    }
    const size_t ti = (size_t)tnx * tny * tnz, tp = (size_t)tnu * tview * tnv;
    float* t_img = dev(seq(ti, 3));
    float* t_prj = dev(seq(tp, 4));
    float* t_det = dev(det);
    float* t_src = dev(src);
    DistanceDrivenTomo tomo;
    tomo.Setup(1, 1, tnx, tny, tnz, 1.f, 1.f, 2.f, 0.f, 0.f, 0.f, tnu, tview, tnv, 1.5f, 1.5f, 0.2f, -0.3f, 0.f, 0.f);
    size_t fpb = 0, bpb = 0;
    throw_if(rn_tomo_sat_bytes(tnx, tny, tnz, tnu, tview, tnv, &fpb, &bpb));
    double* sat = nullptr;
    cudaMalloc((void**)&sat, std::max(fpb, bpb));
    tomo.ProjectionTomo(t_img, d_out, t_det, t_src);
    throw_if(rn_tomo_project(d_ref, t_img, t_det, t_src, sat, 1, 1, tnx, tny, tnz, 1.f, 1.f, 2.f, 0.f, 0.f, 0.f, tnu,
                             tview, tnv, 1.5f, 1.5f, 0.2f, -0.3f, nullptr));
    cudaDeviceSynchronize();
    double e = maxdiff(host(d_out, tp), host(d_ref, tp));
    if (e != 0) {
        std::printf("tomo: ProjectionTomo differs by %g\n", e);
        fails++;
    }
    tomo.BackprojectionTomo(d_out, t_prj, t_det, t_src);
    throw_if(rn_tomo_backproject(d_ref, t_prj, t_det, t_src, sat, 1, 1, tnx, tny, tnz, 1.f, 1.f, 2.f, 0.f, 0.f, 0.f,
                                 tnu, tview, tnv, 1.5f, 1.5f, 0.2f, -0.3f, 0, nullptr));
    cudaDeviceSynchronize();
    e = maxdiff(host(d_out, ti), host(d_ref, ti));
    if (e != 0) {
        std::printf("tomo: BackprojectionTomo differs by %g\n", e);
        fails++;
    }

    // ---- errors throw ----
    bool threw = false;
    try {
        DistanceDrivenFan bad;
        bad.Setup(1, 1, 0, 0, 1, 1.f, 1.f, 1.f, 64, 4, 1, da, 1.f, 0.f, 0.f, dsd, dso);
        bad.Projection(d_img, d_out, d_deg);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    if (!threw) {
        std::printf("invalid geometry did not throw\n");
        fails++;
    }
    std::printf(fails ? "FAILED %d\n" : "OK\n", fails);
    return fails ? 1 : 0;
}
