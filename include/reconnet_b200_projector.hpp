/*
 * reconnet_b200 -- C++ projector classes with the reference's class-level
 * interface (header-only, over the C ABI of reconnet_b200.h).
 *
 * Mirrors ReconNet4D/Projector.h:8-63 (Projector: geometry fields, Setup,
 * SetCudaStream, virtual Projection / Backprojection on device pointers) and
 * ReconNet4D/DistanceDriven.h:3-30 (DistanceDrivenFan, DistanceDrivenTomo):
 * same class, member and method names, same argument order and meaning.
 *
 *  - pcuImg / pcuPrj / pcuDeg / pcuDetCenter / pcuSrc are device pointers in
 *    the reference layouts ([B][nx][ny][nz][C] images, [B][nu][nview][nv][C]
 *    sinograms, nview angles in radians, [nview][3] tomosynthesis vectors).
 *  - DistanceDrivenFan::Projection overwrites pcuPrj; Backprojection adds to
 *    pcuImg (DistanceDriven.cu:500-614 accumulates; callers zero the image).
 *  - DistanceDrivenTomo::BackprojectionTomo overwrites pcuImg and keeps the
 *    reference's view-0-only length pre-weight (DistanceDriven3D.cu:612-621).
 *  - Like the reference (DistanceDriven.cu:291-318), the fan projector reads
 *    the angles back to the host to split views by class; the geometry tables
 *    are rebuilt only when the geometry or the angles change, so repeated calls
 *    with the same views allocate nothing.
 *  - Errors throw std::runtime_error carrying rn_last_error(), where the
 *    reference throws its own exceptions.
 *  - typeProjector: 0 iterative, 1 FBP weighting (as the reference), 2 the
 *    matched transpose of the forward projector.
 */
#pragma once

#include <cuda_runtime_api.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "reconnet_b200.h"

namespace reconnet_b200 {

inline void throw_if(int status) {
    if (status != RN_OK) throw std::runtime_error(std::string("reconnet_b200: ") + rn_last_error());
}

class Projector {
public:
    int nBatches = 1, nChannels = 1;
    int nx = 0, ny = 0, nz = 1;
    float dx = 1, dy = 1, dz = 1;
    float cx = 0, cy = 0, cz = 0;
    int nu = 0, nview = 0, nv = 1;
    float du = 1, dv = 1, off_u = 0, off_v = 0;
    float dsd = 0, dso = 0;
    int typeProjector = 0;

    void Setup(int nBatches_, int nChannels_, int nx_, int ny_, int nz_, float dx_, float dy_, float dz_, int nu_,
               int nview_, int nv_, float du_, float dv_, float off_u_, float off_v_, float dsd_, float dso_,
               int typeProjector_ = 0) {
        Setup(nBatches_, nChannels_, nx_, ny_, nz_, dx_, dy_, dz_, 0.f, 0.f, 0.f, nu_, nview_, nv_, du_, dv_, off_u_,
              off_v_, dsd_, dso_, typeProjector_);
    }

    void Setup(int nBatches_, int nChannels_, int nx_, int ny_, int nz_, float dx_, float dy_, float dz_, float cx_,
               float cy_, float cz_, int nu_, int nview_, int nv_, float du_, float dv_, float off_u_, float off_v_,
               float dsd_, float dso_, int typeProjector_ = 0) {
        nBatches = nBatches_;
        nChannels = nChannels_;
        nx = nx_;
        ny = ny_;
        nz = nz_;
        dx = dx_;
        dy = dy_;
        dz = dz_;
        cx = cx_;
        cy = cy_;
        cz = cz_;
        nu = nu_;
        nview = nview_;
        nv = nv_;
        du = du_;
        dv = dv_;
        off_u = off_u_;
        off_v = off_v_;
        dsd = dsd_;
        dso = dso_;
        typeProjector = typeProjector_;
    }

    void SetCudaStream(const cudaStream_t& stream) { m_stream = stream; }

    virtual void Projection(const float* /*pcuImg*/, float* /*pcuPrj*/, const float* /*pcuDeg*/) {}
    virtual void Backprojection(float* /*pcuImg*/, const float* /*pcuPrj*/, const float* /*pcuDeg*/) {}

    Projector() = default;
    virtual ~Projector() = default;
    Projector(const Projector&) = delete;
    Projector& operator=(const Projector&) = delete;

protected:
    cudaStream_t m_stream = nullptr;

    RnFanGeom geom() const {
        RnFanGeom g;
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
        g.dsd = dsd;
        g.dso = dso;
        return g;
    }
};

class DistanceDrivenFan : public Projector {
public:
    DistanceDrivenFan() : Projector() {}
    ~DistanceDrivenFan() override {
        if (m_plan) rn_fan_plan_destroy(m_plan);
    }

    void Projection(const float* pcuImg, float* pcuPrj, const float* pcuDeg) override {
        throw_if(rn_fan_project(plan_for(pcuDeg), pcuPrj, pcuImg, m_stream));
    }

    void Backprojection(float* pcuImg, const float* pcuPrj, const float* pcuDeg) override {
        throw_if(rn_fan_backproject(plan_for(pcuDeg), pcuImg, pcuPrj, typeProjector, /*accumulate=*/1, m_stream));
    }

private:
    rn_fan_plan* m_plan = nullptr;
    RnFanGeom m_geom{};
    std::vector<float> m_deg;

    rn_fan_plan* plan_for(const float* pcuDeg) {
        if (nview <= 0) throw std::runtime_error("reconnet_b200: Setup() has not been called");
        std::vector<float> deg((size_t)nview);
        if (cudaMemcpyAsync(deg.data(), pcuDeg, sizeof(float) * deg.size(), cudaMemcpyDeviceToHost, m_stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(m_stream) != cudaSuccess)
            throw std::runtime_error("reconnet_b200: cannot read the view angles");
        const RnFanGeom g = geom();
        if (m_plan && deg == m_deg && std::memcmp(&g, &m_geom, sizeof(g)) == 0) return m_plan;
        if (m_plan) {
            rn_fan_plan_destroy(m_plan);
            m_plan = nullptr;
        }
        throw_if(rn_fan_plan_create(&m_plan, &g, deg.data(), m_stream));
        m_geom = g;
        m_deg.swap(deg);
        return m_plan;
    }
};

class DistanceDrivenTomo : public Projector {
public:
    DistanceDrivenTomo() : Projector() {}
    ~DistanceDrivenTomo() override {
        if (m_sat) cudaFree(m_sat);
    }

    void ProjectionTomo(const float* pcuImg, float* pcuPrj, const float* pcuDetCenter, const float* pcuSrc) {
        size_t fp = 0, bp = 0;
        throw_if(rn_tomo_sat_bytes(nx, ny, nz, nu, nview, nv, &fp, &bp));
        throw_if(rn_tomo_project(pcuPrj, pcuImg, pcuDetCenter, pcuSrc, scratch(fp), nBatches, nChannels, nx, ny, nz,
                                 dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v, m_stream));
    }

    void BackprojectionTomo(float* pcuImg, const float* pcuPrj, const float* pcuDetCenter, const float* pcuSrc) {
        size_t fp = 0, bp = 0;
        throw_if(rn_tomo_sat_bytes(nx, ny, nz, nu, nview, nv, &fp, &bp));
        throw_if(rn_tomo_backproject(pcuImg, pcuPrj, pcuDetCenter, pcuSrc, scratch(bp), nBatches, nChannels, nx, ny,
                                     nz, dx, dy, dz, cx, cy, cz, nu, nview, nv, du, dv, off_u, off_v,
                                     /*weightAllViews=*/0, m_stream));
    }

private:
    double* m_sat = nullptr;
    size_t m_sat_bytes = 0;

    double* scratch(size_t bytes) {
        if (bytes > m_sat_bytes) {
            if (m_sat) cudaFree(m_sat);
            m_sat = nullptr;
            m_sat_bytes = 0;
            if (cudaMalloc((void**)&m_sat, bytes) != cudaSuccess)
                throw std::runtime_error("reconnet_b200: cannot allocate the summed-area-table scratch");
            m_sat_bytes = bytes;
        }
        return m_sat;
    }
};

}  // namespace reconnet_b200
