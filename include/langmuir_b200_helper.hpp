// langmuir_b200_helper.hpp -- C++ drop-in for LangmuirCore::OpenClHelper.
//
// Header-only, over the C ABI of langmuir_b200.h.  It keeps the reference
// helper's method names and semantics (src/langmuirCore/include/openclhelper.h:22-241,
// openclhelper.cpp:17-583) so the engine's call sites stay as they are:
//   World::initialize        -> initializeOpenCL(gpuID); toggleOpenCL(use.opencl)
//   Simulation::performIterations -> launchCoulombKernel2() / launchGaussKernel2()
//   ChargeAgent::coulombGPU  -> getOutputHost(id), getOutputHostFuture(id)
//   Logger::saveCoulombEnergy -> launchCoulombKernel1(); getOutputHost(site)
// Differences, by design: every lattice site's value is returned by the
// kernel-1 launches (the reference read back only the first n), host mirrors
// grow with the charge count instead of being sized to the lattice, and
// errors surface as a status (lastStatus / lastError) instead of qFatal.
//
// WorldT must provide (the reference World's accessors, world.h):
//   parameters()  -> a SimulationParameters-like struct with gridX, gridY,
//                    gridZ, electrostaticCutoff, electrostaticPrefactor,
//                    coulombGaussianSigma, defectsCharge, useOpenCL, okCL,
//                    coulombCarriers, workX/Y/Z, workSize, openclThreshold;
//   electrons(), holes() -> iterable of pointers with getCurrentSite(),
//                    getFutureSite(), charge(), setOpenCLID(int);
//   defectSiteIDs() -> iterable of int.
#ifndef LANGMUIR_B200_HELPER_HPP
#define LANGMUIR_B200_HELPER_HPP

#include <cstdint>
#include <string>
#include <vector>

#include "langmuir_b200.h"

namespace langmuir_b200 {

template <class WorldT>
class OpenClHelper {
public:
    explicit OpenClHelper(WorldT& world) : m_world(world) {}
    ~OpenClHelper() { lgm_destroy(m_ctx); }
    OpenClHelper(const OpenClHelper&) = delete;
    OpenClHelper& operator=(const OpenClHelper&) = delete;

    // openclhelper.cpp:17-187: okCL is false until the device is set up; a
    // failure with use.opencl set is an error (the reference's qFatal).
    void initializeOpenCL(int gpuID = -1) {
        auto& p = m_world.parameters();
        p.okCL = false;
        lgm_config cfg;
        lgm_config_default(&cfg);
        cfg.grid_x = p.gridX;
        cfg.grid_y = p.gridY;
        cfg.grid_z = p.gridZ;
        cfg.electrostatic_cutoff = p.electrostaticCutoff;
        cfg.electrostatic_prefactor = p.electrostaticPrefactor;
        cfg.coulomb_gaussian_sigma = p.coulombGaussianSigma;
        cfg.work_x = p.workX;
        cfg.work_y = p.workY;
        cfg.work_z = p.workZ;
        cfg.work_size = p.workSize;
        cfg.opencl_threshold = p.openclThreshold;
        lgm_destroy(m_ctx);
        m_ctx = nullptr;
        m_status = lgm_create(&cfg, gpuID, &m_ctx);
        if (m_status != LGM_OK) {
            m_error = lgm_last_error(nullptr);
            return;
        }
        p.okCL = true;
    }

    // openclhelper.cpp:190-218
    bool toggleOpenCL(bool on) {
        auto& p = m_world.parameters();
        p.useOpenCL = on && p.okCL && p.coulombCarriers;
        return p.useOpenCL;
    }

    void launchCoulombKernel1() { launch1(LGM_POINT); }
    void launchGaussKernel1() { launch1(LGM_GAUSS); }
    void launchCoulombKernel2() { launch2(LGM_POINT); }
    void launchGaussKernel2() { launch2(LGM_GAUSS); }

    void copySiteAndChargeToHostVector(int index, int site, int charge = -1) {
        if ((size_t)index >= m_s.size()) {
            m_s.resize(index + 1);
            m_q.resize(index + 1);
        }
        m_s[index] = site;
        m_q[index] = charge;
    }

    // openclhelper.cpp:567-583
    double getOutputHost(int index) const { return m_o[index]; }
    double getOutputHostFuture(int index) const { return m_o[index + m_offset]; }

    lgm_status lastStatus() const { return m_status; }
    const std::string& lastError() const { return m_error; }
    lgm_ctx* context() const { return m_ctx; }

private:
    // Host packing of openclhelper.cpp:227-255 / 379-424: electrons, holes,
    // charged defects (the sources), then future sites of electrons, holes.
    int pack(bool future) {
        m_s.clear();
        m_q.clear();
        int i = 0;
        for (auto* e : m_world.electrons()) {
            m_s.push_back(e->getCurrentSite());
            m_q.push_back(e->charge());
            e->setOpenCLID(i++);
        }
        for (auto* h : m_world.holes()) {
            m_s.push_back(h->getCurrentSite());
            m_q.push_back(h->charge());
            h->setOpenCLID(i++);
        }
        const int dq = m_world.parameters().defectsCharge;
        if (dq != 0)
            for (int site : m_world.defectSiteIDs()) {
                m_s.push_back(site);
                m_q.push_back(dq);
            }
        m_offset = (int)m_s.size();
        if (future) {
            for (auto* e : m_world.electrons()) {
                m_s.push_back(e->getFutureSite());
                m_q.push_back(e->charge());
            }
            for (auto* h : m_world.holes()) {
                m_s.push_back(h->getFutureSite());
                m_q.push_back(h->charge());
            }
        }
        return m_offset;
    }

    void launch2(lgm_kind kind) {
        const int n = pack(true);
        m_o.assign(m_s.size(), 0.0);
        m_status = lgm_coulomb_kernel2(m_ctx, kind, m_s.data(), m_q.data(), n, (int32_t)m_s.size(),
                                       m_o.data());
        if (m_status != LGM_OK) m_error = lgm_last_error(m_ctx);
    }

    void launch1(lgm_kind kind) {
        const int n = pack(false);
        const auto& p = m_world.parameters();
        m_o.assign((size_t)p.gridX * p.gridY * p.gridZ, 0.0);
        m_status = lgm_coulomb_kernel1(m_ctx, kind, m_s.data(), m_q.data(), n, m_o.data());
        if (m_status != LGM_OK) m_error = lgm_last_error(m_ctx);
    }

    WorldT& m_world;
    lgm_ctx* m_ctx = nullptr;
    std::vector<int32_t> m_s, m_q;
    std::vector<double> m_o;
    int m_offset = 0;
    lgm_status m_status = LGM_OK;
    std::string m_error;
};

}  // namespace langmuir_b200

#endif
