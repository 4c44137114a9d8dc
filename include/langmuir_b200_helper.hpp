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

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "langmuir_b200.h"

namespace langmuir_b200 {

template <class WorldT>
class OpenClHelper {
public:
    explicit OpenClHelper(WorldT& world) : m_world(world) {}
    ~OpenClHelper() {
        lgm_destroy(m_ctx);
        lgm_destroy(m_ctx64);
    }
    OpenClHelper(const OpenClHelper&) = delete;
    OpenClHelper& operator=(const OpenClHelper&) = delete;

    // Extension (no reference counterpart): how the kernels accumulate --
    // LGM_PATH_RSQRT (default), LGM_PATH_TABLE or LGM_PATH_TABLE64 (FP64
    // terms: every potential within the reference's 1e-4 % acceptance test).
    // Takes effect at the next initializeOpenCL.
    void setAccumulationPath(lgm_path path) { m_path = path; }

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
        cfg.path = m_path;
        lgm_destroy(m_ctx);
        lgm_destroy(m_ctx64);
        m_ctx = m_ctx64 = nullptr;
        m_cfg = cfg;
        m_device = gpuID;
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

    // One carrier's check by compareHostAndDeviceForAllCarriers.
    struct CoulombComparison {
        int openclID;
        double gpu1, gpu2;  // last launch: current site, future site minus the carrier's own term
        double cpu1, cpu2;  // the same from FP64 sums over the same charges
        double gpu, cpu;    // energy change q * (V2 - V1) of each
        bool failed;        // the reference's acceptance test
    };

    // openclhelper.cpp:546-558 and ChargeAgent::compareCoulomb
    // (chargeagent.cpp:298-370): every electron's and hole's potentials from
    // the last kernel-2 launch against FP64 sums over the same sources (a
    // second context in LGM_PREC_FP64, made on the first call).  A carrier
    // fails when the energy change differs by more than 1e-4 (signed, as the
    // reference tests it) or either potential by more than 1e-4 percent of
    // the mean of the two magnitudes.  The reference prints each comparison;
    // this returns them in `out` (if given) and returns the number that fail,
    // or -1 with lastStatus() set if the FP64 sums could not be made.
    int compareHostAndDeviceForAllCarriers(std::vector<CoulombComparison>* out = nullptr) {
        if (out) out->clear();
        const int nc = (int)(m_world.electrons().size() + m_world.holes().size());
        if (nc == 0 || m_o.size() < (size_t)(m_offset + nc)) return 0;
        if (!m_ctx64) {
            lgm_config cfg = m_cfg;
            cfg.precision = LGM_PREC_FP64;
            m_status = lgm_create(&cfg, m_device, &m_ctx64);
            if (m_status != LGM_OK) {
                m_error = lgm_last_error(nullptr);
                return -1;
            }
        }
        std::vector<int32_t> tgt(2 * (size_t)nc);
        for (int i = 0; i < nc; ++i) {
            tgt[i] = m_s[i];
            tgt[nc + i] = m_s[m_offset + i];
        }
        std::vector<double> cpu(tgt.size());
        m_status = lgm_potentials(m_ctx64, m_kind, LGM_TERM_DIRECT, m_s.data(), m_q.data(),
                                  m_offset, tgt.data(), (int32_t)tgt.size(), cpu.data());
        if (m_status != LGM_OK) {
            m_error = lgm_last_error(m_ctx64);
            return -1;
        }
        auto pdiff = [](double gpu, double cpu) {
            return std::fabs(gpu - cpu) / (0.5 * (std::fabs(cpu) + std::fabs(gpu))) * 100.0;
        };
        int failed = 0;
        for (int i = 0; i < nc; ++i) {
            const double q = m_q[i];
            const double self = m_cfg.electrostatic_prefactor * q;  // iR[1][0][0] = 1
            CoulombComparison c;
            c.openclID = i;
            c.gpu1 = m_o[i];
            c.gpu2 = m_o[m_offset + i] - self;
            c.cpu1 = cpu[i];
            c.cpu2 = cpu[nc + i] - self;
            c.gpu = q * (c.gpu2 - c.gpu1);
            c.cpu = q * (c.cpu2 - c.cpu1);
            c.failed = (c.gpu - c.cpu) > 1e-4 || pdiff(c.gpu1, c.cpu1) > 1e-4 ||
                       pdiff(c.gpu2, c.cpu2) > 1e-4;
            failed += c.failed;
            if (out) out->push_back(c);
        }
        return failed;
    }

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
        m_kind = kind;
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
    lgm_ctx* m_ctx64 = nullptr;  // FP64 sums for compareHostAndDeviceForAllCarriers
    lgm_config m_cfg{};
    int m_device = -1;
    lgm_path m_path = LGM_PATH_RSQRT;
    lgm_kind m_kind = LGM_POINT;
    std::vector<int32_t> m_s, m_q;
    std::vector<double> m_o;
    int m_offset = 0;
    lgm_status m_status = LGM_OK;
    std::string m_error;
};

}  // namespace langmuir_b200

#endif
