// Drives include/langmuir_b200_helper.hpp the way the reference engine drives
// its OpenClHelper: a World with electrons, holes and charged defects, the
// kernel-2 launch, and the getOutputHost / getOutputHostFuture accessors.
// Input on stdin: X Y Z cutoff ne nh nd defects_charge, then ne+nh lines
// "site future_site", then nd defect sites.  Output: okCL, status, then one
// line per carrier: opencl_id p_current p_future.  With --compare, instead
// compareHostAndDeviceForAllCarriers: "failed N", then per carrier
// "opencl_id gpu1 gpu2 cpu1 cpu2 gpu cpu failed".  A second argument selects
// the accumulation path (lgm_path: 0 rsqrt, 1 table, 2 FP64 table).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "langmuir_b200_helper.hpp"

struct Params {
    int gridX, gridY, gridZ, electrostaticCutoff, defectsCharge;
    double electrostaticPrefactor, coulombGaussianSigma;
    bool useOpenCL, okCL, coulombCarriers;
    int workX, workY, workZ, workSize, openclThreshold;
};

struct Charge {
    int site, fsite, q, id;
    int getCurrentSite() const { return site; }
    int getFutureSite() const { return fsite; }
    int charge() const { return q; }
    void setOpenCLID(int i) { id = i; }
};

struct World {
    Params p;
    std::vector<Charge*> e, h;
    std::vector<int> d;
    Params& parameters() { return p; }
    std::vector<Charge*>& electrons() { return e; }
    std::vector<Charge*>& holes() { return h; }
    std::vector<int>& defectSiteIDs() { return d; }
};

int main(int argc, char** argv) {
    const bool compare = argc > 1 && std::string(argv[1]) == "--compare";
    World w{};
    int ne, nh, nd;
    if (std::scanf("%d %d %d %d %d %d %d %d", &w.p.gridX, &w.p.gridY, &w.p.gridZ,
                   &w.p.electrostaticCutoff, &ne, &nh, &nd, &w.p.defectsCharge) != 8)
        return 2;
    lgm_config def;
    lgm_config_default(&def);
    w.p.electrostaticPrefactor = def.electrostatic_prefactor;
    w.p.coulombCarriers = true;
    w.p.workX = w.p.workY = w.p.workZ = 4;
    w.p.workSize = 256;
    w.p.openclThreshold = 256;
    std::vector<Charge> store(ne + nh);
    for (int i = 0; i < ne + nh; ++i) {
        if (std::scanf("%d %d", &store[i].site, &store[i].fsite) != 2) return 2;
        store[i].q = i < ne ? -1 : 1;
        (i < ne ? w.e : w.h).push_back(&store[i]);
    }
    for (int k = 0; k < nd; ++k) {
        int s;
        if (std::scanf("%d", &s) != 1) return 2;
        w.d.push_back(s);
    }
    langmuir_b200::OpenClHelper<World> helper(w);
    if (argc > 2) helper.setAccumulationPath((lgm_path)std::atoi(argv[2]));
    helper.initializeOpenCL(0);
    const bool on = helper.toggleOpenCL(true);
    std::printf("okCL %d use %d status %d\n", (int)w.p.okCL, (int)on, (int)helper.lastStatus());
    if (!w.p.okCL) return 0;
    helper.launchCoulombKernel2();
    if (helper.lastStatus() != LGM_OK) {
        std::printf("error %s\n", helper.lastError().c_str());
        return 1;
    }
    if (compare) {
        std::vector<langmuir_b200::OpenClHelper<World>::CoulombComparison> cmp;
        const int failed = helper.compareHostAndDeviceForAllCarriers(&cmp);
        std::printf("failed %d\n", failed);
        if (failed < 0) {
            std::printf("error %s\n", helper.lastError().c_str());
            return 1;
        }
        for (const auto& c : cmp)
            std::printf("%d %.17g %.17g %.17g %.17g %.17g %.17g %d\n", c.openclID, c.gpu1, c.gpu2,
                        c.cpu1, c.cpu2, c.gpu, c.cpu, (int)c.failed);
        return 0;
    }
    for (Charge& c : store)
        std::printf("%d %.17g %.17g\n", c.id, helper.getOutputHost(c.id),
                    helper.getOutputHostFuture(c.id));
    return 0;
}
