// refkmc.cpp -- the reference's own kMC code, compiled, as a checker.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile (target refkmc) compiles the
// reference's src/langmuirCore/{world,cubicgrid,potential,rand,chargeagent,
// sourceagent,drainagent,fluxagent}.cpp from where they lie, against the Qt
// and Boost stand-ins of this directory, and links them with this file into
// oracle/_ref/librefkmc.so.  Only tests/ use it, to pin the GPU step and the
// FP64 oracle to the reference's own behaviour.
//
// What runs is the reference's code: World::initialize (world.cpp:507-657:
// placeDefects, placeElectrons/placeHoles through SourceAgent::tryToSeed,
// Potential::setPotentialZero/Linear/Gate/Traps, precalculateArrays,
// updateCouplingConstants, createSources/createDrains), Grid::neighborsSite,
// ChargeAgent::chooseFuture/coulombCPU/decideFuture/completeTick,
// Random::metropolisWithCoupling/chooseYes, DrainAgent/RecombinationAgent::
// tryToAccept and SourceAgent::tryToInject.  What this file restates is
// only the loop of Simulation::performIterations (simulation.cpp:29-111)
// and nextTick (simulation.cpp:355-414), because the random draws are keyed
// per call: before each agent call the loop points the draw source (see
// boost/random.hpp here) at the counter the GPU step and the oracle use for
// that call -- {step, list index, purpose, 0} -- so the reference code runs
// on the same draws.  World set-up draws come from one sequential stream
// {n, 0, 64, 0}, n = 0, 1, ..., in the order the reference consumes them.
//
// Error behaviour: the reference's qFatal throws here; every entry point
// catches it and returns -1 with the message in err.
#include <cmath>
#include <cstring>
#include <ctime>
#include <exception>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "boost/multi_array.hpp"
#include "boost/random.hpp"
#include "langmuir_b200_kmc.h"
#include "qshim.h"

// The harness reads the energy change each carrier computed (a protected
// member of ChargeAgent); opening the access specifiers changes no layout.
#define protected public
#define private public
#include "chargeagent.h"
#include "cubicgrid.h"
#include "drainagent.h"
#include "openclhelper.h"
#include "parameters.h"
#include "potential.h"
#include "rand.h"
#include "sourceagent.h"
#include "world.h"
#undef protected
#undef private

namespace refshim {
Draws& draws() {
    static Draws d;
    return d;
}
}  // namespace refshim

// The OpenCL helper is never used (use.opencl is off); World::initialize
// still creates one and asks it to initialise.
namespace LangmuirCore {
OpenClHelper::OpenClHelper(World& world, QObject* parent) : QObject(parent), m_world(world) {}
void OpenClHelper::initializeOpenCL(int) {}
bool OpenClHelper::toggleOpenCL(bool) { return false; }
double OpenClHelper::getOutputHost(int) const { return 0.0; }
double OpenClHelper::getOutputHostFuture(int) const { return 0.0; }
}  // namespace LangmuirCore

using namespace LangmuirCore;

namespace {

// Purposes of the Philox counter (the GPU's lgm_rng.cuh and the oracle use
// the same numbers).
enum : uint32_t {
    P_CHOOSE_E = 1, P_DECIDE_E = 2, P_CHOOSE_H = 3, P_DECIDE_H = 4, P_RECOMB = 5,
    P_SOURCE = 16, P_EXCITON = 20, P_BALANCE_E = 24, P_BALANCE_SIDE_E = 25, P_BALANCE_H = 26,
    P_BALANCE_SIDE_H = 27, P_SETUP = 64
};

void set_err(char* err, int len, const std::string& m) {
    if (err && len > 0) std::snprintf(err, (size_t)len, "%s", m.c_str());
}

SimulationParameters to_reference(const lgm_params& p) {
    SimulationParameters s;
    s.simulationType = QString(p.simulation_type);
    s.currentStep = p.current_step;
    s.iterationsReal = p.iterations_real;
    s.randomSeed = p.random_seed;
    s.gridZ = p.grid_z; s.gridY = p.grid_y; s.gridX = p.grid_x;
    s.hoppingRange = p.hopping_range;
    s.outputIsOn = false;
    s.iterationsPrint = p.iterations_print;
    s.electronPercentage = p.electron_percentage;
    s.holePercentage = p.hole_percentage;
    s.seedCharges = p.seed_charges;
    s.defectPercentage = p.defect_percentage;
    s.trapPercentage = p.trap_percentage;
    s.trapPotential = p.trap_potential;
    s.gaussianStdev = p.gaussian_stdev;
    s.seedPercentage = p.seed_percentage;
    s.voltageRight = p.voltage_right;
    s.voltageLeft = p.voltage_left;
    s.slopeZ = p.slope_z;
    s.coulombCarriers = p.coulomb_carriers != 0;
    s.coulombGaussianSigma = p.coulomb_gaussian_sigma;
    s.defectsCharge = p.defects_charge;
    s.excitonBinding = p.exciton_binding;
    s.temperatureKelvin = p.temperature_kelvin;
    s.sourceRate = p.source_rate;
    s.eSourceLRate = p.e_source_l_rate; s.eSourceRRate = p.e_source_r_rate;
    s.hSourceLRate = p.h_source_l_rate; s.hSourceRRate = p.h_source_r_rate;
    s.generationRate = p.generation_rate;
    s.sourceMetropolis = p.source_metropolis != 0;
    s.sourceCoulomb = p.source_coulomb != 0;
    s.sourceScaleArea = p.source_scale_area;
    s.balanceCharges = p.balance_charges != 0;
    s.drainRate = p.drain_rate;
    s.eDrainLRate = p.e_drain_l_rate; s.eDrainRRate = p.e_drain_r_rate;
    s.hDrainLRate = p.h_drain_l_rate; s.hDrainRRate = p.h_drain_r_rate;
    s.recombinationRate = p.recombination_rate;
    s.recombinationRange = p.recombination_range;
    s.useOpenCL = false;
    s.boltzmannConstant = p.boltzmann_constant;
    s.dielectricConstant = p.dielectric_constant;
    s.elementaryCharge = p.elementary_charge;
    s.permittivitySpace = p.permittivity_space;
    s.gridFactor = p.grid_factor;
    s.electrostaticCutoff = p.electrostatic_cutoff;
    setCalculatedValues(s);  // prefactor, 1/kT (parameters.h:384-390)
    return s;
}

// decideFuture's outcome (the codes the GPU step and the oracle report)
enum : int32_t { O_OCCUPIED = 0, O_MET_ACCEPT = 1, O_MET_REJECT = 2, O_DRAIN_ACCEPT = 3,
                 O_DRAIN_REJECT = 4 };

}  // namespace

struct ref_kmc {
    SimulationParameters params;
    World* world = nullptr;
    uint32_t replica = 0;
};

extern "C" {

ref_kmc* ref_kmc_create(const lgm_params* p, uint32_t replica, const int32_t* e, int ne,
                        const int32_t* h, int nh, const int32_t* d, int nd, const int32_t* traps,
                        int nt, const double* trap_pots, int ntp, char* err, int errlen) {
    if (!p) return nullptr;
    ref_kmc* k = new ref_kmc();
    try {
        k->params = to_reference(*p);
        k->replica = replica;
        ConfigurationInfo ci;
        for (int i = 0; i < ne; ++i) ci.electrons.push_back(e[i]);
        for (int i = 0; i < nh; ++i) ci.holes.push_back(h[i]);
        for (int i = 0; i < nd; ++i) ci.defects.push_back(d[i]);
        for (int i = 0; i < nt; ++i) ci.traps.push_back(traps[i]);
        for (int i = 0; i < ntp; ++i) ci.trapPotentials.push_back(trap_pots[i]);
        refshim::Draws& dr = refshim::draws();
        dr.replica = replica;
        dr.set_sequential(P_SETUP);
        k->world = new World(k->params, ci, -1, -1, nullptr);
        if (k->world->randomNumberGenerator().seed() == 0)
            throw std::runtime_error("random.seed 0 means the clock to the reference");
    } catch (const std::exception& x) {
        set_err(err, errlen, x.what());
        delete k->world;
        delete k;
        return nullptr;
    }
    return k;
}

void ref_kmc_destroy(ref_kmc* k) {
    if (!k) return;
    try {
        delete k->world;
    } catch (...) {
    }
    delete k;
}

// out: electrons, holes, defects, traps, max electrons, max holes, volume, current step
int ref_kmc_sizes(ref_kmc* k, int32_t* out) {
    if (!k || !out) return -1;
    World& w = *k->world;
    out[0] = w.numElectronAgents();
    out[1] = w.numHoleAgents();
    out[2] = w.numDefects();
    out[3] = w.numTraps();
    out[4] = w.maxElectronAgents();
    out[5] = w.maxHoleAgents();
    out[6] = w.electronGrid().volume();
    out[7] = (int32_t)w.parameters().currentStep;
    return 0;
}

// Site energies of both grids, defect and trap lists, trap potentials.
int ref_kmc_world(ref_kmc* k, double* pot_e, double* pot_h, int32_t* defects, int32_t* traps,
                  double* trap_pots) {
    if (!k) return -1;
    World& w = *k->world;
    const int V = w.electronGrid().volume();
    for (int s = 0; s < V; ++s) {
        if (pot_e) pot_e[s] = w.electronGrid().potential(s);
        if (pot_h) pot_h[s] = w.holeGrid().potential(s);
    }
    for (int i = 0; i < w.defectSiteIDs().size(); ++i)
        if (defects) defects[i] = w.defectSiteIDs()[i];
    for (int i = 0; i < w.trapSiteIDs().size(); ++i) {
        if (traps) traps[i] = w.trapSiteIDs()[i];
        if (trap_pots) trap_pots[i] = w.trapSitePotentials()[i];
    }
    return 0;
}

int ref_kmc_carriers(ref_kmc* k, int32_t* e, int32_t* h) {
    if (!k) return -1;
    World& w = *k->world;
    for (int i = 0; i < w.electrons().size(); ++i) e[i] = w.electrons()[i]->getCurrentSite();
    for (int i = 0; i < w.holes().size(); ++i) h[i] = w.holes()[i]->getCurrentSite();
    return 0;
}

// One step: Simulation::performIterations(1) (simulation.cpp:34-111) with
// every draw keyed as the GPU step keys it.  outcome/de: per carrier of the
// lists at the start of the step, electrons then holes.
int ref_kmc_step(ref_kmc* k, int32_t* outcome, double* de, char* err, int errlen) {
    if (!k) return -1;
    World& w = *k->world;
    refshim::Draws& dr = refshim::draws();
    try {
        const uint32_t step = w.parameters().currentStep;
        foreach (FluxAgent* flux, w.fluxes()) flux->storeLast();
        QList<ChargeAgent*>& electrons = w.electrons();
        QList<ChargeAgent*>& holes = w.holes();
        const int ne = electrons.size(), nh = holes.size();
        for (int i = 0; i < ne; i++) {
            dr.set_keyed(step, (uint32_t)i, P_CHOOSE_E);
            electrons.at(i)->chooseFuture();
        }
        for (int i = 0; i < nh; i++) {
            dr.set_keyed(step, (uint32_t)i, P_CHOOSE_H);
            holes.at(i)->chooseFuture();
        }
        if (w.parameters().coulombCarriers) {
            // QtConcurrent::map over both lists in the reference; no draws
            for (int i = 0; i < ne; i++) electrons.at(i)->coulombCPU();
            for (int i = 0; i < nh; i++) holes.at(i)->coulombCPU();
        }
        auto decide = [&](ChargeAgent* c, uint32_t index, uint32_t purpose, int slot) {
            const Agent::Type t = c->getGrid().agentType(c->getFutureSite());
            dr.set_keyed(step, index, purpose);
            c->decideFuture();
            const bool moved = c->getFutureSite() != c->getCurrentSite();
            int32_t code = O_OCCUPIED;
            if (t == Agent::Empty) code = moved ? O_MET_ACCEPT : O_MET_REJECT;
            else if (t == Agent::Drain) code = moved ? O_DRAIN_ACCEPT : O_DRAIN_REJECT;
            if (outcome) outcome[slot] = code;
            if (de) de[slot] = c->m_de;
        };
        for (int i = 0; i < ne; i++) decide(electrons.at(i), (uint32_t)i, P_DECIDE_E, i);
        for (int i = 0; i < nh; i++) decide(holes.at(i), (uint32_t)i, P_DECIDE_H, ne + i);
        // performRecombinations (simulation.cpp:219-231)
        if (w.parameters().simulationType == "solarcell" && w.parameters().recombinationRate > 0)
            for (int i = 0; i < electrons.size(); ++i) {
                dr.set_keyed(step, (uint32_t)i, P_RECOMB);
                w.recombinationAgent().tryToAccept(electrons[i]);
            }
        // nextTick (simulation.cpp:355-414, outputIdsOnDelete off)
        for (int i = 0; i < electrons.size(); ++i) {
            electrons[i]->completeTick();
            if (electrons[i]->removed()) {
                delete electrons[i];
                electrons.removeAt(i);
                --i;
            }
        }
        for (int i = 0; i < holes.size(); ++i) {
            holes[i]->completeTick();
            if (holes[i]->removed()) {
                delete holes[i];
                holes.removeAt(i);
                --i;
            }
        }
        // performInjections (simulation.cpp:233-251)
        if (w.parameters().simulationType == "solarcell") {
            dr.set_keyed(step, 0u, P_EXCITON);
            w.excitonSourceAgent().tryToInject();
            // Simulation::balanceCharges (simulation.cpp:253-353), restated
            // for its draws: try t of a species injects on {step, t, 24 / 26},
            // the side draw of equal voltages is on {step, t, 25 / 27}
            if (w.parameters().balanceCharges) {
                const double VL = w.parameters().voltageLeft, VR = w.parameters().voltageRight;
                int tries = 0;
                while (w.electronsMinusHoles() < 0 && !w.atMaxElectrons()) {
                    SourceAgent* src;
                    if (VR > VL) src = &w.electronSourceAgentLeft();
                    else if (VL > VR) src = &w.electronSourceAgentRight();
                    else {
                        dr.set_keyed(step, (uint32_t)tries, P_BALANCE_SIDE_E);
                        src = w.randomNumberGenerator().random() > 0.5
                                  ? static_cast<SourceAgent*>(&w.electronSourceAgentLeft())
                                  : static_cast<SourceAgent*>(&w.electronSourceAgentRight());
                    }
                    dr.set_keyed(step, (uint32_t)tries, P_BALANCE_E);
                    src->tryToInject();
                    tries += 1;
                    if (tries > 1024) qFatal("langmuir: can not balance electrons");
                }
                tries = 0;
                while (w.holesMinusElectrons() < 0 && !w.atMaxHoles()) {
                    SourceAgent* src;
                    if (VR > VL) src = &w.holeSourceAgentRight();
                    else if (VL > VR) src = &w.holeSourceAgentLeft();
                    else {
                        dr.set_keyed(step, (uint32_t)tries, P_BALANCE_SIDE_H);
                        src = w.randomNumberGenerator().random() > 0.5
                                  ? static_cast<SourceAgent*>(&w.holeSourceAgentRight())
                                  : static_cast<SourceAgent*>(&w.holeSourceAgentLeft());
                    }
                    dr.set_keyed(step, (uint32_t)tries, P_BALANCE_H);
                    src->tryToInject();
                    tries += 1;
                    if (tries > 1024) qFatal("langmuir: can not balance holes");
                }
            }
        } else {
            dr.set_keyed(step, 0u, P_SOURCE + 0);
            w.electronSourceAgentLeft().tryToInject();
            dr.set_keyed(step, 0u, P_SOURCE + 1);
            w.electronSourceAgentRight().tryToInject();
            dr.set_keyed(step, 0u, P_SOURCE + 2);
            w.holeSourceAgentLeft().tryToInject();
            dr.set_keyed(step, 0u, P_SOURCE + 3);
            w.holeSourceAgentRight().tryToInject();
        }
        w.parameters().currentStep += 1;
    } catch (const std::exception& x) {
        set_err(err, errlen, x.what());
        return -1;
    }
    return 0;
}

// Flux counters (attempts, successes) in the GPU step's layout: eSourceL,
// eSourceR, hSourceL, hSourceR, eDrainL, eDrainR, hDrainL, hDrainR, the
// exciton source, the recombination agent.
int ref_kmc_counters(ref_kmc* k, uint64_t* c) {
    if (!k || !c) return -1;
    World& w = *k->world;
    FluxAgent* a[10] = {&w.electronSourceAgentLeft(), &w.electronSourceAgentRight(),
                        &w.holeSourceAgentLeft(),     &w.holeSourceAgentRight(),
                        &w.electronDrainAgentLeft(),  &w.electronDrainAgentRight(),
                        &w.holeDrainAgentLeft(),      &w.holeDrainAgentRight(),
                        &w.excitonSourceAgent(),      &w.recombinationAgent()};
    for (int i = 0; i < 10; ++i) {
        c[2 * i] = a[i]->attempts();
        c[2 * i + 1] = a[i]->successes();
    }
    return 0;
}

// Grid::neighborsSite (cubicgrid.cpp:207-471) on the electron grid: lattice
// neighbours in the reference's order, then the face drains.
int ref_kmc_neighbors(ref_kmc* k, int site, int range, int32_t* out, int cap) {
    if (!k) return -1;
    try {
        QVector<int> nb = k->world->electronGrid().neighborsSite(site, range);
        for (int i = 0; i < nb.size() && i < cap; ++i) out[i] = nb[i];
        return nb.size();
    } catch (const std::exception&) {
        return -1;
    }
}

// Potential::updateCouplingConstants (potential.cpp:326-349): (h+1)^3 table.
int ref_kmc_coupling(ref_kmc* k, double* out) {
    if (!k) return -1;
    World& w = *k->world;
    const int h = w.parameters().hoppingRange + 1;
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < h; ++j)
            for (int l = 0; l < h; ++l) out[(i * h + j) * h + l] = w.couplingConstants()[i][j][l];
    return 0;
}

}  // extern "C"
