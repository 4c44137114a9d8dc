/*
 * lgm_oracle.h -- CPU FP64 oracle for the Coulomb hot path of Langmuir.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, in plain C++ and FP64, the
 * reference engine's CPU Coulomb path and the semantics of its OpenCL kernels.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load it, and only as the checker or the timed CPU baseline.  The
 * product library (langmuir_b200) never links or calls it.
 *
 * Pins (what ties this restatement to the reference's own behaviour):
 *   - the compiled reference kernels: oracle/ref_kernel_cl.c builds the
 *     reference's own src/langmuirCore/kernel.cl as C (pthread work-groups)
 *     into oracle/_ref/, and tests compare orc_kernel2/orc_kernel1 with it;
 *   - LangmuirPython/langmuir/grid.py PrecalculatedMesh (imported from the
 *     reference by tests/golden/make_golden.py) pins the r^2, r, 1/r tables and
 *     the plain 1/r sums;
 *   - LangmuirPython/test/test.py:177-201 (tables vs brute force, 3x4x5 grid);
 *   - analytic known answers (one charge, cutoff shell, r = 0 skip, prefactor).
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the reference project root).
 */
#ifndef LGM_ORACLE_H
#define LGM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* Lattice and electrostatics set-up: World::initialize order
 * (src/langmuirCore/world.cpp:589-647), tables from
 * Potential::precalculateArrays (potential.cpp:246-324) and coupling
 * constants from Potential::updateCouplingConstants (potential.cpp:326-349). */
orc_ctx* orc_create(int grid_x, int grid_y, int grid_z, int cutoff,
                    int hopping_range, double sigma, double prefactor);
void orc_destroy(orc_ctx* ctx);

/* Copy out a (cutoff+1)^3 table: which = 0 R1, 1 R2, 2 iR, 3 eR.
 * Index [dx][dy][dz] row-major (Boost multi_array default order). */
void orc_table(const orc_ctx* ctx, int which, double* out);
/* Copy out the (h+1)^3 sI table (potential.cpp:313-323). */
void orc_self_table(const orc_ctx* ctx, double* out);
/* Copy out the (h+1)^3 coupling table (potential.cpp:326-349). */
void orc_coupling_table(const orc_ctx* ctx, double* out);

/* Grid index math, Grid::getIndexX/Y/Z/S (cubicgrid.cpp:132-165). */
int orc_index_x(const orc_ctx* ctx, int site);
int orc_index_y(const orc_ctx* ctx, int site);
int orc_index_z(const orc_ctx* ctx, int site);
int orc_index_s(const orc_ctx* ctx, int x, int y, int z);

/* Grid::neighborsSite (cubicgrid.cpp:207-471) without the drain entries:
 * writes up to 32 site ids (range 2 in 3-D), returns the count. */
int orc_neighbors(const orc_ctx* ctx, int site, int hopping_range, int* out);

/* One species sum as Potential::coulombE/H/D, gaussE/H/D and the Image
 * variants compute it (potential.cpp:351-753): table gathers iR (x eR when
 * gauss), per-axis distance < cutoff and R1 < cutoff, minus sign and
 * x-image distance x_i + x_j + 1 when image != 0; result x prefactor. */
double orc_species_potential(const orc_ctx* ctx, int site_i, const int32_t* sites,
                             const int32_t* charges, int n, int gauss, int image);

/* Right-electrode image sum: the same as image != 0 above but mirrored about
 * x = X - 1/2 (dx = 2X - 1 - x_i - x_j).  The reference has the left mirror
 * only (cubicgrid.cpp:117-120); this extension is restated here so the GPU
 * extension has an oracle. */
double orc_species_potential_right_image(const orc_ctx* ctx, int site_i,
                                         const int32_t* sites, const int32_t* charges,
                                         int n, int gauss);

/* Potentials at t targets from n sources the way the reference's CPU path
 * forms them (Potential::coulomb* / gauss* and, per `terms`, the image sums,
 * potential.cpp:351-753): direct sum (terms bit 0), minus the x = -1/2 image
 * sum (bit 1), minus the x = X - 1/2 image sum (bit 2, extension).  The
 * per-target loop runs over host threads (threads <= 0: all cores). */
void orc_potentials(const orc_ctx* ctx, int gauss, unsigned terms, const int32_t* src,
                    const int32_t* q, int n, const int32_t* tgt, int t, double* out,
                    int threads);

/* OpenCL kernel 2 semantics (kernel.cl:222-369), FP64:
 *   o[g] = prefactor * sum_{j<n} q_j * w(r2),  0 < r2 < cutoff^2 (int),
 *   w = 1/sqrt(r2) (coulomb2) or erf(erffactor*r)/r (gauss2),
 * for every g < total; site of target g is s[g] (w aliases s).
 * kind: 0 point, 1 gauss.  threads <= 0 means hardware concurrency. */
void orc_kernel2(const orc_ctx* ctx, int kind, const int32_t* s, const int32_t* q,
                 int n, int total, double* o, int threads);

/* OpenCL kernel 1 semantics (kernel.cl:56-220): potential at every site
 * k < volume from the n charges (s, q). */
void orc_kernel1(const orc_ctx* ctx, int kind, const int32_t* s, const int32_t* q,
                 int n, double* o, int threads);

/* ChargeAgent::coulombCPU for every carrier (chargeagent.cpp:215-271), the
 * reference's CPU hot loop, run over host threads as QtConcurrent::map does
 * (simulation.cpp:85-88).
 *   e_site/e_fsite: ne electrons (charge -1), h_site/h_fsite: nh holes (+1),
 *   d_site: nd defect sites with charge defects_charge,
 *   e_type/h_type: per-site agent type of the electron and hole grids
 *     (volume + 35 entries, values of orc_agent_type) -- used by
 *     bindingPotential (chargeagent.cpp:463-481),
 *   exciton_binding: parameter exciton.binding,
 *   de_out: ne + nh values, electrons first then holes (m_de).
 * p1_out/p2_out (optional, may be NULL): p1 and p2 before the final
 * subtraction, i.e. the potentials at the current and future sites. */
void orc_coulomb_cpu(const orc_ctx* ctx,
                     const int32_t* e_site, const int32_t* e_fsite, int ne,
                     const int32_t* h_site, const int32_t* h_fsite, int nh,
                     const int32_t* d_site, int nd, int defects_charge,
                     const uint8_t* e_type, const uint8_t* h_type,
                     double exciton_binding,
                     double* de_out, double* p1_out, double* p2_out,
                     int threads);

/* Agent::Type values used in the per-site type arrays (include/agent.h). */
enum orc_agent_type {
    ORC_EMPTY = 0, ORC_ELECTRON = 1, ORC_HOLE = 2, ORC_DEFECT = 3,
    ORC_SOURCE = 4, ORC_DRAIN = 5
};

/* Philox4x32-10 counter-based generator (Salmon et al., SC'11), the
 * random stream shared by the GPU kMC and this oracle. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Context accessors. */
void orc_dims(const orc_ctx* ctx, int dims[3]);
int orc_hopping_range(const orc_ctx* ctx);
double orc_sigma(const orc_ctx* ctx);

/* ---- one kMC step (transistor set-up), see lgm_oracle_kmc.cpp ------------- */
typedef struct orc_kmc_config {
    double inverse_kt;          /* inverse.kt = e / (k_B T) (parameters.h:387)   */
    double exciton_binding;     /* exciton.binding                               */
    int32_t coulomb_carriers;   /* coulomb.carriers                              */
    int32_t defects_charge;     /* defects.charge                                */
    uint32_t image_terms;       /* 2: left, 4: right electrode images (extension) */
    double rate_e_source_l, rate_e_source_r, rate_h_source_l, rate_h_source_r;
    double rate_e_drain_l, rate_e_drain_r, rate_h_drain_l, rate_h_drain_r;
    int32_t max_electrons, max_holes;
    uint32_t seed, replica;     /* Philox key                                    */
    /* solar-cell set-up (simulation.cpp:219-243): exciton source at
     * generation_rate (already scaled by the plane area), recombination */
    int32_t solar;
    double generation_rate, recombination_rate;
    int32_t recombination_range, hopping_range_neighbors;  /* the latter: hopping.range */
    /* extensions: phase[site] (0 donor, 1 acceptor); confine: holes only on
     * donor and electrons only on acceptor sites; bonds (donor, acceptor site
     * pairs): excitons generated across a random bond instead of at one site */
    const uint8_t* phase;
    int32_t confine;
    const int32_t* bonds;
    int32_t nbonds;
    /* injection energetics (sourceagent.cpp:125-181): source.metropolis takes
     * the Metropolis test on the injection energy instead of chooseYes;
     * source.coulomb adds the Coulomb and left-image sums of every charge at
     * the injection site; balance.charges (solar cell) injects from the
     * electrodes until electrons and holes balance (simulation.cpp:253-353),
     * the side set by voltage.left / voltage.right */
    int32_t source_metropolis, source_coulomb, balance_charges;
    double voltage_left, voltage_right;
} orc_kmc_config;

/* decideFuture outcomes per carrier */
enum orc_outcome { ORC_OCCUPIED = 0, ORC_MET_ACCEPT = 1, ORC_MET_REJECT = 2,
                   ORC_DRAIN_ACCEPT = 3, ORC_DRAIN_REJECT = 4 };

/* Advance one step.  pot: site energies (volume entries); defects: nd sites.
 * e_site/h_site: in/out carrier lists in list order (capacity max_electrons /
 * max_holes), with their lengths in ne_io and nh_io.  counters: 20 uint64, (attempts,
 * successes) of eSourceL, eSourceR, hSourceL, hSourceR, eDrainL, eDrainR,
 * hDrainL, hDrainR, the exciton source and the recombination agent.  outcome / de_out (optional): per carrier of the lists as
 * they were at the start of the step, electrons then holes. */
int orc_kmc_step(const orc_ctx* ctx, const orc_kmc_config* cfg, const double* pot,
                 const int32_t* defects, int nd, uint32_t step, int32_t* e_site, int32_t* ne_io,
                 int32_t* h_site, int32_t* nh_io, uint64_t* counters, int32_t* outcome,
                 double* de_out, int threads);

#ifdef __cplusplus
}
#endif

#endif
