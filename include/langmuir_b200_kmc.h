/*
 * langmuir_b200_kmc.h -- input keys and the GPU kMC step (C ABI).
 *
 * lgm_params carries every key the reference registers
 * (src/langmuirCore/keyvalueparser.cpp:15-105) with the defaults of
 * SimulationParameters (include/parameters.h:285-378).  lgm_params_parse reads
 * the [Parameters] section of a Langmuir input or checkpoint file with the
 * reference's rules (KeyValueParser::parse, keyvalueparser.cpp:112-173;
 * CheckPointer::loadParameters, checkpointer.cpp:403-429) and lgm_params_check
 * applies setCalculatedValues / checkSimulationParameters (parameters.h:384-646),
 * returning a status and a message where the reference called qFatal.
 *
 * lgm_kmc is one simulation replica whose whole step -- proposals, Coulomb
 * energy changes, Metropolis decisions, conflict resolution, drains and the
 * electrode sources -- runs on the GPU (Simulation::performIterations,
 * simulation.cpp:34-111, transistor set-up).
 */
#ifndef LANGMUIR_B200_KMC_H
#define LANGMUIR_B200_KMC_H

#include "langmuir_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lgm_params {
    char simulation_type[16];           /* simulation.type: transistor | solarcell */
    uint32_t current_step;              /* current.step        */
    int32_t iterations_real;            /* iterations.real     */
    uint64_t random_seed;               /* random.seed         */
    int32_t grid_z, grid_y, grid_x;     /* grid.z, grid.y, grid.x */
    int32_t hopping_range;              /* hopping.range       */
    int32_t output_is_on;               /* output.is.on        */
    int32_t iterations_print;           /* iterations.print    */
    int32_t output_precision, output_width;
    char output_stub[64];               /* output.stub         */
    int32_t output_ids_on_delete, output_ids_on_encounter, output_coulomb, output_step_chk;
    int32_t output_chk_trap_potential, output_potential;
    int32_t output_xyz, output_xyz_e, output_xyz_h, output_xyz_d, output_xyz_t, output_xyz_mode;
    int32_t image_traps, image_defects, image_carriers;
    double electron_percentage, hole_percentage, seed_charges, defect_percentage;
    double trap_percentage, trap_potential, gaussian_stdev, seed_percentage;
    double voltage_right, voltage_left, slope_z;
    int32_t coulomb_carriers;           /* coulomb.carriers        */
    double coulomb_gaussian_sigma;      /* coulomb.gaussian.sigma  */
    int32_t defects_charge;             /* defects.charge          */
    double exciton_binding, temperature_kelvin;
    double source_rate, e_source_l_rate, e_source_r_rate, h_source_l_rate, h_source_r_rate;
    double generation_rate;
    int32_t source_metropolis, source_coulomb;
    double source_scale_area;
    int32_t balance_charges;
    double drain_rate, e_drain_l_rate, e_drain_r_rate, h_drain_l_rate, h_drain_r_rate;
    double recombination_rate;
    int32_t recombination_range;
    int32_t use_opencl, work_x, work_y, work_z, work_size, opencl_threshold, opencl_device_id;
    int32_t max_threads;
    /* constants: registered as Constant in the reference, so an input file
     * cannot change them (variable.h:267-276); set them here directly */
    double boltzmann_constant, dielectric_constant, elementary_charge, permittivity_space;
    double grid_factor;
    int32_t electrostatic_cutoff;
    double electrostatic_prefactor, inverse_kt;
    /* extensions (keys the reference does not have):
     *   image.charges: electrode images in the hop energy, 0 none, 1 x = -1/2,
     *                  2 x = X - 1/2, 3 both;
     *   site.disorder: standard deviation (eV) of a Gaussian energy on every site */
    int32_t image_charges;
    double site_disorder;
    /*   morphology.confine: holes only on donor, electrons only on acceptor sites
     *                       (phase from lgm_kmc_set_morphology);
     *   generation.interface: excitons split across a random donor-acceptor bond */
    int32_t morphology_confine;
    int32_t generation_interface;
    /* Not an input key: the width of the FP64 guard band of the Metropolis
     * decisions, relative to the error scale N of the decision's two
     * potentials.  A decision whose FP32C energy lies within
     * guard_band * (N_current + N_future) of its acceptance threshold is taken
     * again from FP64 sums.  Default LGM_GUARD_BAND_MIN, the smallest width
     * that covers the FP32C error bound (lgm_params_check rejects less); a
     * wider band sends more decisions through the FP64 re-evaluation, which
     * tests use to exercise it. */
    double guard_band;
} lgm_params;
#define LGM_GUARD_BAND_MIN 8e-6

void lgm_params_default(lgm_params* p);
/* sizeof(lgm_params), for bindings that declare the struct themselves. */
int32_t lgm_params_size(void);

/* Parse `text` (an input file, or a checkpoint whose first section is
 * [Parameters]) into *p, starting from its current values.  Rules of the
 * reference: '#' starts a comment, one '=' per line, keys case-insensitive,
 * values may be quoted, empty values are skipped, the section ends at a line
 * "end" or at the end of the text, and -- as std::getline at EOF does there
 * -- a last line without a trailing newline is not read.  Unknown keys and
 * malformed lines fail with LGM_ERR_PARSE and a message in err. */
lgm_status lgm_params_parse(const char* text, lgm_params* p, char* err, int32_t err_len);

/* setCalculatedValues + checkSimulationParameters: derives
 * electrostatic_prefactor and inverse_kt, then validates; LGM_ERR_INVALID_ARGUMENT
 * with the reference's message on failure. */
lgm_status lgm_params_check(lgm_params* p, char* err, int32_t err_len);

/* The [Parameters] section of a checkpoint as the reference writes it
 * (CheckPointer::saveParameters, checkpointer.cpp; KeyValueParser stream
 * operator, keyvalueparser.cpp:217-228; TypedVariable::keyValue,
 * variable.h:196-238): every non-constant key in registration order, the key
 * left-aligned in 30 columns, then "=", then the value (doubles in scientific
 * notation with 15 digits, booleans True/False).  Extension keys are written
 * only when set, so that the reference reads the text.  Unlike the reference
 * the text ends with a newline, so its last key is not lost on reading.
 * Returns the size needed including the terminating zero (out may be NULL). */
int32_t lgm_params_format(const lgm_params* p, char* out, int32_t cap);

/* ---- one replica on the GPU ------------------------------------------------ */
typedef struct lgm_kmc lgm_kmc;

/* Builds the world on the host -- defects, traps (seeds and growth,
 * potential.cpp:74-244), site energies (linear field, gate, traps,
 * potential.cpp:17-72), seeded carriers (world.cpp:759-959) -- from a
 * Philox stream keyed by (random.seed, replica), then uploads it.  Transistor
 * and solar-cell set-ups. */
lgm_status lgm_kmc_create(const lgm_params* p, int32_t device, uint32_t replica, lgm_kmc** out);
/* The world lgm_kmc_create builds, on the host alone (no device is touched):
 * site energies [volume], defect sites, trap sites and potentials, and the
 * seeded electron and hole lists in list order.  counts receives the numbers
 * of defects, traps, electrons and holes; LGM_ERR_CAPACITY when a list does
 * not fit its capacity (counts are still set).  Every set-up draw comes from
 * one Philox stream in the order World::initialize consumes its generator
 * (world.cpp:589-650): placeDefects, placeElectrons, placeHoles,
 * setPotentialTraps. */
lgm_status lgm_kmc_world_host(const lgm_params* p, uint32_t replica, double* site_energy,
                              int32_t* defects, int32_t d_cap, int32_t* traps, double* trap_pots,
                              int32_t t_cap, int32_t* electrons, int32_t e_cap, int32_t* holes,
                              int32_t h_cap, int32_t* counts);
lgm_status lgm_kmc_destroy(lgm_kmc* k);
/* A world restored from a checkpoint (ConfigurationInfo filled by
 * CheckPointer::load, checkpointer.cpp:22-163): site lists in the reference's
 * section order.  Every count may be 0 (section absent).  As World::initialize
 * does (world.cpp:619-657), the listed defects, carriers and traps are placed
 * first and the rest are drawn as without a checkpoint: defects up to
 * defect.percentage, carriers up to (electron|hole).percentage * seed.charges,
 * traps up to trap.percentage (placeDefects world.cpp:659-757, placeElectrons
 * world.cpp:759-859, setPotentialTraps potential.cpp:74-244).  trap_potentials
 * is empty (trap.potential applies) or one per listed trap.  flux holds the
 * [FluxState] values in one of World::setFluxInfo's layouts (world.cpp:1189-1318):
 * 4 (transistor legacy), 10 or 12 (solar-cell legacy) or 20 (current). */
typedef struct lgm_world_config {
    const int32_t* electrons;
    int32_t n_electrons;
    const int32_t* holes;
    int32_t n_holes;
    const int32_t* defects;
    int32_t n_defects;
    const int32_t* traps;
    int32_t n_traps;
    const double* trap_potentials;
    int32_t n_trap_potentials;
    const uint64_t* flux;
    int32_t n_flux;
} lgm_world_config;

/* lgm_kmc_create with the world taken from `w`.  The step counter starts at
 * p->current_step; with the same random.seed and replica the counter-based
 * stream continues where the checkpointed run left off. */
lgm_status lgm_kmc_create_from(const lgm_params* p, const lgm_world_config* w, int32_t device,
                               uint32_t replica, lgm_kmc** out);

/* Text of the last error on `k`; k == NULL: why lgm_kmc_create failed on this thread. */
const char* lgm_kmc_last_error(const lgm_kmc* k);

/* Advance `steps` steps.  The first call records one step as a CUDA graph;
 * later steps replay it.  Synchronous. */
lgm_status lgm_kmc_run(lgm_kmc* k, int32_t steps);

typedef struct lgm_kmc_stats {
    uint32_t step;                 /* current.step                                       */
    int32_t electrons, holes;      /* carriers now                                       */
    int32_t max_electrons, max_holes;
    int32_t defects, traps;
    uint64_t proposals;            /* carrier proposals processed (hops attempted)        */
    uint64_t accepted;             /* proposals that moved a carrier or left by a drain   */
    uint64_t guard_evaluations;    /* decisions re-evaluated in FP64 (near the threshold) */
    uint64_t counters[20];         /* (attempts, successes) of eSourceL, eSourceR,
                                      hSourceL, hSourceR, eDrainL, eDrainR, hDrainL, hDrainR,
                                      the exciton source and the recombination agent */
} lgm_kmc_stats;
lgm_status lgm_kmc_stats_get(lgm_kmc* k, lgm_kmc_stats* s);

/* Carrier lists in list order (capacities in entries). */
lgm_status lgm_kmc_get_carriers(lgm_kmc* k, int32_t* e_sites, int32_t e_cap, int32_t* h_sites,
                                int32_t h_cap);
/* Replace the carriers (distinct sites per species, no defect sites). */
lgm_status lgm_kmc_set_carriers(lgm_kmc* k, const int32_t* e_sites, int32_t ne,
                                const int32_t* h_sites, int32_t nh);
/* Site energies (volume values), defect sites, trap sites and potentials. */
lgm_status lgm_kmc_get_world(lgm_kmc* k, double* site_energy, int32_t* defects, int32_t d_cap,
                             int32_t* traps, double* trap_potentials, int32_t t_cap);
/* Donor (0) / acceptor (1) phase of every lattice site, for
 * morphology.confine and generation.interface (extensions: carriers confined
 * to their phase, excitons generated across donor-acceptor bonds).  Call
 * before the first step. */
lgm_status lgm_kmc_set_morphology(lgm_kmc* k, const uint8_t* phase);

/* Per-carrier outcome of the last step (electrons then holes as listed at its
 * start: 0 occupied, 1 Metropolis accept, 2 Metropolis reject, 3 drain
 * accept, 4 drain reject) and the Coulomb energy change used. */
lgm_status lgm_kmc_last_outcomes(lgm_kmc* k, int32_t* outcome, double* de, int32_t cap);

/* ---- batched replicas --------------------------------------------------------
 * `count` independent replicas, params[i] for replica i (sizes, occupancies,
 * voltages and traps may all differ; the interaction kind must not), advanced
 * together.  Replica i uses the random stream of a single replica with id
 * replica0 + i, so its trajectory equals that of
 * lgm_kmc_create(&params[i], device, replica0 + i).
 * Two step forms share the batch:
 *  - fused: each replica runs the whole step inside one block, many steps
 *    per launch;
 *  - per phase: each phase of the step is one launch over the replicas, with
 *    the pair-sum tile shape and work split tuned on the batch before the
 *    first step; a batched step is one CUDA graph.
 * By default a batch whose replicas all have room for at most 2048 charges
 * (electron plus hole capacity) takes the fused form, any other the per-phase
 * form.  lgm_kmc_batch_set_fused splits a batch by capacity: both forms then
 * run in one graph, the fused kernel on a parallel branch. */
typedef struct lgm_kmc_batch lgm_kmc_batch;
lgm_status lgm_kmc_batch_create(const lgm_params* params, int32_t count, int32_t device,
                                uint32_t replica0, lgm_kmc_batch** out);
lgm_status lgm_kmc_batch_destroy(lgm_kmc_batch* b);
/* b == NULL: why lgm_kmc_batch_create failed on this thread. */
const char* lgm_kmc_batch_last_error(const lgm_kmc_batch* b);
lgm_status lgm_kmc_batch_run(lgm_kmc_batch* b, int32_t steps);
int32_t lgm_kmc_batch_size(const lgm_kmc_batch* b);
/* Replica i, owned by the batch: use the lgm_kmc_* accessors on it (stats,
 * carriers, world, outcomes); do not destroy or run it. */
lgm_kmc* lgm_kmc_batch_replica(lgm_kmc_batch* b, int32_t i);
/* Replicas with room for at most `max_charges` charges take the fused step,
 * the others the per-phase kernels (0: none fused).  Only before the first
 * lgm_kmc_batch_run. */
lgm_status lgm_kmc_batch_set_fused(lgm_kmc_batch* b, int32_t max_charges);
/* How many replicas take the fused step. */
int32_t lgm_kmc_batch_fused_count(const lgm_kmc_batch* b);
/* The tuned pair-sum shape: threads per CTA, target pairs per thread, source
 * chunks per work item, and the number of work items. */
lgm_status lgm_kmc_batch_tuning(const lgm_kmc_batch* b, int32_t* threads, int32_t* target_pairs,
                                int32_t* chunks_per_item, int32_t* items);
/* Times the batched pair sum on its own over the charges the last step
 * packed, `reps` times, each bracketed by CUDA events on the batch stream;
 * *ms is the median.  The pair sum is the culled replicas' chunk boxes, tile
 * culls and culled launch (per-phase replicas of point charges with room for
 * at least 1024 charges) followed by the tuned work-item kernel over the
 * other per-phase replicas.  The sums it writes are the last step's sums
 * again, so the simulation is unchanged.  Needs at least one step run on the
 * per-phase kernels (LGM_ERR_STATE otherwise).  Measurement aid with no
 * counterpart in the reference. */
lgm_status lgm_kmc_batch_time_pair(lgm_kmc_batch* b, int32_t reps, float* ms);
/* Runs the batched pair sum once more (as lgm_kmc_batch_time_pair) and counts
 * the source-target pairs it examined: for culled replicas, the pairs of the
 * 16-source groups whose boxes lie within the cutoff of a warp's targets; for
 * the others, every target against every packed source.  Measurement aid. */
lgm_status lgm_kmc_batch_count_pairs(lgm_kmc_batch* b, uint64_t* pairs);
/* How many replicas of the batch take the culled pair sum. */
int32_t lgm_kmc_batch_culled_count(const lgm_kmc_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* LANGMUIR_B200_KMC_H */
