/*
 * langmuir_b200.h -- C ABI of the B200 Coulomb hot path for Langmuir.
 *
 * Drop-in for the engine's OpenCL helper (class OpenClHelper,
 * src/langmuirCore/include/openclhelper.h:22-241 in the reference): the same
 * packed site/charge buffers, the same kernel-1 / kernel-2 results, status
 * codes instead of qFatal, no exceptions across the boundary, caller-owned
 * buffers.  Plain C types only; a CUDA stream travels as `void*`.
 *
 * Threading: one lgm_ctx is used by one host thread at a time.  Results
 * written to caller buffers are plain memory once a synchronous call returns
 * and may be read concurrently (as the reference's QtConcurrent workers read
 * getOutputHost, simulation.cpp:77-80).
 *
 * Units: potentials in volts (prefactor * sum q_j w(r_ij)), as the reference.
 */
#ifndef LANGMUIR_B200_H
#define LANGMUIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LGM_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------- */
typedef int32_t lgm_status;
#define LGM_OK                     0
#define LGM_ERR_INVALID_ARGUMENT   1  /* null pointer, bad size or enum         */
#define LGM_ERR_OUT_OF_RANGE       2  /* a site id outside the lattice          */
#define LGM_ERR_CUDA               3  /* a CUDA runtime call failed              */
#define LGM_ERR_NO_DEVICE          4  /* no usable sm_100 device                 */
#define LGM_ERR_CAPACITY           5  /* more charges/targets than configured    */
#define LGM_ERR_TIMEOUT            6  /* a bounded device wait ran out           */
#define LGM_ERR_PARSE              7  /* input-file key/value error              */
#define LGM_ERR_UNSUPPORTED        8  /* valid in the reference, not supported   */
#define LGM_ERR_STATE              9  /* call out of order                       */

/* ---- enums --------------------------------------------------------------- */
/* Interaction kind: point charges (coulomb1/coulomb2, kernel.cl:56,222) or
 * Gaussian-smeared charges (gauss1/gauss2, kernel.cl:139,296). */
typedef enum lgm_kind { LGM_POINT = 0, LGM_GAUSS = 1 } lgm_kind;

/* Pair-sum arithmetic.  FP32C: FP32 terms, FP32 runs of up to 32 terms (16,
 * one source group, in the default variants) folded into FP64 accumulators.  FP64: every term in FP64 (the guard-band and
 * reference-precision path). */
typedef enum lgm_precision { LGM_PREC_FP32C = 0, LGM_PREC_FP64 = 1 } lgm_precision;

/* How 1/r is formed in FP32C: MUFU reciprocal square root, or a per-r^2
 * shared-memory table of correctly rounded values (r^2 is an integer).
 * TABLE64: r^2 exact in FP32 as in the other paths, each term w(r^2) read
 * from a per-r^2 table of FP64 values (1/sqrt(k), or erf(f sqrt(k))/sqrt(k)
 * for Gaussian charges, both correctly rounded) and accumulated in FP64: the
 * sums are as accurate as the FP64 path's.  Served by the culled tile
 * variants (LGM_VARIANT_CULLED); needs 8 (cutoff^2 + 1) bytes of shared
 * memory per CTA. */
typedef enum lgm_path { LGM_PATH_RSQRT = 0, LGM_PATH_TABLE = 1, LGM_PATH_TABLE64 = 2 } lgm_path;

/* Terms of lgm_potentials: direct sum, and the images of the sources in the
 * x = -1/2 electrode (Potential::coulombImage*, potential.cpp:384-753) and,
 * as an extension, in the x = X - 1/2 electrode.  Image terms enter with the
 * opposite sign, as in the reference. */
#define LGM_TERM_DIRECT       1u
#define LGM_TERM_IMAGE_LEFT   2u
#define LGM_TERM_IMAGE_RIGHT  4u

/* ---- configuration -------------------------------------------------------- */
/* The input keys of the reference that reach its OpenCL path
 * (include/parameters.h:205-223, 241-244; openclhelper.cpp:125-168). */
typedef struct lgm_config {
    int32_t grid_x, grid_y, grid_z;     /* grid.x / grid.y / grid.z                    */
    int32_t electrostatic_cutoff;       /* electrostatic.cutoff (sites, default 50)    */
    double  electrostatic_prefactor;    /* electrostatic.prefactor (V, see below)      */
    double  coulomb_gaussian_sigma;     /* coulomb.gaussian.sigma (sites)              */
    int32_t work_x, work_y, work_z;     /* work.x/y/z  (accepted; tiles are autotuned) */
    int32_t work_size;                  /* work.size   (accepted; tiles are autotuned) */
    int32_t opencl_threshold;           /* opencl.threshold (used by the shim)         */
    int32_t max_charges;                /* capacity: sources per call                  */
    int32_t max_targets;                /* capacity: targets per call                  */
    int32_t precision;                  /* lgm_precision                               */
    int32_t path;                       /* lgm_path                                    */
} lgm_config;

/* Defaults of SimulationParameters (parameters.h:285-378) for these keys;
 * electrostatic_prefactor = e / (4 pi eps_r eps_0 a) with eps_r = 3.5
 * (setCalculatedValues, parameters.h:384-390). */
void lgm_config_default(lgm_config* cfg);

typedef struct lgm_ctx lgm_ctx;

/* OpenClHelper::OpenClHelper + initializeOpenCL(gpuID) (openclhelper.cpp:12-187).
 * device < 0 selects device 0.  Allocates the device buffers for the
 * configured capacities. */
lgm_status lgm_create(const lgm_config* cfg, int32_t device, lgm_ctx** out);
lgm_status lgm_destroy(lgm_ctx* ctx);

/* Text of the last error on this context (ctx == NULL: last error of a failed
 * lgm_create on this thread).  Valid until the next call on the context. */
const char* lgm_last_error(const lgm_ctx* ctx);
const char* lgm_status_string(lgm_status status);
int32_t lgm_abi_version(void);

/* Potentials at t target sites from n source charges:
 *   out[g] = prefactor * sum_j q_j w(r(tgt_site[g], src_site[j])), 0 < r^2 < cutoff^2,
 *   w = 1/r (LGM_POINT) or erf(r / (sqrt(2) sigma)) / r (LGM_GAUSS),
 * plus the image terms selected by `terms` (subtracted).  Sources must be
 * lattice sites [0, volume); targets may also be the electrode ids
 * [volume, volume + 35) that the reference packs for drains
 * (openclhelper.cpp:411-424), whose values are defined but meaningless.
 * Host buffers, synchronous.  A site outside its range returns
 * LGM_ERR_OUT_OF_RANGE naming the first bad one (sources before targets) and
 * leaves out untouched; the check runs on the device with the sums, so the
 * call still does its device work first. */
lgm_status lgm_potentials(lgm_ctx* ctx, lgm_kind kind, uint32_t terms,
                          const int32_t* src_site, const int32_t* src_q, int32_t n,
                          const int32_t* tgt_site, int32_t t, double* out);

/* The same on device buffers, ordered on `stream` (a cudaStream_t; NULL =
 * the context's stream).  Returns once the work is enqueued; range errors
 * found on the device are reported by lgm_sync. */
lgm_status lgm_potentials_async(lgm_ctx* ctx, lgm_kind kind, uint32_t terms,
                                const int32_t* d_src_site, const int32_t* d_src_q, int32_t n,
                                const int32_t* d_tgt_site, int32_t t, double* d_out,
                                void* stream);

/* Wait for the context's work on `stream` and report device-side errors. */
lgm_status lgm_sync(lgm_ctx* ctx, void* stream);

/* OpenClHelper::launchCoulombKernel2 / launchGaussKernel2
 * (openclhelper.cpp:372-544, kernel.cl:222-369): s[total], q[total] packed as
 * the reference packs them (current sites of electrons, holes, charged
 * defects = the n sources, then the future sites of electrons and holes);
 * o[g] is the potential at s[g] from the n sources, for all g < total. */
lgm_status lgm_coulomb_kernel2(lgm_ctx* ctx, lgm_kind kind, const int32_t* s,
                               const int32_t* q, int32_t n, int32_t total, double* o);

/* OpenClHelper::launchCoulombKernel1 / launchGaussKernel1
 * (openclhelper.cpp:220-370, kernel.cl:56-220): potential at every lattice
 * site k < volume from the n charges (s, q); o holds `volume` values (the
 * reference reads back only n of them, openclhelper.cpp:261,284). */
lgm_status lgm_coulomb_kernel1(lgm_ctx* ctx, lgm_kind kind, const int32_t* s,
                               const int32_t* q, int32_t n, double* o);
lgm_status lgm_coulomb_kernel1_async(lgm_ctx* ctx, lgm_kind kind, const int32_t* d_s,
                                     const int32_t* d_q, int32_t n, double* d_o,
                                     void* stream);

/* Kernel-2 potentials that allocate no device memory.  No counterpart in the
 * reference: its OpenCL helper always allocated its own buffers.
 *
 * For callers that cannot call cudaMalloc: a host engine that sets up all of
 * its device memory once at start-up and forbids allocations afterwards, a
 * plugin whose device memory is owned by the application that loads it, or
 * code running where an allocation could stall or fail.  Such a caller owns
 * the inputs and the output; this entry needs no lgm_ctx.  Its working memory
 * is one fixed array of LGM_NOALLOC_SCRATCH_BYTES (4.25 MiB) in the library,
 * which every GPU that loads the library holds until the process exits.
 *
 * Same results as lgm_coulomb_kernel2 with LGM_POINT and the default FP32C
 * precision: d_s[total] / d_q[total] are device buffers packed as for
 * kernel 2 (the first n entries are the sources), d_o[total] receives the
 * potentials.  Limits: n <= LGM_NOALLOC_MAX_SOURCES and total <=
 * LGM_NOALLOC_MAX_TARGETS, else LGM_ERR_CAPACITY (nothing is launched).
 * Runs on `stream` (a cudaStream_t, NULL = legacy default) on the current
 * device and returns when the result is in d_o, with LGM_ERR_OUT_OF_RANGE
 * for a site outside the lattice.
 *
 * Each call waits for its own work before it returns: it reads the device
 * error word back on `stream`.  A leftover error of the caller's earlier CUDA
 * work is neither reported as this call's nor cleared.
 *
 * Set-up: the first call in a CUDA context (the primary context of the
 * current device, or a driver context the caller made current) looks up the
 * array's device address in that context and caches it under the context's
 * unique id; make that first call before any stream capture begins.  After
 * cudaDeviceReset the new primary context gets its own set-up.  All calls
 * share the array, so calls that overlap on the GPU race: serialize them. */
#define LGM_NOALLOC_MAX_SOURCES 32768
#define LGM_NOALLOC_MAX_TARGETS 65536
#define LGM_NOALLOC_SCRATCH_BYTES 4456704
lgm_status lgm_coulomb_kernel2_noalloc(int32_t grid_x, int32_t grid_y, int32_t grid_z,
                                       int32_t cutoff, double prefactor, const int32_t* d_s,
                                       const int32_t* d_q, int32_t n, int32_t total,
                                       double* d_o, void* stream);

/* Measured arithmetic peaks of one device (no reference counterpart): the
 * pair sums are bounded by FP32 FMA issue and by the MUFU pipe (rsqrt).  Each
 * probe runs 8 independent chains per thread on 8 blocks of 256 threads per
 * SM and reports the best of five launches (CUDA events): scalar FFMA and
 * packed FFMA2 in FP32 FLOP/s (2 per FMA lane), MUFU rsqrt per second.
 * clock_mhz_attribute is the device's clock-rate attribute (its maximum),
 * not the clock the probe ran at. */
typedef struct lgm_peaks {
    double ffma_tflops;
    double ffma2_tflops;
    double rsqrt_per_s;
    int32_t sm_count;
    double clock_mhz_attribute;
} lgm_peaks;
lgm_status lgm_probe_peaks(int32_t device, lgm_peaks* out);

/* Failure-detection self test (no reference counterpart): kernels whose
 * bulk-copy pipeline stages are armed but never filled -- the two-stage
 * pipeline of the classic tiles and the four-stage ring of the
 * warp-specialised culled kernel -- run the pair kernels' bounded waits with
 * `wait_limit` tries (1 .. 2^20) and their drains; the waits run out, the
 * device error word reports it, and the call returns LGM_ERR_TIMEOUT with the
 * context still usable (LGM_ERR_STATE if either kernel reported anything
 * else).  Nothing faults or hangs. */
lgm_status lgm_selftest_timeout(int32_t device, int32_t wait_limit);

/* Launch statistics of the last pair-sum launch on the context. */
typedef struct lgm_launch_info {
    int64_t pairs_tested;      /* (physical targets) x (sources), padding excluded */
    int32_t ctas;              /* CTAs of the pair kernel                          */
    int32_t splits;            /* source splits                                     */
    int32_t threads;           /* threads per CTA                                   */
    int32_t targets_per_thread;
    int32_t kernel_launches;   /* kernels launched by the call                      */
    float pair_kernel_ms;      /* device time of the pair kernel (timing on), else -1 */
    int32_t variant;           /* tile variant of the pair kernel, -1 if none ran   */
    int64_t pairs_examined;    /* culled variants with counting on (lgm_set_counting):
                                  the pairs whose r^2 the kernel computed; else -1    */
} lgm_launch_info;
/* Waits for the last launch when timing is on. */
lgm_status lgm_last_launch(lgm_ctx* ctx, lgm_launch_info* info);

/* Timing on: CUDA events on the launch stream bracket the pair kernel of
 * every call, read back by lgm_last_launch. */
lgm_status lgm_set_timing(lgm_ctx* ctx, int32_t enable);
/* Overlap on (the default): the kernels of a call are launched with
 * programmatic stream serialization, so each may be scheduled while the one
 * ahead of it is still running and waits for it on the device; the launch
 * gaps between them overlap the kernel ahead.  Off: plain stream order.  The
 * results are the same bits either way.  A measurement aid. */
lgm_status lgm_set_launch_overlap(lgm_ctx* ctx, int32_t enable);
/* Counting on: culled pair sums count the pairs they examine (one atomic add
 * per warp and live source chunk), read back by lgm_last_launch as
 * pairs_examined.  A measurement aid: leave it off in timed runs. */
lgm_status lgm_set_counting(lgm_ctx* ctx, int32_t enable);

/* ---- tile autotuner --------------------------------------------------------
 * The pair kernel is compiled in several tile shapes (threads per CTA, target
 * pairs per thread, FP32 run length).  lgm_autotune times each on synthetic
 * charges of the given size (n sources, t targets, `terms`) with CUDA events,
 * remembers the fastest for that size bucket (half-octaves of targets and
 * source chunks) on this context, and reports it; calls in an untuned bucket
 * use variant 0.  It allocates, so call it before any stream capture. */
lgm_status lgm_autotune(lgm_ctx* ctx, lgm_kind kind, uint32_t terms, int32_t n, int32_t t,
                        int32_t* chosen);
/* Force a variant (0 .. lgm_variant_count()-1) for every call, -1 = automatic. */
lgm_status lgm_set_variant(lgm_ctx* ctx, int32_t variant);
int32_t lgm_variant_count(void);
lgm_status lgm_variant_info(int32_t variant, int32_t* threads, int32_t* target_pairs,
                            int32_t* run);
/* Variant flags.  LGM_VARIANT_WARP_SKIP: a warp owns 64 * target_pairs
 * consecutive targets of the spatially sorted order (every call sorts its
 * targets by lattice cell) and skips the 1/r and accumulation of a source
 * that no pair of its targets has inside the cutoff; r^2 is still tested for
 * every pair and the sums are unchanged. */
#define LGM_VARIANT_WARP_SKIP 1
/* LGM_VARIANT_CULLED: the sources are sorted by lattice cell as well; each
 * source chunk (128 sources) and each group of 16 gets a bounding box, a cull
 * pass lists per tile of targets the chunks whose box comes within the cutoff,
 * and a persistent kernel sums over those work items only, a warp skipping any
 * group whose box lies beyond the cutoff of its own targets.  Skipped pairs
 * all have r >= cutoff, so the sums are those of the full tile over the same
 * source order. */
#define LGM_VARIANT_CULLED 2
/* LGM_VARIANT_WARP_SPECIALISED (with LGM_VARIANT_CULLED): one producer warp
 * per CTA streams the chunks through a ring of stages and the CTAs take work
 * items from a shared counter; the target warps do not wait for one another.
 * The sums equal those of the other culled variants bit for bit.  `threads`
 * of lgm_variant_info counts the target warps' threads only. */
#define LGM_VARIANT_WARP_SPECIALISED 4
lgm_status lgm_variant_flags(int32_t variant, int32_t* flags);
/* Culled variants: source chunks per work item (at least; more when a
 * tile's live chunks exceed 32 items) and, warp-specialised, the stages of
 * the copy ring (0 otherwise); both 0 for the other variants. */
lgm_status lgm_variant_items(int32_t variant, int32_t* chunks_per_item, int32_t* stages);

#ifdef __cplusplus
}
#endif

#endif /* LANGMUIR_B200_H */
