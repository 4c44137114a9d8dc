/*
 * ref_kernel_cl.c -- runs the reference's own OpenCL kernels on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY (the compiled-reference checker).  This file holds
 * no reference code: it defines the handful of OpenCL C builtins that the
 * reference's src/langmuirCore/kernel.cl uses, then #includes that file from
 * where it lies (the include path is given by oracle/Makefile, which writes
 * the result only into oracle/_ref/).  Work-groups run one after another; the
 * work-items of a group are host threads that meet at a pthread barrier for
 * every barrier(CLK_LOCAL_MEM_FENCE).  __local arrays become function-static
 * storage, shared by the work-items of the running group as in OpenCL.
 *
 * OpenCL leaves the accuracy of double rsqrt to the implementation; here it
 * is 1.0 / sqrt(x).  erf is the C library's.
 */
#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

/* ---- OpenCL C surface used by kernel.cl ---------------------------------- */
#define __kernel
#define __global
#define __local static
#define __write_only
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP 0
#define CLK_FILTER_NEAREST 0
typedef int image2d_t;
typedef int sampler_t;
#define int2 long
struct ref_float4 { float x, y, z, w; };
#define float4 struct ref_float4
#define write_imagef(img, coord, val) ((void)(img), (void)(coord), (void)(val))

static __thread size_t tl_local[3];
static __thread size_t tl_group[3];
static size_t g_local_size[3];
static size_t g_num_groups[3];
static pthread_barrier_t g_barrier;

static size_t get_local_id(int d) { return tl_local[d]; }
static size_t get_group_id(int d) { return tl_group[d]; }
static size_t get_local_size(int d) { return g_local_size[d]; }
static size_t get_num_groups(int d) { return g_num_groups[d]; }
static size_t get_global_id(int d) { return tl_group[d] * g_local_size[d] + tl_local[d]; }
static size_t get_global_size(int d) { return g_num_groups[d] * g_local_size[d]; }
static void barrier(int flags) { (void)flags; pthread_barrier_wait(&g_barrier); }
static double rsqrt(double x) { return 1.0 / sqrt(x); }

#pragma GCC diagnostic ignored "-Wunknown-pragmas"
#pragma GCC diagnostic ignored "-Wunused-value"
#pragma GCC diagnostic ignored "-Wunused-variable"
#include REF_KERNEL_CL

/* ---- NDRange driver ------------------------------------------------------ */
enum { REF_COULOMB1 = 0, REF_GAUSS1 = 1, REF_COULOMB2 = 2, REF_GAUSS2 = 3 };

struct ref_launch {
    int which;
    double* o; int* s; int* q; int n; int c2; int* w;
    int xsize; int ysize; double prefactor; double erffactor;
};

struct ref_item { const struct ref_launch* L; size_t local[3]; };

static void run_one(const struct ref_launch* L) {
    switch (L->which) {
    case REF_COULOMB1: coulomb1(L->o, L->s, L->q, L->n, L->c2, L->prefactor); break;
    case REF_GAUSS1: gauss1(L->o, L->s, L->q, L->n, L->c2, L->prefactor, L->erffactor); break;
    case REF_COULOMB2:
        coulomb2(L->o, L->s, L->q, L->n, L->c2, L->w, L->xsize, L->ysize, L->prefactor);
        break;
    default:
        gauss2(L->o, L->s, L->q, L->n, L->c2, L->w, L->xsize, L->ysize, L->prefactor,
               L->erffactor);
        break;
    }
}

/* Each work-item thread walks every group in order; the barrier at the end of
 * a group keeps the groups from overlapping (their __local storage is shared). */
static void* item_main(void* arg) {
    struct ref_item* it = (struct ref_item*)arg;
    tl_local[0] = it->local[0]; tl_local[1] = it->local[1]; tl_local[2] = it->local[2];
    for (size_t gz = 0; gz < g_num_groups[2]; ++gz)
        for (size_t gy = 0; gy < g_num_groups[1]; ++gy)
            for (size_t gx = 0; gx < g_num_groups[0]; ++gx) {
                tl_group[0] = gx; tl_group[1] = gy; tl_group[2] = gz;
                run_one(it->L);
                pthread_barrier_wait(&g_barrier);
            }
    return NULL;
}

static int launch(const struct ref_launch* L, const size_t groups[3], const size_t local[3]) {
    const size_t nitems = local[0] * local[1] * local[2];
    for (int d = 0; d < 3; ++d) { g_num_groups[d] = groups[d]; g_local_size[d] = local[d]; }
    if (pthread_barrier_init(&g_barrier, NULL, (unsigned)nitems) != 0) return -1;
    pthread_t* th = (pthread_t*)malloc(nitems * sizeof(pthread_t));
    struct ref_item* items = (struct ref_item*)malloc(nitems * sizeof(struct ref_item));
    size_t k = 0;
    for (size_t lz = 0; lz < local[2]; ++lz)
        for (size_t ly = 0; ly < local[1]; ++ly)
            for (size_t lx = 0; lx < local[0]; ++lx, ++k) {
                items[k].L = L;
                items[k].local[0] = lx; items[k].local[1] = ly; items[k].local[2] = lz;
                pthread_create(&th[k], NULL, item_main, &items[k]);
            }
    for (k = 0; k < nitems; ++k) pthread_join(th[k], NULL);
    pthread_barrier_destroy(&g_barrier);
    free(th); free(items);
    return 0;
}

/* Kernel 2 as OpenClHelper::launchCoulombKernel2 / launchGaussKernel2 set it
 * up (openclhelper.cpp:125-168, 372-544): global = total * workSize, local =
 * workSize, w aliases s, o has `total` entries.  gauss != 0 selects gauss2. */
int ref_kernel2(int gauss, const int* s, const int* q, int n, int total, int cutoff,
                int xsize, int ysize, double prefactor, double sigma, int work_size,
                double* o) {
    if (work_size < 1 || work_size > 1024) return -2;
    struct ref_launch L;
    L.which = gauss ? REF_GAUSS2 : REF_COULOMB2;
    L.o = o; L.s = (int*)s; L.q = (int*)q; L.n = n; L.c2 = cutoff * cutoff;
    L.w = (int*)s; L.xsize = xsize; L.ysize = ysize; L.prefactor = prefactor;
    L.erffactor = sigma > 0 ? 1.0 / (sqrt(2.0) * sigma) : 0.0;
    size_t groups[3] = {(size_t)total, 1, 1};
    size_t local[3] = {(size_t)work_size, 1, 1};
    return launch(&L, groups, local);
}

/* Kernel 1 as launchCoulombKernel1 / launchGaussKernel1 set it up
 * (openclhelper.cpp:220-370): global = grid * work, local = work.x,y,z.
 * o must hold grid_x*grid_y*grid_z values (the reference reads back only n,
 * openclhelper.cpp:261,284; here every site is returned). */
int ref_kernel1(int gauss, const int* s, const int* q, int n, int cutoff, int grid_x,
                int grid_y, int grid_z, double prefactor, double sigma, int work_x,
                int work_y, int work_z, double* o) {
    if (work_x * work_y * work_z > 64 || work_x < 1 || work_y < 1 || work_z < 1) return -2;
    struct ref_launch L;
    L.which = gauss ? REF_GAUSS1 : REF_COULOMB1;
    L.o = o; L.s = (int*)s; L.q = (int*)q; L.n = n; L.c2 = cutoff * cutoff;
    L.w = NULL; L.xsize = grid_x; L.ysize = grid_y; L.prefactor = prefactor;
    L.erffactor = sigma > 0 ? 1.0 / (sqrt(2.0) * sigma) : 0.0;
    size_t groups[3] = {(size_t)grid_x, (size_t)grid_y, (size_t)grid_z};
    size_t local[3] = {(size_t)work_x, (size_t)work_y, (size_t)work_z};
    return launch(&L, groups, local);
}
