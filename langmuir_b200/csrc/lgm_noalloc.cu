// lgm_noalloc.cu -- kernel-2 potentials without any device allocation.
//
// For callers that must not allocate device memory: a host engine that
// preallocates every buffer at start-up and forbids cudaMalloc afterwards, a
// plugin whose device memory belongs to the host application, or code that
// runs where an allocation would stall or fail.  They pass their own input
// and output buffers; the working memory of the computation (source and
// target records, split partial sums, the device error word) lives in one
// file-scope device array of fixed size, loaded with the library and held
// by every GPU that loads it until the process exits.
//
// Set-up: the array's name is only a host-side stand-in (a kernel given that
// name from host code would read the wrong memory), so the first call in a
// CUDA context looks up the array's device address in that context with
// cudaGetSymbolAddress and caches it under the context's unique id
// (cuCtxGetId).  A call in another context -- a driver context the caller
// made current, or the primary context created anew after cudaDeviceReset --
// does its own set-up.  Make the first call in a context before any stream
// capture begins.
//
// Every call shares the array and leaves the previous call's contents in
// it; the error word is cleared at the start of each call, everything else
// is fully written before it is read.  Calls that overlap on the GPU (two
// streams, two host threads, two devices' worth of work aimed at one device)
// race on the array: serialize them.
#include <cuda.h>  // CUcontext and the driver entry points' types (no link to libcuda)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "langmuir_b200.h"
#include "lgm_pairs.cuh"

using namespace lgm;

namespace {

constexpr int kNalThreads = 128;     // tile shape of the pair kernel used here
constexpr int kNalRP = 4;
constexpr int kNalSub = 32;
constexpr int kNalTile = kNalThreads * 2 * kNalRP;
constexpr int kNalMaxSplits = 4;
constexpr int kNalDrainIds = 35;     // electrode ids volume .. volume+34 (cubicgrid.cpp:22)

constexpr size_t kSrcPad = LGM_NOALLOC_MAX_SOURCES;                         // multiple of CH
constexpr size_t kTgtPad = (LGM_NOALLOC_MAX_TARGETS + kNalTile - 1) / kNalTile * kNalTile;
constexpr size_t kGeoOff = 0;
constexpr size_t kQqOff = kGeoOff + kSrcPad * 2 * sizeof(float4);
constexpr size_t kTgtOff = kQqOff + kSrcPad * sizeof(float2);
constexpr size_t kPartOff = kTgtOff + kTgtPad * sizeof(float4);
constexpr size_t kErrOff = kPartOff + (size_t)kNalMaxSplits * kTgtPad * sizeof(double);
constexpr size_t kScratchBytes = kErrOff + 256;
static_assert(kSrcPad % CH == 0, "source capacity must be whole chunks");
static_assert(kScratchBytes == LGM_NOALLOC_SCRATCH_BYTES, "header states the scratch size");

// The scratch array.  Device code could name it directly; host code must use
// the address obtained from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct ContextSetup {
    unsigned long long ctx_id = 0;   // cuCtxGetId of the context the entry was set up in
    unsigned char* base = nullptr;   // device address of g_noalloc_scratch in that context
    int sm_count = 0;
    int blocks_per_sm = 0;
};
constexpr int kMaxContexts = 64;
ContextSetup g_setup[kMaxContexts];
int g_setup_count = 0;
int g_setup_next = 0;                // slot replaced when every slot is taken
std::mutex g_setup_mutex;

using NalPairFn = void (*)(PairArgs);
constexpr NalPairFn kNalPair = &pair_kernel<0, 0, kNalThreads, kNalRP, kNalSub>;

// The driver's cuCtxGetCurrent and cuCtxGetId, found through the runtime so
// that the library does not link libcuda itself.
typedef CUresult(CUDAAPI* CtxGetCurrentFn)(CUcontext*);
typedef CUresult(CUDAAPI* CtxGetIdFn)(CUcontext, unsigned long long*);
struct DriverFns {
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
};
const DriverFns& driver_fns() {
    static const DriverFns fns = [] {
        DriverFns f;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_id = reinterpret_cast<CtxGetIdFn>(p);
        return f;
    }();
    return fns;
}

// The unique id of the calling thread's current context on `dev`.  With no
// context current yet, the device's primary context is made current first
// (cudaSetDevice initialises it); a context the caller made current is kept.
lgm_status current_context_id(int dev, unsigned long long* id) {
    const DriverFns& f = driver_fns();
    if (!f.get_current || !f.get_id) return LGM_ERR_NO_DEVICE;
    CUcontext ctx = nullptr;
    if (f.get_current(&ctx) != CUDA_SUCCESS) return LGM_ERR_CUDA;
    if (!ctx) {
        if (cudaSetDevice(dev) != cudaSuccess) return LGM_ERR_CUDA;
        if (f.get_current(&ctx) != CUDA_SUCCESS || !ctx) return LGM_ERR_CUDA;
    }
    return f.get_id(ctx, id) == CUDA_SUCCESS ? LGM_OK : LGM_ERR_CUDA;
}

// Once per context, with that context current on `dev`.
lgm_status setup_context(int dev, ContextSetup* out) {
    unsigned long long id = 0;
    lgm_status st = current_context_id(dev, &id);
    if (st != LGM_OK) return st;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    for (int i = 0; i < g_setup_count; ++i)
        if (g_setup[i].ctx_id == id) {
            *out = g_setup[i];
            return LGM_OK;
        }
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        major != 10)
        return LGM_ERR_NO_DEVICE;
    ContextSetup s;
    s.ctx_id = id;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
        return LGM_ERR_CUDA;
    s.base = static_cast<unsigned char*>(p);
    if (cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return LGM_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s.blocks_per_sm, kNalPair, kNalThreads,
                                                      pair_smem_bytes(0)) != cudaSuccess)
        return LGM_ERR_CUDA;
    int slot = g_setup_count;
    if (slot < kMaxContexts) {
        ++g_setup_count;
    } else {
        slot = g_setup_next;
        g_setup_next = (g_setup_next + 1) % kMaxContexts;
    }
    g_setup[slot] = s;
    *out = s;
    return LGM_OK;
}

// A launch whose own status is returned (a leftover error of the caller's
// earlier work is neither reported as this entry's nor cleared).
template <class... Args>
cudaError_t launch(void (*kern)(Args...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                   Args... args) {
    void* argv[] = {static_cast<void*>(&args)...};
    return cudaLaunchKernel(reinterpret_cast<const void*>(kern), grid, block, argv, smem, st);
}

__global__ void nal_prep_sources(const int32_t* __restrict__ s, const int32_t* __restrict__ q,
                                 int n, int n_pad, int X, int Y, int XY, int volume,
                                 float4* __restrict__ geo, float2* __restrict__ qq,
                                 unsigned* err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_pad) return;
    float a = 0.f, b = 0.f, c = 0.f, d = -0.5f, qf = 0.f;
    if (j < n) {
        const int sj = s[j];
        if (sj < 0 || sj >= volume) {
            atomicOr(err, DEVERR_SOURCE_RANGE);
        } else {
            const int z = sj / XY, y = sj / X - z * Y, x = sj % X;
            a = -2.f * x; b = -2.f * y; c = -2.f * z;
            d = (float)(x * x + y * y + z * z) - 0.5f;
            qf = (float)q[j];
        }
    }
    geo[2 * j] = make_float4(a, a, b, b);
    geo[2 * j + 1] = make_float4(c, c, d, d);
    qq[j] = make_float2(qf, qf);
}

__global__ void nal_prep_targets(const int32_t* __restrict__ ts, int t, int t_pad, int X, int Y,
                                 int XY, int volume, float4* __restrict__ tgt, unsigned* err) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= t_pad) return;
    int x = 0, y = 0, z = 0;
    if (g < t) {
        const int sg = ts[g];
        if (sg < 0 || sg >= volume + kNalDrainIds) {
            atomicOr(err, DEVERR_TARGET_RANGE);
        } else {
            z = sg / XY; y = sg / X - z * Y; x = sg % X;
        }
    }
    tgt[g] = make_float4((float)x, (float)y, (float)z, (float)(x * x + y * y + z * z));
}

__global__ void nal_finalize(const double* __restrict__ part, int splits, int t_phys, int t,
                             double prefactor, double* __restrict__ out) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= t) return;
    double s = 0.0;
    for (int sp = 0; sp < splits; ++sp) s += part[(size_t)sp * t_phys + g];
    out[g] = prefactor * s;
}

}  // namespace

extern "C" lgm_status lgm_coulomb_kernel2_noalloc(int32_t grid_x, int32_t grid_y, int32_t grid_z,
                                                  int32_t cutoff, double prefactor,
                                                  const int32_t* d_s, const int32_t* d_q,
                                                  int32_t n, int32_t total, double* d_o,
                                                  void* stream) {
    if (grid_x < 1 || grid_y < 1 || grid_z < 1 || cutoff < 1 || cutoff > 1000 ||
        !std::isfinite(prefactor) || n < 0 || total < 0 || n > total)
        return LGM_ERR_INVALID_ARGUMENT;
    if (n > LGM_NOALLOC_MAX_SOURCES || total > LGM_NOALLOC_MAX_TARGETS) return LGM_ERR_CAPACITY;
    const long long L = std::max<long long>({grid_y, grid_z + 1, (long long)grid_x});
    if (6 * L * L >= (1LL << 22) || (long long)grid_x * grid_y * grid_z + kNalDrainIds > INT32_MAX)
        return LGM_ERR_UNSUPPORTED;
    if (total == 0) return LGM_OK;
    if (!d_s || !d_q || !d_o) return LGM_ERR_INVALID_ARGUMENT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return LGM_ERR_NO_DEVICE;
    ContextSetup S;
    lgm_status st = setup_context(dev, &S);
    if (st != LGM_OK) return st;

    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    float4* geo = reinterpret_cast<float4*>(S.base + kGeoOff);
    float2* qq = reinterpret_cast<float2*>(S.base + kQqOff);
    float4* tgt = reinterpret_cast<float4*>(S.base + kTgtOff);
    double* part = reinterpret_cast<double*>(S.base + kPartOff);
    unsigned* err = reinterpret_cast<unsigned*>(S.base + kErrOff);
    const int XY = grid_x * grid_y, volume = XY * grid_z;
    const int t_phys = (total + 63) / 64 * 64;

    if (cudaMemsetAsync(err, 0, sizeof(unsigned), cs) != cudaSuccess) return LGM_ERR_CUDA;
    // The target records, with the range check of every target, also when
    // there are no sources (the potentials are then all zero).
    if (launch(nal_prep_targets, dim3((t_phys + 255) / 256), dim3(256), 0, cs,
               d_s, (int)total, t_phys, (int)grid_x, (int)grid_y, XY, volume, tgt, err) !=
        cudaSuccess)
        return LGM_ERR_CUDA;
    if (n == 0) {
        if (cudaMemsetAsync(d_o, 0, sizeof(double) * total, cs) != cudaSuccess) return LGM_ERR_CUDA;
    } else {
        const int n_pad = (n + CH - 1) / CH * CH;
        const int n_chunks = n_pad / CH;
        const int tiles = (t_phys + kNalTile - 1) / kNalTile;
        const int splits = std::max(
            1, std::min({kNalMaxSplits, S.sm_count * std::max(1, S.blocks_per_sm) / tiles,
                         n_chunks}));
        if (launch(nal_prep_sources, dim3((n_pad + 255) / 256), dim3(256), 0, cs, d_s, d_q,
                   (int)n, n_pad, (int)grid_x, (int)grid_y, XY, volume, geo, qq, err) !=
            cudaSuccess)
            return LGM_ERR_CUDA;
        PairArgs A;
        A.geo = geo; A.qq = qq; A.n_chunks = n_chunks; A.splits = splits;
        A.tgt = tgt; A.t_phys = t_phys; A.part = part;
        A.c2 = (float)(cutoff * cutoff);
        A.tab = nullptr; A.tab_k = 0;  // point charges, MUFU path: no table
        A.err = err;
        if (launch(kNalPair, dim3(tiles, splits), dim3(kNalThreads), pair_smem_bytes(0), cs, A) !=
                cudaSuccess ||
            launch(nal_finalize, dim3((total + 255) / 256), dim3(256), 0, cs,
                   (const double*)part, splits, t_phys, (int)total, prefactor, d_o) != cudaSuccess)
            return LGM_ERR_CUDA;
    }

    // The call returns once its work is done: the device error word is read
    // back on `stream`.
    unsigned h_err = 0;
    if (cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
        cudaStreamSynchronize(cs) != cudaSuccess)
        return LGM_ERR_CUDA;
    if (h_err & DEVERR_TIMEOUT) return LGM_ERR_TIMEOUT;
    if (h_err & (DEVERR_SOURCE_RANGE | DEVERR_TARGET_RANGE)) return LGM_ERR_OUT_OF_RANGE;
    return h_err ? LGM_ERR_STATE : LGM_OK;
}
