// noalloc.cu -- calRHS for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc: host frameworks that
// reserve the device's memory for their own allocator at start-up (a memory
// pool, a serving runtime with a fixed budget) and hand a plugin only buffers
// they allocated -- an allocation behind their back either fails, because the
// pool holds the memory, or breaks their accounting.
// nuosc_calrhs_noalloc serves them: the caller passes the input and output
// state (and the velocity quadrature) in its own device memory, and the one
// piece of scratch the right-hand side needs -- the 12 velocity moments per
// (x,z) cell -- lives in the file-scope device array below, sized for grids
// of up to NUOSC_NOALLOC_MAX_CELLS cells.  Every GPU that loads the library
// holds that array (6 MiB) until the process exits.
//
// The kernels are the library's own moment pass and direct stage kernel
// (kernels.cu), unchanged; only the scratch pointer differs.
#include "../../include/nuosc_b200.h"
#include "internal.cuh"

#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace nuosc {
namespace {

// 12 moments per cell for at most NUOSC_NOALLOC_MAX_CELLS cells
static __device__ __align__(256) double g_noalloc_moments[(size_t)NUOSC_NOALLOC_MAX_CELLS * NMOM];

// The array's device address belongs to a CUDA context: the primary context
// of a device gets a new one after cudaDeviceReset, and a host framework that
// makes its own context on the same device gets its own copy of the array.
// So the address is looked up once per context (keyed by the context's
// process-unique id, cuCtxGetId) and cached.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
constexpr size_t kMaxContexts = 64;
std::mutex g_mu;
std::vector<std::pair<unsigned long long, double *>> g_scratch;  // (context id, array address)

int fail(int code, const char *msg) { return set_last_error(code, msg); }

template <typename F>
F driver_fn(const char *name) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return (F)p;
}

// id of the calling thread's current context; the runtime's primary context
// of the current device is made current first when none is
bool current_context_id(unsigned long long *id) {
    static const CtxGetCurrentFn get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return false;
    if (!ctx) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return false;
        if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    }
    return get_id(ctx, id) == CUDA_SUCCESS;
}

}  // namespace
}  // namespace nuosc

using namespace nuosc;

extern "C" int nuosc_calrhs_noalloc(const nuosc_rhs_desc *d, const void *in, void *out, void *stream) {
    if (!d || !in || !out) return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: null argument");
    if (d->nx < 4 || d->nz < 4 || d->nv < 1 || d->nv_stride < d->nv)
        return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: bad geometry");
    if (!(d->dx > 0.0) || !(d->dz > 0.0) || !std::isfinite(d->dx) || !std::isfinite(d->dz) || !std::isfinite(d->ko) ||
        !std::isfinite(d->mu) || !std::isfinite(d->pmo))
        return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: bad spacing or coefficient (dx, dz > 0; ko, mu, pmo finite)");
    if ((long long)d->nx * d->nz > NUOSC_NOALLOC_MAX_CELLS)
        return fail(NUOSC_ERR_INVALID,
                    "calrhs_noalloc: nx*nz exceeds NUOSC_NOALLOC_MAX_CELLS (65536) cells of device scratch");
    if (d->precision != NUOSC_FP64 && d->precision != NUOSC_FP32)
        return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: precision must be NUOSC_FP64 or NUOSC_FP32");
    if (d->ko_order != 6 && d->ko_order != 4) return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: ko_order must be 6 or 4");
    if (!d->vx || !d->vy || !d->vz || !d->vw) return fail(NUOSC_ERR_INVALID, "calrhs_noalloc: null quadrature");

    // device address of the scratch array in the current context: looked up
    // on the first call in that context (with its device current) and cached;
    // that first call should come before any stream capture begins
    unsigned long long ctx = 0;
    if (!current_context_id(&ctx)) return fail(NUOSC_ERR_CUDA, "calrhs_noalloc: no current CUDA context");
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        for (const auto &e : g_scratch)
            if (e.first == ctx) scratch = e.second;
        if (!scratch) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_moments);
            if (e != cudaSuccess) return fail(NUOSC_ERR_CUDA, "calrhs_noalloc: cudaGetSymbolAddress failed");
            if (g_scratch.size() >= kMaxContexts) g_scratch.clear();  // entries of contexts that are gone
            g_scratch.emplace_back(ctx, (double *)p);
            scratch = (double *)p;
        }
    }

    Geom g;
    g.nx = d->nx;
    g.nz = d->nz;
    g.nv = d->nv;
    g.nvs = d->nv_stride;
    g.ncell = (long long)d->nx * d->nz;
    g.fs = g.ncell * d->nv_stride;
    const bool ko6 = d->ko_order == 6;
    Coeffs c{};
    c.fxs = -1.0 / (12 * d->dx);
    c.fzs = -1.0 / (12 * d->dz);
    c.kx = ko6 ? -d->ko / d->dx / 64.0 : -d->ko / d->dx / 16.0;
    c.kz = ko6 ? -d->ko / d->dz / 64.0 : -d->ko / d->dz / 16.0;
    const double theta = 37 * M_PI / 180.;
    c.ct = std::cos(2 * theta);
    c.st = std::sin(2 * theta);
    c.mu = d->mu;
    c.pmo = d->pmo;
    const Quad q{d->vx, d->vy, d->vz, d->vw};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (d->precision == NUOSC_FP64) {
        StageArgs<double> a{};
        a.in = (const double *)in;
        a.acc_dst = (double *)out;
        a.mom_in = scratch;
        a.q = q;
        a.g = g;
        a.c = c;
        a.cA = 1.0;
        e = launch_moments<double>(a.in, scratch, q, g, s);
        if (e == cudaSuccess) e = launch_stage_direct<double>(a, MODE_RHS, ko6, s);
    } else {
        StageArgs<float> a{};
        a.in = (const float *)in;
        a.acc_dst = (float *)out;
        a.mom_in = scratch;
        a.q = q;
        a.g = g;
        a.c = c;
        a.cA = 1.0;
        e = launch_moments<float>(a.in, scratch, q, g, s);
        if (e == cudaSuccess) e = launch_stage_direct<float>(a, MODE_RHS, ko6, s);
    }
    if (e != cudaSuccess) return fail(NUOSC_ERR_CUDA, cudaGetErrorString(e));
    return NUOSC_OK;
}
