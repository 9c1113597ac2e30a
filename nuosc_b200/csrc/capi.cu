// capi.cu -- the C ABI of include/nuosc_b200.h: handle, device memory,
// stage sequencing of step_rk4, analysis and snapshot I/O.
//
// Register roles inside step_rk4 (classic RK4 of nuosc_class.cpp:374-427,
// rearranged so each stage is one fused pass):
//   U = v_stat, A = v_rhs (accumulator), Ya = v_pre, Yb = v_cor
//   S1: k1 = L(U)  ; A = U + dt/6 k1 ; Ya = U + dt/2 k1
//   S2: k2 = L(Ya) ; A = A + dt/3 k2 ; Yb = U + dt/2 k2
//   S3: k3 = L(Yb) ; A = A + dt/3 k3 ; Ya = U + dt   k3
//   S4: k4 = L(Ya) ; U = A + dt/6 k4
// which is U + dt/6 (k1 + 2k2 + 2k3 + k4), the reference's update, with
// 16 state passes per step instead of the reference's 4 calRHS + 6 vectorize
// (the direct and cp.async paths).  The TMA path folds the stages' sums into
// one stored register B (registers U = v_stat, Y2 and Y4 = v_pre, Y3 =
// v_cor, B = v_rhs):
//   S1: k1 = L(U)  ; Y2 = U + dt/2 k1                           2 passes
//   S2: k2 = L(Y2) ; Y3 = U + dt/2 k2 ; B = U + Y2 + dt k2      4
//   S3: k3 = L(Y3) ; Y4 = U + dt k3                             3
//   S4: k4 = L(Y4) ; U = (B + Y4)/3 + dt/6 k4                   3
// (B + Y4)/3 = U + dt/6 k1 + dt/3 k2 + dt/3 k3, so S4 needs no read of U:
// 12 state passes per step.
#include "../../include/nuosc_b200.h"
#include "internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <list>
#include <mutex>
#include <string>
#include <vector>

namespace nuosc {
void icosahedron(int nn, std::vector<double> &vx, std::vector<double> &vy, std::vector<double> &vz,
                 std::vector<double> &vw);
int icosahedron_count(int nn);
XTile autotune_lookup(int nv, int precision);
}  // namespace nuosc

using namespace nuosc;

namespace {
thread_local std::string g_err;
}  // namespace

int nuosc::set_last_error(int code, const char *msg) {
    g_err = msg;
    return code;
}

namespace {

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) return fail(NUOSC_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                           \
    } while (0)

struct Snapshot {
    std::vector<int> fields;
    std::string fntpl;
    int every;
    std::vector<int> xidx, vidx;
};

}  // namespace

struct nuosc_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int precision = NUOSC_FP64;
    size_t esize = 8;
    int gx = 3, gz = 3;
    bool ko6 = true;
    Geom g{};
    double x0 = 0, x1 = 0, z0 = 0, z1 = 0, dx = 0, dz = 0, cfl = 0, ko = 0;
    double dt = 0, ds_L = 0, phy_time = 0;
    double mu = 1.0, pmo = 0.1;  // NuOsc's defaults (nuosc_class.h:124-125)
    bool renorm = false;
    double n_nue0[2] = {0, 0};
    int kernel = NUOSC_KERNEL_AUTO;
    XTile tile{16, 64, 32};
    long long launches = 0;
    bool mom_valid = false;  // d_mom holds the moments of v_stat
    unsigned fault_tx = 0;   // self-test of the TMA kernels' bounded waits (nuosc_selftest_overdeclare_tx)
    // x-slab of a domain-decomposed solve (nuosc_create_slab): slab `rank` of
    // `px`, global planes xoff .. xoff+nx-1 of nx_global; halo = the R planes
    // on each side ([8][2R][nz][nvs]) that the halo exchange fills
    int px = 1, rank = 0, xoff = 0, nx_global = 0;
    void *halo = nullptr;
    size_t halo_bytes = 0;
    long long steps_done = 0;  // RK4 steps since the initial data
    nuosc_batch *batch = nullptr;  // the live batch this handle belongs to

    std::vector<double> vx, vy, vz, vw, G0, G0b;  // host copies (length nv)
    void *reg[4] = {nullptr, nullptr, nullptr, nullptr};
    double *d_quad = nullptr;  // vx | vy | vz | vw | G0 | G0b, each nvs
    double *d_mom = nullptr;   // [ncell][12]
    double *d_part = nullptr;  // x-march partial moments
    size_t part_bytes = 0;
    double *d_ana = nullptr;   // analysis partials + final
    double h_ana[ANA_NQ] = {0};  // analysis read-back
    int *d_status = nullptr;
    double *d_stage = nullptr; // host-layout staging
    size_t stage_bytes = 0;
    int *d_idx = nullptr;      // snapshot index staging
    size_t idx_cap = 0;
    double *d_gather = nullptr;
    size_t gather_bytes = 0;
    size_t device_bytes = 0;

    std::ofstream anafile;
    std::list<Snapshot> snapshots;

    // event-pair profiling of the step kernels (nuosc_set_profiling)
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    double prof_ms[NUOSC_PROF_KINDS] = {0};
    long long prof_n[NUOSC_PROF_KINDS] = {0};

    cudaEvent_t take_event() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    // record a begin event; returns the pending slot (or -1 when profiling is off)
    int prof_begin(int kind) {
        if (!prof_on) return -1;
        cudaEvent_t a = take_event(), b = take_event();
        cudaEventRecord(a, stream);
        ev_pending.push_back({kind, {a, b}});
        return (int)ev_pending.size() - 1;
    }
    void prof_end(int slot) {
        if (slot >= 0) cudaEventRecord(ev_pending[slot].second.second, stream);
    }
    void prof_collect() {
        for (auto &p : ev_pending) {
            float ms = 0;
            cudaEventSynchronize(p.second.second);
            cudaEventElapsedTime(&ms, p.second.first, p.second.second);
            prof_ms[p.first] += ms;
            prof_n[p.first] += 1;
            ev_pool.push_back(p.second.first);
            ev_pool.push_back(p.second.second);
        }
        ev_pending.clear();
    }

    Quad quad() const {
        const int s = g.nvs;
        return Quad{d_quad, d_quad + s, d_quad + 2 * s, d_quad + 3 * s};
    }
    const double *dG0() const { return d_quad + 4 * g.nvs; }
    const double *dG0b() const { return d_quad + 5 * g.nvs; }
    Coeffs coeffs() const {
        Coeffs c;
        c.fxs = -1.0 / (12 * dx);
        c.fzs = -1.0 / (12 * dz);
        c.kx = ko6 ? -ko / dx / 64.0 : -ko / dx / 16.0;
        c.kz = ko6 ? -ko / dz / 64.0 : -ko / dz / 16.0;
        const double theta = 37 * M_PI / 180.;  // nuosc_class.h:120
        c.ct = std::cos(2 * theta);
        c.st = std::sin(2 * theta);
        c.mu = mu;
        c.pmo = pmo;
        if (ko6) {
            c.kz3 = c.kz; c.kz2 = -6 * c.kz; c.kz1 = 15 * c.kz;
            c.kx3 = c.kx; c.kx2 = -6 * c.kx; c.kx1 = 15 * c.kx;
            c.kc = -20 * (c.kz + c.kx);
        } else {
            c.kz3 = 0; c.kz2 = c.kz; c.kz1 = -4 * c.kz;
            c.kx3 = 0; c.kx2 = c.kx; c.kx1 = -4 * c.kx;
            c.kc = 6 * (c.kz + c.kx);
        }
        return c;
    }
};

namespace {

bool valid_reg(int r) { return r >= 0 && r < 4; }

// Device memory of handles and batches comes from the device's default
// stream-ordered pool (cudaMallocAsync), whose release threshold is raised
// once per device so that freed blocks stay in the pool for the next handle:
// a server that creates and destroys solves all the time then neither pays
// for cudaMalloc nor stalls the device in cudaFree.  nuosc_release_cached_memory
// returns the pool's unused blocks to the device.
cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static std::vector<int> done;
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), device) == done.end()) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        done.push_back(device);
    }
    return pool;
}

// bytes the device can still give: free memory plus the pool's unused blocks
size_t device_available(int device) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if (cudaMemPool_t pool = device_pool(device)) {
        uint64_t reserved = 0, used = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
        if (reserved > used) free_b += (size_t)(reserved - used);
    }
    return free_b;
}

// pool allocation, complete (usable from any stream) on return
cudaError_t dev_alloc(void **p, size_t bytes, int device, cudaStream_t s) {
    device_pool(device);
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

// back to the pool once the work queued on s is done
void dev_free(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

int ensure(void **p, size_t *cap, size_t bytes, nuosc_handle *h) {
    if (*cap >= bytes) return 0;
    if (*p) {
        dev_free(*p, h->stream);
        h->device_bytes -= *cap;
    }
    *p = nullptr;
    *cap = 0;
    CUDA_TRY(dev_alloc(p, bytes, h->device, h->stream));
    *cap = bytes;
    h->device_bytes += bytes;
    return 0;
}

int prof_kind(int mode) {
    switch (mode) {
    case MODE_S1: return 0;
    case MODE_S1Y: return 0;
    case MODE_S23: return 1;
    case MODE_SY: return 6;
    case MODE_S2B: return 1;
    case MODE_S4: return 2;
    case MODE_S4B: return 2;
    default: return 3;
    }
}

// one RK4 stage in the direct path: moments of `in`, then the fused stencil
template <typename T>
int run_stage_direct(nuosc_handle *h, int mode, int in, int u, int acc_src, int acc_dst, int y_dst, double cA,
                     double cY) {
    StageArgs<T> a{};
    a.in = (const T *)h->reg[in];
    a.u = u >= 0 ? (const T *)h->reg[u] : nullptr;
    a.acc_src = acc_src >= 0 ? (const T *)h->reg[acc_src] : nullptr;
    a.acc_dst = (T *)h->reg[acc_dst];
    a.y_dst = y_dst >= 0 ? (T *)h->reg[y_dst] : nullptr;
    a.mom_in = h->d_mom;
    a.q = h->quad();
    a.g = h->g;
    a.c = h->coeffs();
    a.cA = cA;
    a.cY = cY;
    a.status = h->d_status;
    if (!(mode == MODE_S1 && in == NUOSC_REG_STAT && h->mom_valid)) {
        const int ps = h->prof_begin(4);
        CUDA_TRY(launch_moments<T>((const T *)h->reg[in], h->d_mom, a.q, h->g, h->stream));
        h->prof_end(ps);
        h->launches++;
    }
    const int ps = h->prof_begin(prof_kind(mode));
    CUDA_TRY(launch_stage_direct<T>(a, mode, h->ko6, h->stream));
    h->prof_end(ps);
    h->launches++;
    return 0;
}

// one RK4 stage in the x-march path (moments of the stage output fused)
template <typename T>
int run_stage_xmarch(nuosc_handle *h, bool tma, const XTile &tile, int mode, int in, int u, int acc_src, int acc_dst,
                     int y_dst, double cA, double cY) {
    StageArgs<T> a{};
    a.in = (const T *)h->reg[in];
    a.u = u >= 0 ? (const T *)h->reg[u] : nullptr;
    a.acc_src = acc_src >= 0 ? (const T *)h->reg[acc_src] : nullptr;
    a.acc_dst = acc_dst >= 0 ? (T *)h->reg[acc_dst] : nullptr;
    a.y_dst = y_dst >= 0 ? (T *)h->reg[y_dst] : nullptr;
    a.mom_in = h->d_mom;
    a.mom_part = h->d_part;
    a.q = h->quad();
    a.g = h->g;
    a.c = h->coeffs();
    a.cA = cA;
    a.cY = cY;
    a.status = h->d_status;
    a.fault_tx = tma ? h->fault_tx : 0u;
    a.halo = tma ? (const T *)h->halo : nullptr;
    if (!h->mom_valid) {
        const int ps = h->prof_begin(4);
        CUDA_TRY(launch_moments<T>((const T *)h->reg[in], h->d_mom, a.q, h->g, h->stream));
        h->prof_end(ps);
        h->launches++;
    }
    int ps = h->prof_begin(prof_kind(mode));
    if (tma) {
        CUDA_TRY(launch_stage_xtma<T>(a, mode, h->ko6, tile, h->stream));
        const int v0 = xtma_tail_v0<T>(h->g);
        if (v0 < h->g.nvs) {  // the nearly empty last velocity block
            CUDA_TRY(launch_stage_tail<T>(a, mode, h->ko6, v0, xtma_num_vblocks<T>(h->g), h->stream));
            h->launches++;
        }
    } else {
        CUDA_TRY(launch_stage_xmarch<T>(a, mode, h->ko6, tile, h->stream));
    }
    h->prof_end(ps);
    ps = h->prof_begin(5);
    const int nvb = tma ? xtma_num_vblocks<T>(h->g) : xmarch_num_vblocks(h->g, tile);
    CUDA_TRY(launch_moment_finalize(h->d_part, h->d_mom, h->g, nvb, h->stream));
    h->prof_end(ps);
    h->launches += 2;
    h->mom_valid = true;  // d_mom now holds the moments of the register this stage wrote
    return 0;
}

// stage-kernel path for this handle: 0 direct, 1 cp.async x-march, 2 TMA x-march (-1: unsupported request).
// `tile` is the handle's tile, with 8-row tiles in place of 16-row ones when
// nz only fits those (the TMA kernel is preferred at either height).
template <typename T>
int stage_path(nuosc_handle *h, XTile &tile) {
    tile = h->tile;
    if (!xtma_supported<T>(h->g, tile) && tile.tz == 16) {
        XTile t8 = tile;
        t8.tz = 8;
        if (xtma_supported<T>(h->g, t8)) tile = t8;
    }
    const bool tma = xtma_supported<T>(h->g, tile), cpa = xmarch_supported<T>(h->g, h->ko6, h->tile);
    switch (h->kernel) {
    case NUOSC_KERNEL_DIRECT: return 0;
    case NUOSC_KERNEL_XMARCH: return cpa ? 1 : -1;
    case NUOSC_KERNEL_XTMA: return tma ? 2 : -1;
    default:
        if (h->tile.kind == NUOSC_KERNEL_XMARCH && cpa) return 1;
        return tma ? 2 : cpa ? 1 : 0;
    }
}

// end of an RK4 step: renormalisation (nuosc_ana.cpp:140-166) and the counters
template <typename T>
int finish_step(nuosc_handle *h) {
    if (h->renorm) {
        CUDA_TRY(launch_renormalize<T>((T *)h->reg[0], h->dG0(), h->dG0b(), h->g, h->stream));
        h->launches++;
        h->mom_valid = false;
    }
    h->phy_time += h->dt;
    h->steps_done++;
    return 0;
}

// the stencil input register of stage k of the 12-pass TMA step
constexpr int kStageInput[4] = {0, 2, 3, 2};

// stage k (0..3) of the 12-pass TMA step (registers 0 U, 2 Y2 then Y4, 3 Y3,
// 1 B); the step ends with stage 3
template <typename T>
int tma_stage(nuosc_handle *h, const XTile &tile, int k) {
    const double dt = h->dt;
    int rc;
    switch (k) {
    case 0: rc = run_stage_xmarch<T>(h, true, tile, MODE_S1Y, 0, -1, -1, -1, 2, 0.0, 0.5 * dt); break;
    case 1: rc = run_stage_xmarch<T>(h, true, tile, MODE_S2B, 2, 0, -1, 1, 3, dt, 0.5 * dt); break;
    case 2: rc = run_stage_xmarch<T>(h, true, tile, MODE_SY, 3, 0, -1, -1, 2, 0.0, dt); break;
    default: rc = run_stage_xmarch<T>(h, true, tile, MODE_S4B, 2, -1, 1, 0, -1, dt / 6.0, 0.0); break;
    }
    if (rc || k < 3) return rc;
    return finish_step<T>(h);
}

// The halo pieces of stage k's input of one slab: per field, its first and
// last R planes (sent to the left / right neighbour) and the places of the
// neighbours' planes in the halo buffer.
void halo_pieces(const nuosc_handle *h, int k, nuosc_halo *o) {
    const int R = h->ko6 ? 3 : 2;
    const long long P = (long long)h->g.nz * h->g.nvs;
    char *reg = (char *)h->reg[kStageInput[k]], *halo = (char *)h->halo;
    for (int f = 0; f < NF; ++f) {
        o->send_lo[f] = reg + (f * h->g.fs) * (long long)h->esize;
        o->send_hi[f] = reg + (f * h->g.fs + (long long)(h->g.nx - R) * P) * (long long)h->esize;
        o->recv_lo[f] = halo + halo_offset(f, -R, h->g.nx, R, P) * (long long)h->esize;
        o->recv_hi[f] = halo + halo_offset(f, h->g.nx, h->g.nx, R, P) * (long long)h->esize;
    }
    o->bytes = (size_t)R * P * h->esize;
    o->left = (h->rank - 1 + h->px) % h->px;
    o->right = (h->rank + 1) % h->px;
}

// Halo exchange of n slabs of one solve held by this process on one device
// (slab i's neighbours are i-1 and i+1, periodic): every copy runs on slab
// 0's stream after all slabs' queued work, and every slab's stream waits for
// the copies, so no stage overwrites a register a copy still reads.
int halo_exchange_local(nuosc_handle *const *s, int n, int k) {
    cudaStream_t cs = s[0]->stream;
    std::vector<cudaEvent_t> evs;
    auto event_on = [&](cudaStream_t st) -> cudaEvent_t {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        evs.push_back(e);
        if (cudaEventRecord(e, st) != cudaSuccess) return nullptr;
        return e;
    };
    int rc = 0;
    for (int i = 1; i < n && !rc; ++i) {
        cudaEvent_t e = event_on(s[i]->stream);
        if (!e || cudaStreamWaitEvent(cs, e, 0) != cudaSuccess) rc = fail(NUOSC_ERR_CUDA, "halo exchange: event");
    }
    for (int i = 0; i < n && !rc; ++i) {
        nuosc_halo me, lo, hi;
        halo_pieces(s[i], k, &me);
        halo_pieces(s[(i - 1 + n) % n], k, &lo);
        halo_pieces(s[(i + 1) % n], k, &hi);
        for (int f = 0; f < NF && !rc; ++f) {
            if (cudaMemcpyAsync(me.recv_lo[f], lo.send_hi[f], me.bytes, cudaMemcpyDeviceToDevice, cs) != cudaSuccess ||
                cudaMemcpyAsync(me.recv_hi[f], hi.send_lo[f], me.bytes, cudaMemcpyDeviceToDevice, cs) != cudaSuccess)
                rc = fail(NUOSC_ERR_CUDA, "halo exchange: copy");
        }
    }
    if (!rc) {
        cudaEvent_t e = event_on(cs);
        for (int i = 1; i < n && !rc; ++i)
            if (!e || cudaStreamWaitEvent(s[i]->stream, e, 0) != cudaSuccess)
                rc = fail(NUOSC_ERR_CUDA, "halo exchange: event");
    }
    for (cudaEvent_t e : evs) cudaEventDestroy(e);  // released once complete
    return rc;
}

template <typename T>
int step_impl(nuosc_handle *h, int nsteps) {
    const double dt = h->dt;
    XTile tile;
    const int path = stage_path<T>(h, tile);
    if (path < 0) return fail(NUOSC_ERR_UNSUPPORTED, "the requested stage kernel does not support this geometry/tile");
    const bool xm = path > 0, tma = path == 2;
    if (!tma) tile = h->tile;
    if (h->halo && !tma)
        return fail(NUOSC_ERR_UNSUPPORTED, "x-slabs of a decomposed solve run on the TMA kernel only (nz %% 8 == 0)");
    if (h->halo && h->px > 1)
        return fail(NUOSC_ERR_UNSUPPORTED,
                    "slab %d of %d: step with nuosc_stage and a halo exchange between the stages", h->rank, h->px);
    if (xm) {
        const size_t need = (size_t)h->g.ncell * xmarch_num_vblocks(h->g, h->tile) * 2 * NMOM * sizeof(double);
        if (int rc = ensure((void **)&h->d_part, &h->part_bytes, need, h)) return rc;
    }
    for (int n = 0; n < nsteps; ++n) {
        int rc;
        if (tma) {
            for (int k = 0; k < 4; ++k) {
                nuosc_handle *self = h;  // a single slab is its own neighbour on both sides
                if (h->halo && (rc = halo_exchange_local(&self, 1, k))) return rc;
                if ((rc = tma_stage<T>(h, tile, k))) return rc;
            }
            continue;
        } else if (xm) {
            if ((rc = run_stage_xmarch<T>(h, tma, tile, MODE_S1, 0, -1, -1, 1, 2, dt / 6.0, 0.5 * dt))) return rc;
            if ((rc = run_stage_xmarch<T>(h, tma, tile, MODE_S23, 2, 0, 1, 1, 3, dt / 3.0, 0.5 * dt))) return rc;
            if ((rc = run_stage_xmarch<T>(h, tma, tile, MODE_S23, 3, 0, 1, 1, 2, dt / 3.0, dt))) return rc;
            if ((rc = run_stage_xmarch<T>(h, tma, tile, MODE_S4, 2, -1, 1, 0, -1, dt / 6.0, 0.0))) return rc;
        } else {
            if ((rc = run_stage_direct<T>(h, MODE_S1, 0, -1, -1, 1, 2, dt / 6.0, 0.5 * dt))) return rc;
            h->mom_valid = false;
            if ((rc = run_stage_direct<T>(h, MODE_S23, 2, 0, 1, 1, 3, dt / 3.0, 0.5 * dt))) return rc;
            if ((rc = run_stage_direct<T>(h, MODE_S23, 3, 0, 1, 1, 2, dt / 3.0, dt))) return rc;
            if ((rc = run_stage_direct<T>(h, MODE_S4, 2, -1, 1, 0, -1, dt / 6.0, 0.0))) return rc;
        }
        if (h->renorm) {
            CUDA_TRY(launch_renormalize<T>((T *)h->reg[0], h->dG0(), h->dG0b(), h->g, h->stream));
            h->launches++;
            h->mom_valid = false;
        }
        h->phy_time += dt;
        h->steps_done++;
    }
    return 0;
}

template <typename T>
int stage_impl(nuosc_handle *h, int k) {
    XTile tile;
    if (stage_path<T>(h, tile) != 2)
        return fail(NUOSC_ERR_UNSUPPORTED, "nuosc_stage runs the TMA stage kernel, which does not take this geometry");
    const size_t need = (size_t)h->g.ncell * xmarch_num_vblocks(h->g, h->tile) * 2 * NMOM * sizeof(double);
    if (int rc = ensure((void **)&h->d_part, &h->part_bytes, need, h)) return rc;
    return tma_stage<T>(h, tile, k);
}

template <typename T>
int calrhs_impl(nuosc_handle *h, int out, int in) {
    h->mom_valid = false;
    int rc = run_stage_direct<T>(h, MODE_RHS, in, -1, -1, out, -1, 1.0, 0.0);
    h->mom_valid = false;
    return rc;
}

int check_status(nuosc_handle *h) {
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (st != 0) {
        CUDA_TRY(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
        return fail(NUOSC_ERR_TIMEOUT, "a bounded in-kernel wait expired (status %d)", st);
    }
    return 0;
}

// host spectra G0/G0b (nuosc_init.cpp:74-96)
void compute_spectra(nuosc_handle *h, double alpha, double lnue, double lnueb, double lnuex, double lnuebx) {
    if (lnuex <= 0) lnuex = DBL_MAX;
    if (lnuebx <= 0) lnuebx = DBL_MAX;
    const int nv = h->g.nv;
    std::vector<double> ng(nv), ngb(nv);
    double ing0 = 0, ing1 = 0;
    for (int v = 0; v < nv; ++v) {
        ng[v] = std::exp(-(h->vx[v] - 1.0) * (h->vx[v] - 1.0) / (2.0 * lnuex * lnuex) -
                         (h->vz[v] - 1.0) * (h->vz[v] - 1.0) / (2.0 * lnue * lnue));
        ngb[v] = std::exp(-(h->vx[v] - 1.0) * (h->vx[v] - 1.0) / (2.0 * lnuebx * lnuebx) -
                          (h->vz[v] - 1.0) * (h->vz[v] - 1.0) / (2.0 * lnueb * lnueb));
        ing0 += h->vw[v] * ng[v];
        ing1 += h->vw[v] * ngb[v];
    }
    ing0 = 1.0 / ing0;
    ing1 = 1.0 / ing1;
    h->G0.resize(nv);
    h->G0b.resize(nv);
    for (int v = 0; v < nv; ++v) {
        h->G0[v] = ng[v] * ing0;
        h->G0b[v] = alpha * ngb[v] * ing1;
    }
}

// ipt = 4 spectra (nuosc_init.cpp:8-13, 49-50): G0 = g(vz, lnue), G0b = alpha
// g(vz, lnueb) with g normalised analytically over vz in [-1, 1] (erf), not by
// the quadrature sum of the generic branch
void noc_spectra(nuosc_handle *h, double alpha, double lnue, double lnueb) {
    auto g = [](double v, double sigma) {
        const double v0 = 1.0;
        const double N = sigma * std::sqrt(0.5 * M_PI) *
                         (std::erf((1.0 + v0) / sigma / std::sqrt(2.0)) + std::erf((1.0 - v0) / sigma / std::sqrt(2.0)));
        return std::exp(-(v - v0) * (v - v0) / (2.0 * sigma * sigma)) / N;
    };
    const int nv = h->g.nv;
    h->G0.resize(nv);
    h->G0b.resize(nv);
    for (int v = 0; v < nv; ++v) {
        h->G0[v] = g(h->vz[v], lnue);
        h->G0b[v] = alpha * g(h->vz[v], lnueb);
    }
}

// ipt = 4 perturbation in z (nuosc_init.cpp:28-46): amax = nz/20 Fourier modes
// k = -amax .. amax-1 (k != 0) of amplitude 1e-7/|k| with phases phi[k + amax];
// out[j] = sum cos(2 pi k Z_j / (z0 - z1) + phi), out[nz + j] the same with sin.
// The reference draws the phases with rand(); here phi[m] = 2 pi U(seed, m),
// U the seeded counter hash that ipt = 1 uses per cell, with the second key -1.
std::vector<double> noc_profile(int nz, double z0, double z1, double dz, uint64_t seed) {
    const int amax = nz / 2 / 10;
    std::vector<double> phi(2 * amax + 1), out(2 * (size_t)nz, 0.0);
    for (int m = 0; m <= 2 * amax; ++m) phi[m] = 2.0 * M_PI * seeded_uniform(seed, m, -1);
    const double pi2oL = 2.0 * M_PI / (z0 - z1);
    for (int j = 0; j < nz; ++j) {
        const double Zj = z0 + (j + 0.5) * dz;
        double tr = 0.0, ti = 0.0;
        for (int k = -amax; k < amax; ++k) {
            if (k == 0) continue;
            tr += 1.e-7 / std::abs(k) * std::cos(pi2oL * k * Zj + phi[k + amax]);
            ti += 1.e-7 / std::abs(k) * std::sin(pi2oL * k * Zj + phi[k + amax]);
        }
        out[j] = tr;
        out[nz + j] = ti;
    }
    return out;
}

int upload_spectra(nuosc_handle *h) {
    const int s = h->g.nvs;
    CUDA_TRY(cudaMemsetAsync(h->d_quad + 4 * s, 0, 2 * s * sizeof(double), h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->d_quad + 4 * s, h->G0.data(), h->g.nv * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->d_quad + 5 * s, h->G0b.data(), h->g.nv * sizeof(double), cudaMemcpyHostToDevice,
                             h->stream));
    return 0;
}

template <typename T>
int analysis_raw(nuosc_handle *h, double *q) {
    CUDA_TRY(launch_analysis<T>((const T *)h->reg[0], h->dG0(), h->dG0b(), h->quad().vw, h->g, h->d_ana,
                                h->d_ana + ANA_BLOCKS * ANA_NQ, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->h_ana, h->d_ana + ANA_BLOCKS * ANA_NQ, ANA_NQ * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    memcpy(q, h->h_ana, ANA_NQ * sizeof(double));
    return 0;
}

int analysis_dispatch(nuosc_handle *h, double *q) {
    return h->precision == NUOSC_FP64 ? analysis_raw<double>(h, q) : analysis_raw<float>(h, q);
}

bool host_layout_ok(int layout) { return layout == NUOSC_LAYOUT_COMPACT || layout == NUOSC_LAYOUT_GHOSTED; }
size_t host_field_elems(const nuosc_handle *h, int layout) {
    if (layout == NUOSC_LAYOUT_COMPACT) return (size_t)h->g.ncell * h->g.nv;
    return (size_t)(h->g.nx + 2 * h->gx) * (h->g.nz + 2 * h->gz) * h->g.nv;
}

template <typename T>
int set_state_impl(nuosc_handle *h, int reg, int field, const double *host, int layout) {
    T *dst = (T *)h->reg[reg] + (size_t)field * h->g.fs;
    const size_t n = host_field_elems(h, layout);
    if (sizeof(T) == 8 && layout == NUOSC_LAYOUT_COMPACT && h->g.nvs == h->g.nv) {
        CUDA_TRY(cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    } else {
        if (int rc = ensure((void **)&h->d_stage, &h->stage_bytes, n * sizeof(double), h)) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->d_stage, host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(launch_import<T>(dst, h->d_stage, h->g, layout, h->gx, h->gz, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

template <typename T>
int get_state_impl(nuosc_handle *h, int reg, int field, double *host, int layout) {
    const T *src = (const T *)h->reg[reg] + (size_t)field * h->g.fs;
    const size_t n = host_field_elems(h, layout);
    if (sizeof(T) == 8 && layout == NUOSC_LAYOUT_COMPACT && h->g.nvs == h->g.nv) {
        CUDA_TRY(cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    } else {
        if (int rc = ensure((void **)&h->d_stage, &h->stage_bytes, n * sizeof(double), h)) return rc;
        if (layout == NUOSC_LAYOUT_GHOSTED) {
            // ghost entries are copied back as they were given (zeros for a fresh buffer)
            CUDA_TRY(cudaMemcpyAsync(h->d_stage, host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        }
        CUDA_TRY(launch_export<T>(src, h->d_stage, h->g, layout, h->gx, h->gz, h->stream));
        CUDA_TRY(cudaMemcpyAsync(host, h->d_stage, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

// A snapshot file-name template is a printf format given one int (the step):
// at most one integer conversion (flags, width and precision allowed, no '*'
// and no length modifier), every other '%' written as "%%".
bool step_template_ok(const char *t) {
    int conversions = 0;
    for (const char *p = t; *p; ++p) {
        if (*p != '%') continue;
        if (*++p == '%') continue;
        while (*p && strchr("-+ #0", *p)) ++p;
        while (*p >= '0' && *p <= '9') ++p;
        if (*p == '.')
            for (++p; *p >= '0' && *p <= '9';) ++p;
        if (!*p || !strchr("diuoxX", *p) || ++conversions > 1) return false;
    }
    return true;
}

int write_meta(nuosc_handle *h, const Snapshot &s, bool at_xv) {
    char filename[4096];
    std::string tmp = s.fntpl + ".meta";
    snprintf(filename, sizeof filename, tmp.c_str(), 0);
    std::ofstream out(filename, std::ofstream::out | std::ofstream::trunc);
    if (!out) return fail(NUOSC_ERR_INVALID, "cannot open %s", filename);
    // text layout of addSnapShotAtV / addSnapShotAtXV (nuosc_snapshot.cpp:31-39, 64-72)
    const int sx = (int)s.xidx.size(), sv = (int)s.vidx.size();
    out << h->dt << " " << sx << " " << h->g.nz << " " << sv << std::endl;
    out << h->x0 << " " << h->x1 << std::endl;
    out << h->z0 << " " << h->z1 << std::endl;
    if (at_xv) {
        for (int j = 0; j < h->g.nz; ++j) out << h->z0 + (j + 0.5) * h->dz << " ";
        out << std::endl;
        for (int x : s.xidx) out << h->x0 + (x + 0.5) * h->dx << " ";
        out << std::endl;
    } else {
        for (int i = 0; i < h->g.nx; ++i) out << h->x0 + (i + 0.5) * h->dx << " ";
        out << std::endl;
        for (int j = 0; j < h->g.nz; ++j) out << h->z0 + (j + 0.5) * h->dz << " ";
        out << std::endl;
    }
    for (int v : s.vidx) out << h->vx[v] << " ";
    out << std::endl;
    for (int v : s.vidx) out << h->vy[v] << " ";
    out << std::endl;
    for (int v : s.vidx) out << h->vz[v] << " ";
    out << std::endl;
    return 0;
}

template <typename T>
int gather_impl(nuosc_handle *h, int field, const int *xidx, int sx, const int *vidx, int sv, double *host) {
    const size_t nidx = (size_t)sx + sv;
    if (int rc = ensure((void **)&h->d_idx, &h->idx_cap, nidx * sizeof(int), h)) return rc;
    const size_t n = (size_t)sx * h->g.nz * sv;
    if (int rc = ensure((void **)&h->d_gather, &h->gather_bytes, n * sizeof(double), h)) return rc;
    CUDA_TRY(cudaMemcpyAsync(h->d_idx, xidx, sx * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->d_idx + sx, vidx, sv * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(launch_gather<T>((const T *)h->reg[0], field, h->d_idx, sx, h->d_idx + sx, sv, h->dG0(), h->dG0b(),
                              h->g, h->d_gather, h->stream));
    CUDA_TRY(cudaMemcpyAsync(host, h->d_gather, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return 0;
}

int gather_dispatch(nuosc_handle *h, int field, const int *xidx, int sx, const int *vidx, int sv, double *host) {
    return h->precision == NUOSC_FP64 ? gather_impl<double>(h, field, xidx, sx, vidx, sv, host)
                                      : gather_impl<float>(h, field, xidx, sx, vidx, sv, host);
}

int check_indices(const nuosc_handle *h, const int *fields, int nfields, const int *xidx, int nx_, const int *vidx,
                  int nv_) {
    if (nfields <= 0 || !fields) return fail(NUOSC_ERR_INVALID, "no fields");
    for (int k = 0; k < nfields; ++k)
        if (fields[k] < 0 || fields[k] > 15) return fail(NUOSC_ERR_INVALID, "field id %d out of range", fields[k]);
    for (int k = 0; k < nx_; ++k)
        if (xidx[k] < 0 || xidx[k] >= h->g.nx) return fail(NUOSC_ERR_INVALID, "x index %d out of range", xidx[k]);
    if (nv_ <= 0 || !vidx) return fail(NUOSC_ERR_INVALID, "no velocity indices");
    for (int k = 0; k < nv_; ++k)
        if (vidx[k] < 0 || vidx[k] >= h->g.nv) return fail(NUOSC_ERR_INVALID, "v index %d out of range", vidx[k]);
    return 0;
}

// analysis record from the raw sums of k_analysis (nuosc_ana.cpp:110-117)
void diag_from_sums(const nuosc_handle *h, const double *q, double phy_time, nuosc_diag *o) {
    nuosc_diag d;
    d.phy_time = phy_time;
    d.maxdP = q[0];
    d.surv = q[1] / q[8];
    d.survb = q[2] / q[9];
    d.avgP = q[3] / q[8];
    d.avgPb = q[4] / q[9];
    d.aM0 = std::sqrt(q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) * h->ds_L;
    d.Lex = q[7] * h->ds_L;
    d.ELNe = std::fabs(h->n_nue0[0] * (1.0 - d.surv) - h->n_nue0[1] * (1.0 - d.survb)) / (h->n_nue0[0] + h->n_nue0[1]);
    d.nonfinite = (long long)q[10];
    d.I1 = q[1] / q[8];
    d.I2 = q[11] / q[8];
    *o = d;
}

// the reference stops when max||P|-1| leaves 10 (nuosc_ana.cpp:131)
int diag_check(const nuosc_diag &d) {
    if (d.nonfinite > 0 || !(d.maxdP < 10))
        return fail(NUOSC_ERR_NUMERIC, "state blew up: max||P|-1| = %g, %lld non-finite values", d.maxdP, d.nonfinite);
    return NUOSC_OK;
}

#define HANDLE_CHECK(h)                                                           \
    do {                                                                          \
        if (!(h)) return fail(NUOSC_ERR_INVALID, "null handle");                  \
        cudaError_t e_ = cudaSetDevice((h)->device);                              \
        if (e_ != cudaSuccess) return fail(NUOSC_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_)); \
    } while (0)

#define DISPATCH(h, fn, ...) ((h)->precision == NUOSC_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

}  // namespace

// The box, spacing and coefficients of nuosc_params: finite, positive
// spacing, and cell counts int((x1 - x0)/dx), int((z1 - z0)/dz) below 2^30.
static bool box_ok(const nuosc_params *p) {
    for (double x : {p->x0, p->x1, p->z0, p->z1, p->dx, p->dz, p->cfl, p->ko})
        if (!std::isfinite(x)) return false;
    if (!(p->dx > 0) || !(p->dz > 0) || !(p->x1 > p->x0) || !(p->z1 > p->z0)) return false;
    return (p->x1 - p->x0) / p->dx < 1073741824.0 && (p->z1 - p->z0) / p->dz < 1073741824.0;
}

extern "C" {

const char *nuosc_last_error(void) { return g_err.c_str(); }

int nuosc_velocity_quadrature(int nn, double *vx, double *vy, double *vz, double *vw, int *n_out) {
    if (nn < 1 || nn > 64) return fail(NUOSC_ERR_INVALID, "icosahedron subdivision nn=%d out of range", nn);
    std::vector<double> x, y, z, w;
    icosahedron(nn, x, y, z, w);
    const size_t n = x.size() * sizeof(double);
    if (vx) memcpy(vx, x.data(), n);
    if (vy) memcpy(vy, y.data(), n);
    if (vz) memcpy(vz, z.data(), n);
    if (vw) memcpy(vw, w.data(), n);
    if (n_out) *n_out = (int)x.size();
    return NUOSC_OK;
}

int nuosc_create(const nuosc_params *p, nuosc_handle **out) {
    g_err.clear();
    if (!p || !out) return fail(NUOSC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (p->px != 1 || p->pz != 1)
        return fail(NUOSC_ERR_UNSUPPORTED, "px=%d pz=%d: one solve lives on one GPU (px = pz = 1)", p->px, p->pz);
    if (p->nv < 1 || p->nv > 64) return fail(NUOSC_ERR_INVALID, "icosahedron subdivision nv=%d out of range", p->nv);
    if (p->gx != p->gz || (p->gx != 2 && p->gx != 3))
        return fail(NUOSC_ERR_INVALID, "ghost width gx=%d gz=%d: must be equal and 2 or 3", p->gx, p->gz);
    if (!box_ok(p)) return fail(NUOSC_ERR_INVALID, "bad box, spacing or coefficient (finite; dx, dz > 0)");
    if (p->precision != NUOSC_FP64 && p->precision != NUOSC_FP32)
        return fail(NUOSC_ERR_INVALID, "precision %d", p->precision);
    nuosc_handle *h = new nuosc_handle;
    h->device = p->device;
    h->precision = p->precision;
    h->esize = p->precision == NUOSC_FP64 ? 8 : 4;
    h->gx = p->gx;
    h->gz = p->gz;
    h->ko6 = p->gx == 3;
    h->x0 = p->x0; h->x1 = p->x1; h->z0 = p->z0; h->z1 = p->z1;
    h->dx = p->dx; h->dz = p->dz; h->cfl = p->cfl; h->ko = p->ko;
    const int nx = (int)((p->x1 - p->x0) / p->dx), nz = (int)((p->z1 - p->z0) / p->dz);
    if (nx < 4 || nz < 4) {
        delete h;
        return fail(NUOSC_ERR_INVALID, "grid %dx%d too small (need at least 4x4)", nx, nz);
    }
    h->dt = p->dz * p->cfl;
    h->ds_L = p->dx * p->dz / (p->z1 - p->z0) / (p->x1 - p->x0);
    icosahedron(p->nv, h->vx, h->vy, h->vz, h->vw);
    const int nv = (int)h->vx.size();
    const int align = (int)(16 / h->esize);
    const int nvs = (nv + align - 1) / align * align;
    h->g.nx = nx;
    h->g.nz = nz;
    h->g.nv = nv;
    h->g.nvs = nvs;
    h->g.ncell = (long long)nx * nz;
    h->g.fs = h->g.ncell * nvs;
    h->tile = autotune_lookup(nv, h->precision);

    auto bail = [&](int rc) {
        nuosc_destroy(h);
        return rc;
    };
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "cudaSetDevice(%d): %s", h->device, cudaGetErrorString(e)));
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e)));
    const size_t reg_bytes = (size_t)h->g.fs * NF * h->esize;
    const size_t free_b = device_available(h->device);
    const size_t need = 4 * reg_bytes + (size_t)h->g.ncell * NMOM * 8;
    if (need > free_b)
        return bail(fail(NUOSC_ERR_OOM, "need %.2f GB for 4 state registers, %.2f GB free", need / 1e9, free_b / 1e9));
    for (int r = 0; r < 4; ++r) {
        e = dev_alloc(&h->reg[r], reg_bytes, h->device, h->stream);
        if (e != cudaSuccess) return bail(fail(NUOSC_ERR_OOM, "allocating register %d (%.2f GB): %s", r, reg_bytes / 1e9,
                                               cudaGetErrorString(e)));
        h->device_bytes += reg_bytes;
        cudaMemsetAsync(h->reg[r], 0, reg_bytes, h->stream);
    }
    const size_t small = 6 * (size_t)nvs * sizeof(double) + (size_t)h->g.ncell * NMOM * sizeof(double) +
                         (ANA_BLOCKS + 1) * ANA_NQ * sizeof(double) + 256;
    char *blk = nullptr;
    e = dev_alloc((void **)&blk, small, h->device, h->stream);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_OOM, "allocating work buffers: %s", cudaGetErrorString(e)));
    h->device_bytes += small;
    cudaMemsetAsync(blk, 0, small, h->stream);
    h->d_status = (int *)blk;
    h->d_quad = (double *)(blk + 256);
    h->d_mom = h->d_quad + 6 * nvs;
    h->d_ana = h->d_mom + h->g.ncell * NMOM;
    cudaMemcpyAsync(h->d_quad, h->vx.data(), nv * 8, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_quad + nvs, h->vy.data(), nv * 8, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_quad + 2 * nvs, h->vz.data(), nv * 8, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->d_quad + 3 * nvs, h->vw.data(), nv * 8, cudaMemcpyHostToDevice, h->stream);
    h->G0.assign(nv, 0.0);
    h->G0b.assign(nv, 0.0);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "create: %s", cudaGetErrorString(e)));
    *out = h;
    return NUOSC_OK;
}

int nuosc_create_slab(const nuosc_params *p, int rank, nuosc_handle **out) {
    g_err.clear();
    if (!p || !out) return fail(NUOSC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (p->px < 1 || p->pz != 1 || rank < 0 || rank >= p->px)
        return fail(NUOSC_ERR_INVALID, "slab %d of px=%d pz=%d (x-slabs: pz = 1, 0 <= rank < px)", rank, p->px, p->pz);
    if (!box_ok(p)) return fail(NUOSC_ERR_INVALID, "bad box, spacing or coefficient (finite; dx, dz > 0)");
    const int nxg = (int)((p->x1 - p->x0) / p->dx), R = p->gx;
    const int base = nxg / p->px, rem = nxg % p->px;
    const int nx = base + (rank < rem ? 1 : 0), xoff = rank * base + std::min(rank, rem);
    if (nx < R || nx < 4) return fail(NUOSC_ERR_INVALID, "slab of %d planes (need at least 4 and the ghost width)", nx);
    nuosc_params q = *p;
    q.px = q.pz = 1;
    q.x0 = p->x0 + xoff * p->dx;
    q.x1 = q.x0 + (nx + 0.5) * p->dx;  // int((x1 - x0)/dx) = nx exactly
    nuosc_handle *h = nullptr;
    if (int rc = nuosc_create(&q, &h)) return rc;
    h->x1 = p->x0 + (xoff + nx) * p->dx;
    h->ds_L = p->dx * p->dz / (p->z1 - p->z0) / (p->x1 - p->x0);  // of the whole box (nuosc_class.cpp:461)
    h->px = p->px;
    h->rank = rank;
    h->xoff = xoff;
    h->nx_global = nxg;
    h->halo_bytes = (size_t)NF * 2 * R * h->g.nz * h->g.nvs * h->esize;
    const cudaError_t e = dev_alloc(&h->halo, h->halo_bytes, h->device, h->stream);
    if (e != cudaSuccess) {
        nuosc_destroy(h);
        return fail(NUOSC_ERR_OOM, "slab halo buffer (%.2f MB): %s", h->halo_bytes / 1e6, cudaGetErrorString(e));
    }
    h->device_bytes += h->halo_bytes;
    cudaMemsetAsync(h->halo, 0, h->halo_bytes, h->stream);
    *out = h;
    return NUOSC_OK;
}

int nuosc_get_slab(const nuosc_handle *h, int *px, int *rank, int *xoff, int *nx_global) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (px) *px = h->px;
    if (rank) *rank = h->rank;
    if (xoff) *xoff = h->xoff;
    if (nx_global) *nx_global = h->halo ? h->nx_global : h->g.nx;
    return NUOSC_OK;
}

int nuosc_destroy(nuosc_handle *h) {
    if (!h) return NUOSC_OK;
    if (h->batch) return fail(NUOSC_ERR_INVALID, "destroy: the handle is a member of a live batch");
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->prof_collect();
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->stream) {  // (no stream: nothing was allocated)
        for (int r = 0; r < 4; ++r) dev_free(h->reg[r], h->stream);
        dev_free(h->d_status, h->stream);
        dev_free(h->d_part, h->stream);
        dev_free(h->d_stage, h->stream);
        dev_free(h->d_idx, h->stream);
        dev_free(h->d_gather, h->stream);
        dev_free(h->halo, h->stream);
        cudaStreamDestroy(h->stream);
    }
    if (h->anafile.is_open()) h->anafile.close();
    delete h;
    return NUOSC_OK;
}

int nuosc_set_mu(nuosc_handle *h, double mu) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    h->mu = mu;
    return NUOSC_OK;
}
int nuosc_set_pmo(nuosc_handle *h, double pmo) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    h->pmo = pmo;
    return NUOSC_OK;
}
int nuosc_set_renorm(nuosc_handle *h, int renorm) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    h->renorm = renorm != 0;
    return NUOSC_OK;
}
int nuosc_set_kernel(nuosc_handle *h, int kind) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (kind < NUOSC_KERNEL_AUTO || kind > NUOSC_KERNEL_XTMA) return fail(NUOSC_ERR_INVALID, "kernel kind %d", kind);
    h->kernel = kind;
    h->mom_valid = false;
    return NUOSC_OK;
}
int nuosc_set_tile(nuosc_handle *h, int tz, int lx) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if ((tz != 4 && tz != 8 && tz != 16) || lx < 1)
        return fail(NUOSC_ERR_INVALID, "tile tz=%d lx=%d (tz 4, 8 or 16, lx >= 1)", tz, lx);
    const int nvb_old = xmarch_num_vblocks(h->g, h->tile);
    h->tile.tz = tz;
    h->tile.lx = lx;
    if (xmarch_num_vblocks(h->g, h->tile) != nvb_old) h->mom_valid = false;
    return NUOSC_OK;
}

int nuosc_get_tile(const nuosc_handle *h, int *tz, int *lx) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (tz) *tz = h->tile.tz;
    if (lx) *lx = h->tile.lx;
    return NUOSC_OK;
}

int nuosc_stage(nuosc_handle *h, int k) {
    HANDLE_CHECK(h);
    if (k < 0 || k > 3) return fail(NUOSC_ERR_INVALID, "stage %d (0..3)", k);
    if (h->kernel != NUOSC_KERNEL_AUTO && h->kernel != NUOSC_KERNEL_XTMA)
        return fail(NUOSC_ERR_UNSUPPORTED, "nuosc_stage runs the TMA stage kernel");
    return h->precision == NUOSC_FP64 ? stage_impl<double>(h, k) : stage_impl<float>(h, k);
}

int nuosc_halo_info(const nuosc_handle *h, int k, nuosc_halo *o) {
    if (!h || !o) return fail(NUOSC_ERR_INVALID, "null argument");
    if (!h->halo) return fail(NUOSC_ERR_INVALID, "not a slab (nuosc_create_slab)");
    if (k < 0 || k > 3) return fail(NUOSC_ERR_INVALID, "stage %d (0..3)", k);
    halo_pieces(h, k, o);
    return NUOSC_OK;
}

int nuosc_halo_exchange_local(nuosc_handle *const *s, int n, int k) {
    if (!s || n < 1) return fail(NUOSC_ERR_INVALID, "null argument");
    if (k < 0 || k > 3) return fail(NUOSC_ERR_INVALID, "stage %d (0..3)", k);
    for (int i = 0; i < n; ++i) {
        if (!s[i] || !s[i]->halo) return fail(NUOSC_ERR_INVALID, "member %d is not a slab", i);
        if (s[i]->px != n || s[i]->rank != i || s[i]->device != s[0]->device || s[i]->g.nz != s[0]->g.nz ||
            s[i]->g.nvs != s[0]->g.nvs || s[i]->esize != s[0]->esize || s[i]->ko6 != s[0]->ko6)
            return fail(NUOSC_ERR_INVALID, "slabs must be ranks 0..%d of one solve on one device, in order", n - 1);
    }
    CUDA_TRY(cudaSetDevice(s[0]->device));
    return halo_exchange_local(s, n, k);
}

int nuosc_analysis_sums(nuosc_handle *h, double *q) {
    HANDLE_CHECK(h);
    if (!q) return fail(NUOSC_ERR_INVALID, "null argument");
    return analysis_dispatch(h, q);
}

int nuosc_diag_from_sums(const nuosc_handle *h, const double *q, nuosc_diag *o) {
    if (!h || !q || !o) return fail(NUOSC_ERR_INVALID, "null argument");
    diag_from_sums(h, q, h->phy_time, o);
    return NUOSC_OK;
}

int nuosc_set_n_nue0(nuosc_handle *h, double n0, double n1) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    h->n_nue0[0] = n0;
    h->n_nue0[1] = n1;
    return NUOSC_OK;
}

int nuosc_set_moment_sum(nuosc_handle *h, int msum) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (msum != 0 && msum != 1) return fail(NUOSC_ERR_INVALID, "moment summation %d (0 float in-block, 1 FP64)", msum);
    h->tile.msum = msum;
    return NUOSC_OK;
}

int nuosc_get_moment_sum(const nuosc_handle *h, int *msum) {
    if (!h || !msum) return fail(NUOSC_ERR_INVALID, "null argument");
    *msum = h->precision == NUOSC_FP64 ? 1 : h->tile.msum;
    return NUOSC_OK;
}

int nuosc_moment_error(nuosc_handle *h, double *err) {
    HANDLE_CHECK(h);
    if (!err) return fail(NUOSC_ERR_INVALID, "null argument");
    if (!h->mom_valid) return fail(NUOSC_ERR_INVALID, "moment_error: no moments of v_stat held (run a step first)");
    const size_t n = (size_t)h->g.ncell * NMOM;
    double *tmp = nullptr;
    CUDA_TRY(dev_alloc((void **)&tmp, n * sizeof(double), h->device, h->stream));
    cudaError_t e = h->precision == NUOSC_FP64
                        ? launch_moments<double>((const double *)h->reg[0], tmp, h->quad(), h->g, h->stream)
                        : launch_moments<float>((const float *)h->reg[0], tmp, h->quad(), h->g, h->stream);
    std::vector<double> a(n), b(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a.data(), h->d_mom, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.data(), tmp, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(tmp, h->stream);
    CUDA_TRY(e);
    double d = 0.0, m = 0.0;
    for (size_t i = 0; i < n; ++i) {
        d = std::max(d, std::fabs(a[i] - b[i]));
        m = std::max(m, std::fabs(b[i]));
    }
    *err = m > 0.0 ? d / m : d;
    return NUOSC_OK;
}

int nuosc_set_time(nuosc_handle *h, double t) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    h->phy_time = t;
    return NUOSC_OK;
}

int nuosc_get_geometry(const nuosc_handle *h, nuosc_geometry *o) {
    if (!h || !o) return fail(NUOSC_ERR_INVALID, "null argument");
    o->nx = h->g.nx; o->nz = h->g.nz; o->nv = h->g.nv; o->nv_stride = h->g.nvs;
    o->gx = h->gx; o->gz = h->gz; o->precision = h->precision;
    o->dt = h->dt; o->ds_L = h->ds_L; o->phy_time = h->phy_time;
    o->x0 = h->x0; o->x1 = h->x1; o->z0 = h->z0; o->z1 = h->z1; o->dx = h->dx; o->dz = h->dz;
    o->n_nue0[0] = h->n_nue0[0]; o->n_nue0[1] = h->n_nue0[1];
    o->device_bytes = h->device_bytes;
    return NUOSC_OK;
}

int nuosc_get_velocities(const nuosc_handle *h, double *vx, double *vy, double *vz, double *vw) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    const size_t n = h->vx.size() * sizeof(double);
    if (vx) memcpy(vx, h->vx.data(), n);
    if (vy) memcpy(vy, h->vy.data(), n);
    if (vz) memcpy(vz, h->vz.data(), n);
    if (vw) memcpy(vw, h->vw.data(), n);
    return NUOSC_OK;
}

int nuosc_get_spectra(const nuosc_handle *h, double *G0, double *G0b) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (G0) memcpy(G0, h->G0.data(), h->G0.size() * sizeof(double));
    if (G0b) memcpy(G0b, h->G0b.data(), h->G0b.size() * sizeof(double));
    return NUOSC_OK;
}

int nuosc_set_spectra(nuosc_handle *h, const double *G0, const double *G0b, double n0, double n1) {
    HANDLE_CHECK(h);
    if (!G0 || !G0b) return fail(NUOSC_ERR_INVALID, "null spectra");
    h->G0.assign(G0, G0 + h->g.nv);
    h->G0b.assign(G0b, G0b + h->g.nv);
    h->n_nue0[0] = n0;
    h->n_nue0[1] = n1;
    if (int rc = upload_spectra(h)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return NUOSC_OK;
}

int nuosc_fill_init(nuosc_handle *h, int ipt, double alpha, double eps0, double sigma, double lnue, double lnueb,
                    double lnuex, double lnuebx, uint64_t seed) {
    HANDLE_CHECK(h);
    if (!((ipt >= 0 && ipt <= 4) || ipt == 10 || ipt == 20 || ipt == 30))
        return fail(NUOSC_ERR_UNSUPPORTED, "ipt=%d: supported initial data are ipt 0..4, 10, 20, 30", ipt);
    if (ipt >= 10 && !(sigma > 0.0)) return fail(NUOSC_ERR_INVALID, "ipt=%d needs sigma > 0", ipt);
    std::vector<double> zprof;
    if (ipt == 4) {
        noc_spectra(h, alpha, lnue, lnueb);
        zprof = noc_profile(h->g.nz, h->z0, h->z1, h->dz, seed);
    } else if (ipt >= 10) {  // advection tests: G0 = G0b = 1 (nuosc_init.cpp:168-169)
        h->G0.assign(h->g.nv, 1.0);
        h->G0b.assign(h->g.nv, 1.0);
    } else {
        compute_spectra(h, alpha, lnue, lnueb, lnuex, lnuebx);
    }
    if (int rc = upload_spectra(h)) return rc;
    double *dprof = nullptr;
    if (!zprof.empty()) {
        CUDA_TRY(dev_alloc((void **)&dprof, zprof.size() * sizeof(double), h->device, h->stream));
        CUDA_TRY(cudaMemcpyAsync(dprof, zprof.data(), zprof.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
    }
    cudaError_t e = h->precision == NUOSC_FP64
                        ? launch_init<double>((double *)h->reg[0], h->dG0(), h->dG0b(), h->g, ipt, eps0, sigma, h->z0,
                                              h->dz, seed, dprof, h->xoff, h->stream)
                        : launch_init<float>((float *)h->reg[0], h->dG0(), h->dG0b(), h->g, ipt, eps0, sigma, h->z0,
                                             h->dz, seed, dprof, h->xoff, h->stream);
    if (dprof) {
        cudaStreamSynchronize(h->stream);  // zprof is host memory of this frame
        dev_free(dprof, h->stream);
    }
    CUDA_TRY(e);
    h->mom_valid = false;
    h->phy_time = 0.0;
    h->steps_done = 0;
    double q[ANA_NQ];
    if (int rc = analysis_dispatch(h, q)) return rc;
    h->n_nue0[0] = q[1] * h->ds_L;  // nuosc_init.cpp:116-130
    h->n_nue0[1] = q[2] * h->ds_L;
    return NUOSC_OK;
}

int nuosc_set_state(nuosc_handle *h, int reg, int field, const double *host, int layout) {
    HANDLE_CHECK(h);
    if (!valid_reg(reg) || field < 0 || field >= NF || !host || !host_layout_ok(layout))
        return fail(NUOSC_ERR_INVALID, "set_state: bad register/field/layout");
    if (reg == NUOSC_REG_STAT) h->mom_valid = false;
    return DISPATCH(h, set_state_impl, h, reg, field, host, layout);
}

int nuosc_get_state(nuosc_handle *h, int reg, int field, double *host, int layout) {
    HANDLE_CHECK(h);
    if (!valid_reg(reg) || field < 0 || field >= NF || !host || !host_layout_ok(layout))
        return fail(NUOSC_ERR_INVALID, "get_state: bad register/field/layout");
    return DISPATCH(h, get_state_impl, h, reg, field, host, layout);
}

int nuosc_update_periodic_boundary(nuosc_handle *h, int reg) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (!valid_reg(reg)) return fail(NUOSC_ERR_INVALID, "register %d", reg);
    return NUOSC_OK;
}

int nuosc_calrhs(nuosc_handle *h, int out, int in) {
    HANDLE_CHECK(h);
    if (!valid_reg(out) || !valid_reg(in) || out == in)
        return fail(NUOSC_ERR_INVALID, "calrhs: registers must be distinct and in 0..3");
    int rc = DISPATCH(h, calrhs_impl, h, out, in);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return NUOSC_OK;
}

int nuosc_vectorize(nuosc_handle *h, int dst, int src1, double a, int src2) {
    HANDLE_CHECK(h);
    if (!valid_reg(dst) || !valid_reg(src1) || !valid_reg(src2)) return fail(NUOSC_ERR_INVALID, "vectorize: register");
    if (h->precision == NUOSC_FP64)
        CUDA_TRY(launch_vectorize<double>((double *)h->reg[dst], (const double *)h->reg[src1], a,
                                          (const double *)h->reg[src2], nullptr, h->g, h->stream));
    else
        CUDA_TRY(launch_vectorize<float>((float *)h->reg[dst], (const float *)h->reg[src1], a,
                                         (const float *)h->reg[src2], nullptr, h->g, h->stream));
    if (dst == NUOSC_REG_STAT) h->mom_valid = false;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return NUOSC_OK;
}

int nuosc_vectorize2(nuosc_handle *h, int dst, int src1, double a, int src2, int src3) {
    HANDLE_CHECK(h);
    if (!valid_reg(dst) || !valid_reg(src1) || !valid_reg(src2) || !valid_reg(src3))
        return fail(NUOSC_ERR_INVALID, "vectorize2: register");
    if (h->precision == NUOSC_FP64)
        CUDA_TRY(launch_vectorize<double>((double *)h->reg[dst], (const double *)h->reg[src1], a,
                                          (const double *)h->reg[src2], (const double *)h->reg[src3], h->g,
                                          h->stream));
    else
        CUDA_TRY(launch_vectorize<float>((float *)h->reg[dst], (const float *)h->reg[src1], a,
                                         (const float *)h->reg[src2], (const float *)h->reg[src3], h->g, h->stream));
    if (dst == NUOSC_REG_STAT) h->mom_valid = false;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return NUOSC_OK;
}

int nuosc_step_rk4(nuosc_handle *h, int nsteps) {
    HANDLE_CHECK(h);
    if (nsteps < 0) return fail(NUOSC_ERR_INVALID, "nsteps %d", nsteps);
    int rc = DISPATCH(h, step_impl, h, nsteps);
    if (rc) return rc;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NUOSC_ERR_CUDA, "step_rk4: %s", cudaGetErrorString(e));
    return NUOSC_OK;
}

int nuosc_analysis(nuosc_handle *h, nuosc_diag *o) {
    HANDLE_CHECK(h);
    if (int rc = check_status(h)) return rc;
    double q[ANA_NQ];
    if (int rc = analysis_dispatch(h, q)) return rc;
    nuosc_diag d;
    diag_from_sums(h, q, h->phy_time, &d);
    if (o) *o = d;
    if (h->anafile.is_open()) {
        // nuosc_ana.cpp:126-129 (precision 13 sticks after the first record)
        h->anafile << d.phy_time << std::setprecision(13) << " " << d.maxdP << " " << d.surv << " " << d.survb << " "
                   << d.avgP << " " << d.avgPb << " " << d.aM0 << " " << d.Lex << " " << d.ELNe << " " << std::endl;
    }
    return diag_check(d);
}

long long nuosc_step_count(const nuosc_handle *h) { return h ? h->steps_done : -1; }

int nuosc_open_analysis_file(nuosc_handle *h, const char *path) {
    if (!h || !path) return fail(NUOSC_ERR_INVALID, "null argument");
    if (h->anafile.is_open()) h->anafile.close();
    h->anafile.open(path, std::ofstream::out | std::ofstream::trunc);
    if (!h->anafile) return fail(NUOSC_ERR_INVALID, "cannot open %s", path);
    h->anafile << "### [ phy_time,   1:maxrelP,    2:surv, survb,    4:avgP, avgPb,      6:aM0    7:Lem   8:ELNe]"
               << std::endl;
    return NUOSC_OK;
}

int nuosc_add_snapshot_at_v(nuosc_handle *h, const int *fields, int nfields, const char *fntpl, int every,
                            const int *vidx, int n_vidx) {
    if (!h || !fntpl) return fail(NUOSC_ERR_INVALID, "null argument");
    if (!step_template_ok(fntpl))
        return fail(NUOSC_ERR_INVALID, "snapshot template %s: one integer conversion at most", fntpl);
    if (int rc = check_indices(h, fields, nfields, nullptr, 0, vidx, n_vidx)) return rc;
    Snapshot s;
    s.fields.assign(fields, fields + nfields);
    s.fntpl = fntpl;
    s.every = every;
    for (int i = 0; i < h->g.nx; ++i) s.xidx.push_back(i);
    s.vidx.assign(vidx, vidx + n_vidx);
    if (int rc = write_meta(h, s, false)) return rc;
    h->snapshots.push_back(s);
    return NUOSC_OK;
}

int nuosc_add_snapshot_at_xv(nuosc_handle *h, const int *fields, int nfields, const char *fntpl, int every,
                             const int *xidx, int n_xidx, const int *vidx, int n_vidx) {
    if (!h || !fntpl) return fail(NUOSC_ERR_INVALID, "null argument");
    if (!step_template_ok(fntpl))
        return fail(NUOSC_ERR_INVALID, "snapshot template %s: one integer conversion at most", fntpl);
    if (n_xidx <= 0 || !xidx) return fail(NUOSC_ERR_INVALID, "no x indices");
    if (int rc = check_indices(h, fields, nfields, xidx, n_xidx, vidx, n_vidx)) return rc;
    Snapshot s;
    s.fields.assign(fields, fields + nfields);
    s.fntpl = fntpl;
    s.every = every;
    s.xidx.assign(xidx, xidx + n_xidx);
    s.vidx.assign(vidx, vidx + n_vidx);
    if (int rc = write_meta(h, s, true)) return rc;
    h->snapshots.push_back(s);
    return NUOSC_OK;
}

// ---------------------------------------------------------------- checkpoints
// File layout (native byte order): "NUOSCCK1" | CkHeader | G0[nv] G0b[nv] |
// v_stat: 8 fields x nx x nz x nv_stride elements of the state type, padding
// velocities included | the 12 FP64 cell moments held for v_stat (ncell x
// 12), when mom_valid.  Restoring the moments with the state makes a resumed
// run bit-identical to an uninterrupted one: the next stage reads exactly the
// moments the previous stage's kernel accumulated.
namespace {
struct CkHeader {
    int32_t version, precision, nx, nz, nv, nvs, ghost, renorm, mom_valid, pad;
    int64_t steps_done;
    double x0, x1, z0, z1, dx, dz, dt, ko, mu, pmo, phy_time, n0, n1;
};
const char kCkMagic[8] = {'N', 'U', 'O', 'S', 'C', 'C', 'K', '1'};
constexpr size_t kCkChunk = 256u << 20;  // bytes per staged device <-> host copy

int ck_copy(nuosc_handle *h, FILE *f, char *dev, size_t bytes, bool save, char *stage) {
    for (size_t off = 0; off < bytes; off += kCkChunk) {
        const size_t n = std::min(kCkChunk, bytes - off);
        if (save) {
            CUDA_TRY(cudaMemcpyAsync(stage, dev + off, n, cudaMemcpyDeviceToHost, h->stream));
            CUDA_TRY(cudaStreamSynchronize(h->stream));
            if (fwrite(stage, 1, n, f) != n) return fail(NUOSC_ERR_INVALID, "checkpoint: write failed");
        } else {
            if (fread(stage, 1, n, f) != n) return fail(NUOSC_ERR_INVALID, "checkpoint: file is truncated");
            CUDA_TRY(cudaMemcpyAsync(dev + off, stage, n, cudaMemcpyHostToDevice, h->stream));
            CUDA_TRY(cudaStreamSynchronize(h->stream));
        }
    }
    return 0;
}

int ck_transfer(nuosc_handle *h, FILE *f, bool save, bool moments) {
    char *stage = nullptr;
    CUDA_TRY(cudaMallocHost((void **)&stage, kCkChunk));
    int rc = ck_copy(h, f, (char *)h->reg[0], (size_t)h->g.fs * NF * h->esize, save, stage);
    if (!rc && moments) rc = ck_copy(h, f, (char *)h->d_mom, (size_t)h->g.ncell * NMOM * sizeof(double), save, stage);
    cudaFreeHost(stage);
    return rc;
}
}  // namespace

int nuosc_save_checkpoint(nuosc_handle *h, const char *path) {
    HANDLE_CHECK(h);
    if (!path) return fail(NUOSC_ERR_INVALID, "null path");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (int rc = check_status(h)) return rc;
    CkHeader c{};
    c.version = 1;
    c.precision = h->precision;
    c.nx = h->g.nx; c.nz = h->g.nz; c.nv = h->g.nv; c.nvs = h->g.nvs;
    c.ghost = h->ko6 ? 3 : 2;
    c.renorm = h->renorm;
    c.mom_valid = h->mom_valid;
    c.steps_done = h->steps_done;
    c.x0 = h->x0; c.x1 = h->x1; c.z0 = h->z0; c.z1 = h->z1; c.dx = h->dx; c.dz = h->dz; c.dt = h->dt;
    c.ko = h->ko; c.mu = h->mu; c.pmo = h->pmo; c.phy_time = h->phy_time; c.n0 = h->n_nue0[0]; c.n1 = h->n_nue0[1];
    FILE *f = fopen(path, "wb");
    if (!f) return fail(NUOSC_ERR_INVALID, "cannot open %s", path);
    const bool ok = fwrite(kCkMagic, 1, 8, f) == 8 && fwrite(&c, sizeof c, 1, f) == 1 &&
                    fwrite(h->G0.data(), sizeof(double), h->g.nv, f) == (size_t)h->g.nv &&
                    fwrite(h->G0b.data(), sizeof(double), h->g.nv, f) == (size_t)h->g.nv;
    int rc = ok ? ck_transfer(h, f, true, h->mom_valid) : fail(NUOSC_ERR_INVALID, "checkpoint: write failed");
    if (fclose(f) != 0 && !rc) rc = fail(NUOSC_ERR_INVALID, "checkpoint: closing %s failed", path);
    return rc;
}

int nuosc_load_checkpoint(nuosc_handle *h, const char *path) {
    HANDLE_CHECK(h);
    if (!path) return fail(NUOSC_ERR_INVALID, "null path");
    FILE *f = fopen(path, "rb");
    if (!f) return fail(NUOSC_ERR_INVALID, "cannot open %s", path);
    char magic[8];
    CkHeader c{};
    int rc = 0;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kCkMagic, 8) || fread(&c, sizeof c, 1, f) != 1 || c.version != 1)
        rc = fail(NUOSC_ERR_INVALID, "%s is not a checkpoint of this library", path);
    else if (c.precision != h->precision || c.nx != h->g.nx || c.nz != h->g.nz || c.nv != h->g.nv ||
             c.nvs != h->g.nvs || c.ghost != (h->ko6 ? 3 : 2) || c.dx != h->dx || c.dz != h->dz || c.dt != h->dt ||
             c.ko != h->ko)
        rc = fail(NUOSC_ERR_INVALID, "checkpoint %s: grid %dx%dx%d (precision %d, ghost %d) does not match the handle",
                  path, c.nx, c.nz, c.nv, c.precision, c.ghost);
    if (!rc) {  // the whole file is checked before the handle is touched
        const long long want = 8 + (long long)sizeof c + 2ll * c.nv * (long long)sizeof(double) +
                               (long long)h->g.fs * NF * h->esize +
                               (c.mom_valid ? (long long)h->g.ncell * NMOM * (long long)sizeof(double) : 0);
        const long here = ftell(f);
        long long size = -1;
        if (here >= 0 && fseek(f, 0, SEEK_END) == 0) size = ftell(f);
        if (size != want || fseek(f, here, SEEK_SET) != 0)
            rc = fail(NUOSC_ERR_INVALID, "checkpoint %s: %lld bytes, expected %lld", path, size, want);
    }
    std::vector<double> G0(c.nv > 0 ? c.nv : 0), G0b(G0.size());
    if (!rc && (fread(G0.data(), sizeof(double), G0.size(), f) != G0.size() ||
                fread(G0b.data(), sizeof(double), G0b.size(), f) != G0b.size()))
        rc = fail(NUOSC_ERR_INVALID, "checkpoint: file is truncated");
    if (!rc) {
        const cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = fail(NUOSC_ERR_CUDA, "checkpoint: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        h->G0 = G0;
        h->G0b = G0b;
        rc = upload_spectra(h);
    }
    if (!rc) rc = ck_transfer(h, f, false, c.mom_valid != 0);
    fclose(f);
    if (rc) {
        h->mom_valid = false;
        return rc;
    }
    h->mom_valid = c.mom_valid != 0;
    h->steps_done = c.steps_done;
    h->phy_time = c.phy_time;
    h->n_nue0[0] = c.n0;
    h->n_nue0[1] = c.n1;
    h->mu = c.mu;
    h->pmo = c.pmo;
    h->renorm = c.renorm != 0;
    return NUOSC_OK;
}

int nuosc_check_snapshot(nuosc_handle *h, int t) {
    HANDLE_CHECK(h);
    // like the reference, every registered snapshot is written on each call
    // (the `every` test is commented out at nuosc_snapshot.cpp:89)
    for (const Snapshot &s : h->snapshots) {
        char filename[4096];
        snprintf(filename, sizeof filename, s.fntpl.c_str(), t);
        std::ofstream out(filename, std::ofstream::out | std::ofstream::trunc | std::ofstream::binary);
        if (!out) return fail(NUOSC_ERR_INVALID, "cannot open %s", filename);
        const unsigned tt = (unsigned)t;
        out.write((const char *)&tt, sizeof(unsigned));
        out.write((const char *)&h->phy_time, sizeof(double));
        std::vector<double> buf((size_t)s.xidx.size() * h->g.nz * s.vidx.size());
        for (int f : s.fields) {
            if (int rc = gather_dispatch(h, f, s.xidx.data(), (int)s.xidx.size(), s.vidx.data(), (int)s.vidx.size(),
                                         buf.data()))
                return rc;
            out.write((const char *)buf.data(), buf.size() * sizeof(double));
        }
    }
    return NUOSC_OK;
}

int nuosc_gather(nuosc_handle *h, int field, const int *xidx, int n_xidx, const int *vidx, int n_vidx, double *host) {
    HANDLE_CHECK(h);
    if (!host || n_xidx <= 0 || !xidx) return fail(NUOSC_ERR_INVALID, "gather: bad arguments");
    if (int rc = check_indices(h, &field, 1, xidx, n_xidx, vidx, n_vidx)) return rc;
    return gather_dispatch(h, field, xidx, n_xidx, vidx, n_vidx, host);
}

int nuosc_synchronize(nuosc_handle *h) {
    HANDLE_CHECK(h);
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

void *nuosc_stream(nuosc_handle *h) { return h ? (void *)h->stream : nullptr; }

long long nuosc_kernel_launches(const nuosc_handle *h) { return h ? h->launches : 0; }

int nuosc_set_profiling(nuosc_handle *h, int on) {
    HANDLE_CHECK(h);
    h->prof_collect();
    h->prof_on = on != 0;
    return NUOSC_OK;
}

int nuosc_get_profile(nuosc_handle *h, double *ms, long long *launches, int nkinds) {
    HANDLE_CHECK(h);
    h->prof_collect();
    for (int k = 0; k < nkinds && k < NUOSC_PROF_KINDS; ++k) {
        if (ms) ms[k] = h->prof_ms[k];
        if (launches) launches[k] = h->prof_n[k];
    }
    for (int k = 0; k < NUOSC_PROF_KINDS; ++k) {
        h->prof_ms[k] = 0;
        h->prof_n[k] = 0;
    }
    return NUOSC_OK;
}

}  // extern "C"

// ====================================================================== batch
// Many independent solves stepped together (no counterpart in the reference).
// Per RK stage: one persistent TMA march kernel over the tiles of all members
// (work-list ordered largest member first), then one moment-finalize kernel
// for all members.  One step is captured in a CUDA graph and replayed.

struct nuosc_batch {
    int device = 0;
    int precision = NUOSC_FP64;
    bool ko6 = true;
    int tz = 16;
    bool vac = false;               // some member has a vacuum term (pmo != 0)
    bool m64 = true;                // moment partials summed in FP64 (the members' tile msum; FP64 always)
    std::vector<nuosc_handle *> m;  // service order: largest first
    std::vector<nuosc_handle *> user;  // the caller's order (record member indices)
    std::vector<int> user_index;       // user index of m[i]
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    char *d_buf = nullptr;          // stage tables | tile starts | cell starts | finalize table | cursors
    size_t item_bytes = 0;
    long long *d_starts = nullptr;
    FinalizeItem *d_fin = nullptr;
    unsigned long long *d_counter = nullptr;  // work-list cursors of the 4 stage launches
    char *d_tail = nullptr;         // tail tables (4 stages) | thread starts
    int ntail = 0;                  // members with a tail block
    long long tail_threads = 0;
    long long *d_fstarts = nullptr;
    long long ntiles = 0, nmom = 0, cells = 0, cellv = 0;
    int grid[4] = {0, 0, 0, 0};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> sig;        // member settings the tables were built from
    long long graph_launches = 0, kernel_launches = 0, per_step = 0;
    // device-side stop of failed members: d_halt[i] = step at which member i
    // (service order) met the stop criterion, 0 while it runs; checked every
    // halt_every of its steps and at every streamed record (0: no checks)
    int *d_halt = nullptr;
    int halt_every = 0;
};

namespace {

// RK4 stage k of step_impl's 12-pass TMA sequence: (mode, in, u, acc_src,
// acc_dst, y_dst) with cA = dt / da (da 0: cA = 0) and cY = fy * dt, the same
// expressions as step_impl
struct StageSpec {
    int mode, in, u, acc_src, acc_dst, y_dst;
    double da, fy;
};
constexpr StageSpec kStages[4] = {{MODE_S1Y, 0, -1, -1, -1, 2, 0.0, 0.5},
                                  {MODE_S2B, 2, 0, -1, 1, 3, 1.0, 0.5},
                                  {MODE_SY, 3, 0, -1, -1, 2, 0.0, 1.0},
                                  {MODE_S4B, 2, -1, 1, 0, -1, 6.0, 0.0}};

std::vector<double> batch_signature(const nuosc_batch *b) {
    std::vector<double> s;
    for (const nuosc_handle *h : b->m) {
        s.push_back(h->mu);
        s.push_back(h->pmo);
        s.push_back(h->dt);
        s.push_back(h->tile.lx);
        s.push_back(h->tile.msum);
        s.push_back(h->fault_tx);
        s.push_back(h->renorm ? 1.0 : 0.0);
        s.push_back((double)(uintptr_t)h->d_part);
    }
    return s;
}

void batch_release_graph(nuosc_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// (re)build the device tables and the step graph from the members' current settings
template <typename T>
int batch_build(nuosc_batch *b) {
    const int n = (int)b->m.size();
    // one persistent kernel runs every member: they must sum their moment
    // partials the same way as their own solo launches do
    b->m64 = sizeof(T) == 8 || b->m[0]->tile.msum != 0;
    for (const nuosc_handle *h : b->m)
        if (sizeof(T) == 4 && (h->tile.msum != 0) != b->m64)
            return fail(NUOSC_ERR_UNSUPPORTED, "batch members must share the moment summation (tile msum)");
    CUDA_TRY(cudaStreamSynchronize(b->stream));  // no replay still reads the tables
    batch_release_graph(b);
    for (nuosc_handle *h : b->m) {
        const size_t need = (size_t)h->g.ncell * xmarch_num_vblocks(h->g, h->tile) * 2 * NMOM * sizeof(double);
        if (int rc = ensure((void **)&h->d_part, &h->part_bytes, need, h)) return rc;
    }
    // x-segment length per member: the member's own tile, shortened (halved,
    // largest members first, down to 8 planes) while the whole work-list would
    // give the persistent grid fewer than 8 tiles per CTA -- a few small
    // members alone cannot fill the GPU with full-length segments.  The tile
    // shape does not change any member's result.
    std::vector<int> lxs(n);
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        const long long target = 8LL * sms * (b->tz == 16 ? 1 : 2);
        auto tiles_of = [&](int i, int lx) {
            const Geom &g = b->m[i]->g;
            return (long long)(g.nz / b->tz) * xtma_num_vblocks<T>(g) * 2 * ((g.nx + lx - 1) / lx);
        };
        long long total = 0;
        for (int i = 0; i < n; ++i) {
            lxs[i] = std::min(b->m[i]->tile.lx, b->m[i]->g.nx);  // (the same single segment)
            total += tiles_of(i, lxs[i]);
        }
        while (total < target) {
            int best = -1;
            for (int i = 0; i < n; ++i)
                if (lxs[i] > 8 && (best < 0 || tiles_of(i, lxs[i]) > tiles_of(best, lxs[best]))) best = i;
            if (best < 0) break;
            total -= tiles_of(best, lxs[best]);
            lxs[best] = std::max(8, lxs[best] / 2);
            total += tiles_of(best, lxs[best]);
        }
    }
    b->item_bytes = xtma_batch_item_bytes<T>();
    const size_t tab = 4 * (size_t)n * b->item_bytes;
    std::vector<char> host(tab);
    std::vector<long long> starts(n), fstarts(n);
    std::vector<FinalizeItem> fin(n);
    std::vector<TailItem<T>> tails[4];
    std::vector<long long> tstarts;
    long long tiles = 0, nmom = 0, tthreads = 0;
    for (int i = 0; i < n; ++i) {
        nuosc_handle *h = b->m[i];
        long long ti = -1;
        const int v0 = xtma_tail_v0<T>(h->g);
        if (v0 < h->g.nvs) {
            tstarts.push_back(tthreads);
            const int twp = tail_lanes(h->g.nvs - v0);
            tthreads += (h->g.ncell * 2 * twp + 31) / 32 * 32;
        }
        for (int k = 0; k < 4; ++k) {
            const StageSpec &sp = kStages[k];
            StageArgs<T> a{};
            a.in = (const T *)h->reg[sp.in];
            a.u = sp.u >= 0 ? (const T *)h->reg[sp.u] : nullptr;
            a.acc_src = sp.acc_src >= 0 ? (const T *)h->reg[sp.acc_src] : nullptr;
            a.acc_dst = sp.acc_dst >= 0 ? (T *)h->reg[sp.acc_dst] : nullptr;
            a.y_dst = sp.y_dst >= 0 ? (T *)h->reg[sp.y_dst] : nullptr;
            a.mom_in = h->d_mom;
            a.mom_part = h->d_part;
            a.q = h->quad();
            a.g = h->g;
            a.c = h->coeffs();
            a.cA = sp.da > 0.0 ? h->dt / sp.da : 0.0;
            a.cY = sp.fy == 1.0 ? h->dt : sp.fy * h->dt;
            a.status = h->d_status;
            a.fault_tx = h->fault_tx;
            ti = xtma_batch_fill<T>(&host[((size_t)k * n + i) * b->item_bytes], a, b->ko6, b->tz, lxs[i]);
            if (v0 < h->g.nvs)
                tails[k].push_back(TailItem<T>{a, v0, tail_lanes(h->g.nvs - v0), xtma_num_vblocks<T>(h->g), i});
            if (ti < 0) return fail(NUOSC_ERR_UNSUPPORTED, "batch member %d (%dx%d) cannot run %d-row TMA tiles", i,
                                    h->g.nx, h->g.nz, b->tz);
        }
        starts[i] = tiles;
        tiles += ti;
        fin[i] = FinalizeItem{h->d_part, h->d_mom, h->g.ncell, xtma_num_vblocks<T>(h->g)};
        fstarts[i] = nmom;
        nmom += h->g.ncell * NMOM;
    }
    if (!b->d_buf) {
        const size_t bytes = tab + 2 * (size_t)n * sizeof(long long) + (size_t)n * sizeof(FinalizeItem) + 256;
        CUDA_TRY(dev_alloc((void **)&b->d_buf, bytes, b->device, b->stream));
        size_t off = tab;
        b->d_starts = (long long *)(b->d_buf + off);
        off += (size_t)n * sizeof(long long);
        b->d_fstarts = (long long *)(b->d_buf + off);
        off += (size_t)n * sizeof(long long);
        b->d_fin = (FinalizeItem *)(b->d_buf + off);
        off += (size_t)n * sizeof(FinalizeItem);
        b->d_counter = (unsigned long long *)(b->d_buf + (off + 63) / 64 * 64);
    }
    CUDA_TRY(cudaMemcpyAsync(b->d_buf, host.data(), tab, cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaMemcpyAsync(b->d_starts, starts.data(), n * sizeof(long long), cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaMemcpyAsync(b->d_fstarts, fstarts.data(), n * sizeof(long long), cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaMemcpyAsync(b->d_fin, fin.data(), n * sizeof(FinalizeItem), cudaMemcpyHostToDevice, b->stream));
    b->ntail = (int)tstarts.size();
    b->tail_threads = tthreads;
    if (b->ntail) {
        const size_t tb = 4 * (size_t)b->ntail * sizeof(TailItem<T>);
        if (!b->d_tail)
            CUDA_TRY(dev_alloc((void **)&b->d_tail, tb + (size_t)b->ntail * sizeof(long long), b->device, b->stream));
        for (int k = 0; k < 4; ++k)
            CUDA_TRY(cudaMemcpyAsync(b->d_tail + (size_t)k * b->ntail * sizeof(TailItem<T>), tails[k].data(),
                                     b->ntail * sizeof(TailItem<T>), cudaMemcpyHostToDevice, b->stream));
        CUDA_TRY(cudaMemcpyAsync(b->d_tail + tb, tstarts.data(), b->ntail * sizeof(long long), cudaMemcpyHostToDevice,
                                 b->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(b->stream));  // host staging is freed on return
    b->ntiles = tiles;
    b->nmom = nmom;
    b->vac = false;
    for (const nuosc_handle *h : b->m) b->vac = b->vac || h->pmo != 0.0;
    for (int k = 0; k < 4; ++k) {
        b->grid[k] = xtma_batch_grid<T>(kStages[k].mode, b->ko6, b->tz, b->vac, b->m64, b->device);
        if (b->grid[k] < 1) return fail(NUOSC_ERR_CUDA, "batch: cannot size the persistent stage grid");
    }

    // one step: reset the work-list cursors, 4 x (stage kernel, finalize), renormalisation
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    long long per_step = 0;
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, 4 * sizeof(unsigned long long), b->stream);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        e = launch_stage_xtma_batch<T>(b->d_buf + (size_t)k * n * b->item_bytes, b->d_starts, n, tiles,
                                       b->d_counter + k, b->d_halt, kStages[k].mode, b->ko6, b->tz, b->vac, b->m64,
                                       b->grid[k], b->stream);
        if (e == cudaSuccess && b->ntail) {
            const size_t tb = 4 * (size_t)b->ntail * sizeof(TailItem<T>);
            e = launch_stage_tail_batch<T>((const TailItem<T> *)(b->d_tail + (size_t)k * b->ntail * sizeof(TailItem<T>)),
                                           (const long long *)(b->d_tail + tb), b->ntail, b->tail_threads,
                                           b->d_halt, kStages[k].mode, b->ko6, b->stream);
            per_step++;
        }
        if (e == cudaSuccess) e = launch_moment_finalize_batch(b->d_fin, b->d_fstarts, n, nmom, b->d_halt, b->stream);
        per_step += 2;
    }
    for (int i = 0; i < n; ++i) {
        nuosc_handle *h = b->m[i];
        if (!h->renorm || e != cudaSuccess) continue;
        e = launch_renormalize<T>((T *)h->reg[0], h->dG0(), h->dG0b(), h->g, b->stream, b->d_halt + i);
        if (e == cudaSuccess)
            e = launch_moments<T>((const T *)h->reg[0], h->d_mom, h->quad(), h->g, b->stream, b->d_halt + i);
        per_step += 2;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(NUOSC_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    b->graph = graph;
    CUDA_TRY(cudaGraphInstantiate(&b->exec, graph, 0));
    b->per_step = per_step;
    b->sig = batch_signature(b);
    return 0;
}

template <typename T>
int batch_step_impl(nuosc_batch *b, int nsteps, int every, nuosc_batch_record *out, int max_out, int *n_out) {
    if (every > 0) {  // the records this call streams must fit before anything is launched
        long long need = 0;
        for (const nuosc_handle *h : b->m) need += (h->steps_done + nsteps) / every - h->steps_done / every;
        if (need > max_out)
            return fail(NUOSC_ERR_INVALID, "batch_step_stream: %lld records for a buffer of %d", need, max_out);
    }
    if (batch_signature(b) != b->sig)
        if (int rc = batch_build<T>(b)) return rc;
    // after everything queued on the members' streams
    for (nuosc_handle *h : b->m) {
        CUDA_TRY(cudaEventRecord(b->ev, h->stream));
        CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ev, 0));
    }
    for (nuosc_handle *h : b->m) {
        if (h->mom_valid) continue;
        CUDA_TRY(launch_moments<T>((const T *)h->reg[0], h->d_mom, h->quad(), h->g, b->stream));
        b->kernel_launches++;
        h->mom_valid = true;
    }
    int nrec = 0;
    for (int s = 0; s < nsteps; ++s) {
        CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
        b->graph_launches++;
        b->kernel_launches += b->per_step;
        for (size_t i = 0; i < b->m.size(); ++i) {
            nuosc_handle *h = b->m[i];
            h->phy_time += h->dt;  // as step_impl: dt added once per step
            h->steps_done++;
            const bool rec = every > 0 && h->steps_done % every == 0;
            const bool chk = b->halt_every > 0 && (rec || h->steps_done % b->halt_every == 0);
            if (!rec && !chk) continue;
            if (rec && nrec >= max_out)
                return fail(NUOSC_ERR_INVALID, "batch_step_stream: more than %d records", max_out);
            double *fin = h->d_ana + ANA_BLOCKS * ANA_NQ;
            CUDA_TRY(launch_analysis<T>((const T *)h->reg[0], h->dG0(), h->dG0b(), h->quad().vw, h->g, h->d_ana, fin,
                                        b->stream));
            b->kernel_launches += 2;
            if (chk) {  // the stop test on the device; a failed member's later work is skipped
                CUDA_TRY(launch_halt_check(fin, b->d_halt + i, (int)h->steps_done, b->stream));
                b->kernel_launches++;
            }
            if (!rec) continue;
            // streamed analysis record: the sums land in out[nrec] when the batch stream gets there
            nuosc_batch_record &r = out[nrec++];
            r.member = b->user_index[i];
            r.step = h->steps_done;
            r.phy_time = h->phy_time;
            CUDA_TRY(cudaMemcpyAsync(r.q, fin, ANA_NQ * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
            if (n_out) *n_out = nrec;
        }
    }
    CUDA_TRY(cudaEventRecord(b->ev, b->stream));
    for (nuosc_handle *h : b->m) CUDA_TRY(cudaStreamWaitEvent(h->stream, b->ev, 0));
    return 0;
}

}  // namespace

extern "C" {

int nuosc_batch_create(nuosc_handle *const *members, int n, nuosc_batch **out) {
    g_err.clear();
    if (!members || !out || n < 1) return fail(NUOSC_ERR_INVALID, "batch_create: null argument or empty batch");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        const nuosc_handle *h = members[i];
        if (!h) return fail(NUOSC_ERR_INVALID, "batch member %d is null", i);
        if (h->batch) return fail(NUOSC_ERR_INVALID, "batch member %d already belongs to a batch", i);
        if (h->halo) return fail(NUOSC_ERR_UNSUPPORTED, "batch member %d is an x-slab of a decomposed solve", i);
        for (int j = 0; j < i; ++j)
            if (members[j] == h) return fail(NUOSC_ERR_INVALID, "batch member %d repeats member %d", i, j);
        if (h->device != members[0]->device || h->precision != members[0]->precision || h->ko6 != members[0]->ko6)
            return fail(NUOSC_ERR_UNSUPPORTED, "batch members must share device, precision and ghost width");
    }
    auto tz_ok = [&](int tz) {
        for (int i = 0; i < n; ++i) {
            const nuosc_handle *h = members[i];
            const bool ok = h->precision == NUOSC_FP64 ? xtma_supported<double>(h->g, XTile{tz, 32, 32})
                                                       : xtma_supported<float>(h->g, XTile{tz, 32, 64});
            if (!ok) return false;
        }
        return true;
    };
    nuosc_batch *b = new nuosc_batch;
    b->device = members[0]->device;
    b->precision = members[0]->precision;
    b->ko6 = members[0]->ko6;
    cudaError_t e = cudaSetDevice(b->device);
    if (e != cudaSuccess) {
        delete b;
        return fail(NUOSC_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    b->tz = tz_ok(16) ? 16 : tz_ok(8) ? 8 : 0;
    if (!b->tz) {
        delete b;
        return fail(NUOSC_ERR_UNSUPPORTED, "batch: every member needs nz %% 8 == 0 and nz >= 14");
    }
    b->user.assign(members, members + n);
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
        return members[x]->g.ncell * members[x]->g.nvs > members[y]->g.ncell * members[y]->g.nvs;
    });
    for (int i : idx) {
        b->m.push_back(members[i]);
        b->user_index.push_back(i);
    }
    for (const nuosc_handle *h : b->m) {
        b->cells += h->g.ncell;
        b->cellv += h->g.ncell * h->g.nv;
    }
    auto bail = [&](int rc) {
        nuosc_batch_destroy(b);
        return rc;
    };
    e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e)));
    e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "cudaEventCreate: %s", cudaGetErrorString(e)));
    for (nuosc_handle *h : b->m) {  // the tables read the members' buffers: let pending work finish
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "batch_create: %s", cudaGetErrorString(e)));
    }
    e = dev_alloc((void **)&b->d_halt, n * sizeof(int), b->device, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_halt, 0, n * sizeof(int), b->stream);
    if (e != cudaSuccess) return bail(fail(NUOSC_ERR_CUDA, "batch_create: %s", cudaGetErrorString(e)));
    const int rc = b->precision == NUOSC_FP64 ? batch_build<double>(b) : batch_build<float>(b);
    if (rc) return bail(rc);
    for (nuosc_handle *h : b->m) h->batch = b;
    *out = b;
    return NUOSC_OK;
}

int nuosc_batch_step_stream(nuosc_batch *b, int nsteps, int every, nuosc_batch_record *out, int max_out,
                            int *n_out) {
    if (n_out) *n_out = 0;
    if (!b) return fail(NUOSC_ERR_INVALID, "null batch");
    if (nsteps < 0) return fail(NUOSC_ERR_INVALID, "nsteps %d", nsteps);
    if (every > 0 && (!out || max_out < 0)) return fail(NUOSC_ERR_INVALID, "batch_step_stream: no record buffer");
    CUDA_TRY(cudaSetDevice(b->device));
    const int rc = b->precision == NUOSC_FP64 ? batch_step_impl<double>(b, nsteps, every, out, max_out, n_out)
                                              : batch_step_impl<float>(b, nsteps, every, out, max_out, n_out);
    if (rc) return rc;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NUOSC_ERR_CUDA, "batch_step: %s", cudaGetErrorString(e));
    return NUOSC_OK;
}

int nuosc_batch_step(nuosc_batch *b, int nsteps) { return nuosc_batch_step_stream(b, nsteps, 0, nullptr, 0, nullptr); }

int nuosc_batch_set_halt(nuosc_batch *b, int check_every) {
    if (!b) return fail(NUOSC_ERR_INVALID, "null batch");
    if (check_every < 0) return fail(NUOSC_ERR_INVALID, "batch_set_halt: check_every %d", check_every);
    b->halt_every = check_every;
    return NUOSC_OK;
}

int nuosc_batch_halted(nuosc_batch *b, int *steps, int n) {
    if (!b || !steps) return fail(NUOSC_ERR_INVALID, "null argument");
    if (n != (int)b->m.size())
        return fail(NUOSC_ERR_INVALID, "batch_halted: %d entries for %d members", n, (int)b->m.size());
    CUDA_TRY(cudaSetDevice(b->device));
    std::vector<int> h(n);
    CUDA_TRY(cudaMemcpyAsync(h.data(), b->d_halt, n * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; ++i) steps[b->user_index[i]] = h[i];
    return NUOSC_OK;
}

int nuosc_batch_record_diag(const nuosc_batch *b, const nuosc_batch_record *r, nuosc_diag *d) {
    if (!b || !r || !d) return fail(NUOSC_ERR_INVALID, "null argument");
    if (r->member < 0 || r->member >= (int)b->user.size()) return fail(NUOSC_ERR_INVALID, "record member %d", r->member);
    diag_from_sums(b->user[r->member], r->q, r->phy_time, d);
    return diag_check(*d);
}

void *nuosc_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        fail(NUOSC_ERR_OOM, "cudaMallocHost(%zu) failed", bytes);
        return nullptr;
    }
    return p;
}

void nuosc_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

int nuosc_batch_synchronize(nuosc_batch *b) {
    if (!b) return fail(NUOSC_ERR_INVALID, "null batch");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (nuosc_handle *h : b->m)
        if (int rc = check_status(h)) return rc;
    return NUOSC_OK;
}

int nuosc_batch_get_info(const nuosc_batch *b, nuosc_batch_info *o) {
    if (!b || !o) return fail(NUOSC_ERR_INVALID, "null argument");
    o->n = (int)b->m.size();
    o->tz = b->tz;
    o->ctas = b->grid[1];
    o->tiles = b->ntiles;
    o->cells = b->cells;
    o->cell_velocities = b->cellv;
    o->device_bytes = 0;
    for (const nuosc_handle *h : b->m) o->device_bytes += h->device_bytes;
    o->graph_launches = b->graph_launches;
    o->kernel_launches = b->kernel_launches;
    return NUOSC_OK;
}

void *nuosc_batch_stream(nuosc_batch *b) { return b ? (void *)b->stream : nullptr; }

int nuosc_selftest_wait_timeout(int device, unsigned spins, double *ms) {
    if (spins < 1) return fail(NUOSC_ERR_INVALID, "selftest: spins must be positive");
    CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int *d = nullptr, st = 0;
    float el = 0.f;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = dev_alloc((void **)&d, sizeof(int), device, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) e = launch_wait_selftest(d, spins, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, d, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&el, e0, e1);
    if (d) dev_free(d, s);
    if (s) cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (e != cudaSuccess) return fail(NUOSC_ERR_CUDA, "selftest: %s", cudaGetErrorString(e));
    if (ms) *ms = el;
    if (st != NUOSC_TIMEOUT_CODE) return fail(NUOSC_ERR_INVALID, "selftest: the wait did not expire (status %d)", st);
    return fail(NUOSC_ERR_TIMEOUT, "selftest: the bounded wait expired after %u polls (%.3f ms)", spins, el);
}

int nuosc_selftest_overdeclare_tx(nuosc_handle *h, unsigned extra_bytes) {
    if (!h) return fail(NUOSC_ERR_INVALID, "null handle");
    if (extra_bytes % 16 || extra_bytes > 65536)
        return fail(NUOSC_ERR_INVALID, "overdeclare_tx: %u bytes (a multiple of 16, at most 65536)", extra_bytes);
    h->fault_tx = extra_bytes;
    return NUOSC_OK;
}

int nuosc_release_cached_memory(int device) {
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaDeviceSynchronize());
    if (cudaMemPool_t pool = device_pool(device)) CUDA_TRY(cudaMemPoolTrimTo(pool, 0));
    return NUOSC_OK;
}

int nuosc_batch_destroy(nuosc_batch *b) {
    if (!b) return NUOSC_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_release_graph(b);
    for (nuosc_handle *h : b->m)
        if (h->batch == b) h->batch = nullptr;
    if (b->stream) {
        dev_free(b->d_buf, b->stream);
        dev_free(b->d_tail, b->stream);
        dev_free(b->d_halt, b->stream);
    }
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return NUOSC_OK;
}

}  // extern "C"
