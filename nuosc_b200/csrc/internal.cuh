// internal.cuh -- device-side data layout, kernel argument blocks and launch
// entry points shared by the CUDA kernels and the C-ABI host layer.
//
// HBM layout of one register (a FieldVar of the reference): 8 fields, each
// [x][z][v] with the velocity innermost and `nvs` velocities per (x,z) row
// (nv rounded up so every row starts on a 16-byte boundary).  No ghost cells
// are stored: the stencils wrap x and z periodically in-kernel, which is what
// updatePeriodicBoundary's ghost fill amounts to for the plus-shaped stencil
// (nuosc_boundary.cpp:4-52).  Padding velocities carry zero weight, zero
// velocity and zero state, so every kernel may process them and they stay 0.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nuosc {

constexpr int NF = 8;  // ee, mm, emr, emi, bee, bmm, bemr, bemi

// Seeded draws of the initial data: a counter-based hash (splitmix64
// finaliser) of (seed, i, j), uniform in [0, 1) with 53 bits; host and device
// give the same value.  Replaces the reference's rand() (nuosc_init.cpp:5, 33).
__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ inline double seeded_uniform(uint64_t seed, int i, int j) {
    const uint64_t key = ((uint64_t)(uint32_t)i << 32) | (uint64_t)(uint32_t)j;
    return (double)(mix64(mix64(seed) ^ key) >> 11) * 0x1.0p-53;
}
constexpr int NMOM = 12;  // emRm[4], emIp[4], eemm[4] (nuosc_class.cpp:28-31)

struct Geom {
    int nx, nz, nv, nvs;
    long long fs;     // elements per field = nx*nz*nvs
    long long ncell;  // nx*nz
};

// Physics coefficients of calRHS (nuosc_class.cpp:112-183, nuosc_class.h:120-122).
struct Coeffs {
    double fxs, fzs;  // advection: factor_x = vx * fxs, fxs = -1/(12 dx) (same for z)
    double kx, kz;    // KO strength: -ko/dx/64 (6th difference) or -ko/dx/16 (4th)
    double mu, pmo, ct, st;
    // KO weights of the symmetric sums s_k = x[-k] + x[+k] and of the centre,
    // per axis, for the fused stencil of the x-march kernel:
    //   6th difference: k3 = eps, k2 = -6 eps, k1 = 15 eps, centre -20 (eps_x + eps_z)
    //   4th difference: k3 = 0,   k2 = eps,    k1 = -4 eps, centre   6 (eps_x + eps_z)
    double kz3, kz2, kz1, kx3, kx2, kx1, kc;
};

struct Quad {
    const double *vx, *vy, *vz, *vw;  // [nvs], zero in the padding
};

// One RK stage: k = L(in); then, by mode,
//   MODE_RHS : acc_dst = k
//   MODE_S1  : acc_dst = in + cA*k ;          y_dst = in + cY*k
//   MODE_S23 : acc_dst = acc_src + cA*k ;     y_dst = u  + cY*k
//   MODE_S4  : acc_dst = acc_src + cA*k
// (the classic 16-pass sequence of the direct and cp.async paths), and the
// 12-pass sequence of the TMA path:
//   MODE_S1Y : y_dst = in + cY*k                       (Y2 = U + dt/2 k1)
//   MODE_S2B : y_dst = u + cY*k ; acc_dst = (u + in) + cA*k
//                                   (Y3 = U + dt/2 k2, B = U + Y2 + dt k2)
//   MODE_SY  : y_dst = u + cY*k                        (Y4 = U + dt k3)
//   MODE_S4B : acc_dst = (acc_src + in)/3 + cA*k
// In S4B, in = Y4, acc_src = B and cA = dt/6: (B + Y4)/3 = U + dt/6 k1 +
// dt/3 k2 + dt/3 k3, so the update is U + dt/6 (k1 + 2 k2 + 2 k3 + k4)
// without reading U.
enum StageMode {
    MODE_RHS = 0, MODE_S1 = 1, MODE_S23 = 2, MODE_S4 = 3, MODE_S1Y = 5, MODE_SY = 6, MODE_S4B = 7, MODE_S2B = 8
};

template <typename T>
struct StageArgs {
    const T *in;
    const T *u;
    const T *acc_src;
    T *acc_dst;
    T *y_dst;
    const double *mom_in;  // [ncell][12] moments of `in`
    double *mom_part;      // x-march: per-(cell, v-block, half) partial moments of the new state
    Quad q;
    Geom g;
    Coeffs c;
    double cA, cY;
    int *status;           // device status word (bounded waits)
    // test of the TMA kernels' bounded waits (0 in normal use): the first
    // front box of the instance's first tile declares this many bytes more
    // than its copies deliver, so every wait on it runs out
    unsigned fault_tx;
    // x-slab of a domain-decomposed solve (nullptr: the stencil wraps x
    // periodically inside the register): the R planes on each side of the
    // slab, [8 fields][2R planes][nz][nvs], planes 0..R-1 left of plane 0 and
    // R..2R-1 right of plane nx-1, filled by the halo exchange before the stage
    const T *halo;
};

// element offset of plane p in [-R, 0) or [nx, nx + R) of field F (0..7) in a
// slab's halo buffer
__host__ __device__ inline long long halo_offset(int F, int p, int nx, int R, long long P) {
    const int hp = p < 0 ? p + R : p - nx + R;
    return ((long long)F * 2 * R + hp) * P;
}

// ---------------------------------------------------------------- launches
// halt (null by default): a batch member's stop flag; when set, nothing is done
template <typename T>
cudaError_t launch_moments(const T *reg, double *mom, Quad q, Geom g, cudaStream_t s, const int *halt = nullptr);
template <typename T>
cudaError_t launch_stage_direct(const StageArgs<T> &a, int mode, bool ko6, cudaStream_t s);

// x-march kernel: tile shape chosen by the autotuner (tile.cu)
struct XTile {
    int tz;        // z rows per CTA
    int lx;        // x planes marched per CTA
    int vb;        // velocities per CTA (32)
    int kind = 0;  // preferred x-march kernel from the tile table: 2 cp.async, 3 TMA, 0 either
    int msum = 1;  // FP32 TMA march: moment partials summed in FP64 (1) or in float within a block (0)
};
template <typename T>
bool xmarch_supported(const Geom &g, bool ko6, XTile t);
template <typename T>
cudaError_t launch_stage_xmarch(const StageArgs<T> &a, int mode, bool ko6, XTile t, cudaStream_t s);
// TMA-fed variant of the x-march kernel (xtma.cu); needs nz % tz == 0
template <typename T>
bool xtma_supported(const Geom &g, XTile t);
template <typename T>
cudaError_t launch_stage_xtma(const StageArgs<T> &a, int mode, bool ko6, XTile t, cudaStream_t s);
// velocity blocks of the TMA kernel's moment partials (32 velocities per block in FP64, 64 in FP32)
template <typename T>
int xtma_num_vblocks(const Geom &g);
// Batched TMA stage (xtma.cu): one persistent launch runs one RK stage of many
// instances.  Each instance has an entry (its tensor maps and StageArgs) in a
// device table; the CTAs of a persistent grid take the tiles of all
// instances from an atomic work-list cursor.
// Tile k of an instance is the tile its own launch runs as CTA k, so each
// instance gets the same bits as when stepped alone.
template <typename T>
size_t xtma_batch_item_bytes();
// Encodes the table entry of one instance into `item` (host memory,
// xtma_batch_item_bytes bytes); returns the instance's tile count, or -1 when
// the instance cannot run with this tz.
template <typename T>
long long xtma_batch_fill(void *item, const StageArgs<T> &a, bool ko6, int tz, int lx);
// CTAs of a persistent launch on `device` (also sets the kernel's dynamic
// shared-memory limit); -1 on failure.  vac: some instance has pmo != 0;
// m64: FP32 moment partials summed in FP64 (XTile::msum; FP64 always is).
template <typename T>
int xtma_batch_grid(int mode, bool ko6, int tz, bool vac, bool m64, int device);
// starts[i] = tiles of instances 0..i-1 (instances ordered as the caller
// wants them served); grid = xtma_batch_grid(...); *counter must be 0 at the
// launch (the work-list cursor); halt[i] != 0 (halt may be null): instance i
// has stopped, its tiles are skipped
template <typename T>
cudaError_t launch_stage_xtma_batch(const void *items, const long long *starts, int n, long long ntiles,
                                    unsigned long long *counter, const int *halt, int mode, bool ko6, int tz,
                                    bool vac, bool m64, int grid, cudaStream_t s);
// Tail of the TMA x-march stage (tail.cu): when the last velocity block of
// the TMA kernel would hold at most a quarter block of real velocities, the
// velocities from xtma_tail_v0 on are computed by a one-thread-per-(cell,
// velocity) kernel that writes the last block's moment partials; the TMA
// kernel then runs the full blocks only.  Returns nvs when there is no tail.
template <typename T>
int xtma_tail_v0(const Geom &g);
int tail_lanes(int width);  // lanes per cell: width rounded up to a power of 2
template <typename T>
cudaError_t launch_stage_tail(const StageArgs<T> &a, int mode, bool ko6, int v0, int nvb, cudaStream_t s);
template <typename T>
struct TailItem {
    StageArgs<T> a;
    int v0, twp, nvb;
    int member;  // the instance's index in the batch (its halt flag)
};
// starts[i]: first thread of item i (ranges of 2 * ncell * twp threads, one
// per (cell, flavour half, tail lane), each rounded up to a multiple of 32);
// total: threads of all items; halt as for launch_stage_xtma_batch
template <typename T>
cudaError_t launch_stage_tail_batch(const TailItem<T> *items, const long long *starts, int n, long long total,
                                    const int *halt, int mode, bool ko6, cudaStream_t s);
// moment_finalize of many instances in one launch (xmarch.cu); starts[i] =
// sum over instances 0..i-1 of ncell * 12
struct FinalizeItem {
    const double *part;
    double *mom;
    long long ncell;
    int nvb;
};
cudaError_t launch_moment_finalize_batch(const FinalizeItem *items, const long long *starts, int n, long long total,
                                         const int *halt, cudaStream_t s);
// *halt = step when *halt is 0 and the analysis sums `sums` (launch_analysis's
// out) meet the reference's stop criterion: a non-finite value or
// max||P|-1| >= 10 (nuosc_ana.cpp:131) (kernels.cu)
cudaError_t launch_halt_check(const double *sums, int *halt, int step, cudaStream_t s);
// value a kernel writes into StageArgs::status when a bounded wait expires
constexpr int NUOSC_TIMEOUT_CODE = 1;
// one warp waits `spins` polls on an mbarrier that never completes, then sets
// *status = NUOSC_TIMEOUT_CODE (xtma.cu; the self-test of the bounded waits)
cudaError_t launch_wait_selftest(int *status, unsigned spins, cudaStream_t s);

// records msg as the calling thread's nuosc_last_error() and returns code (capi.cu)
int set_last_error(int code, const char *msg);
int xmarch_num_vblocks(const Geom &g, XTile t);
cudaError_t launch_moment_finalize(const double *part, double *mom, Geom g, int nvb, cudaStream_t s);

template <typename T>
cudaError_t launch_init(T *reg, const double *G0, const double *G0b, Geom g, int ipt, double eps0,
                        double sigma, double z0, double dz, uint64_t seed, const double *zprof, int xoff,
                        cudaStream_t s);
// Analysis partial sums; `part` holds ANA_BLOCKS * ANA_NQ doubles, `out` ANA_NQ.
constexpr int ANA_NQ = 12;
constexpr int ANA_BLOCKS = 296;
template <typename T>
cudaError_t launch_analysis(const T *reg, const double *G0, const double *G0b, const double *vw, Geom g,
                            double *part, double *out, cudaStream_t s);
template <typename T>
cudaError_t launch_gather(const T *reg, int field, const int *xidx, int sx, const int *vidx, int sv,
                          const double *G0, const double *G0b, Geom g, double *out, cudaStream_t s);
template <typename T>
cudaError_t launch_import(T *reg_field, const double *src, Geom g, int layout, int gx, int gz, cudaStream_t s);
template <typename T>
cudaError_t launch_export(const T *reg_field, double *dst, Geom g, int layout, int gx, int gz, cudaStream_t s);
template <typename T>
cudaError_t launch_vectorize(T *dst, const T *a, double c, const T *b, const T *d, Geom g, cudaStream_t s);
template <typename T>
cudaError_t launch_renormalize(T *reg, const double *G0, const double *G0b, Geom g, cudaStream_t s,
                               const int *halt = nullptr);

}  // namespace nuosc
