/*
 * nuosc_b200.h -- C ABI of the B200-native nuosc RK4 time step.
 *
 * One handle = one solve on one GPU: the 2D periodic (x,z) box times the
 * icosahedral velocity sphere, with the 8 real fields of rho and rho-bar
 * (ee, mm, Re em, Im em and their barred partners) resident in HBM.  Every
 * entry point returns 0 on success or a NUOSC_ERR_* code; the message of the
 * last failure on the calling thread is available from nuosc_last_error().
 * Device memory is owned by the handle.  Work is ordered on the handle's own
 * CUDA stream; entry points that return host data synchronise that stream.
 *
 * Each declaration names the member of the reference's C++ class NuOsc
 * (chunyulin/nuosc, nuosc_class.h:99-191) that it replaces.  Register ids
 * stand for NuOsc's FieldVar pointers v_stat, v_rhs, v_pre, v_cor
 * (nuosc_class.h:108); field ids follow FieldVar::getAllFields
 * (nuosc_class.h:58-65).
 */
#ifndef NUOSC_B200_H
#define NUOSC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define NUOSC_OK 0
#define NUOSC_ERR_INVALID 1     /* bad argument or call order */
#define NUOSC_ERR_CUDA 2        /* a CUDA runtime call failed */
#define NUOSC_ERR_OOM 3         /* not enough device memory for the request */
#define NUOSC_ERR_NUMERIC 4     /* non-finite state or max||P|-1| >= 10 (nuosc_ana.cpp:131 assert) */
#define NUOSC_ERR_TIMEOUT 5     /* a bounded in-kernel wait expired; the kernel returned early */
#define NUOSC_ERR_UNSUPPORTED 6 /* a configuration this library does not implement */

/* precision of the resident state */
#define NUOSC_FP64 0 /* state and arithmetic in double (the reference's real, common.h:58) */
#define NUOSC_FP32 1 /* state and stencil arithmetic in float; cell moments and diagnostics in double */

/* registers (NuOsc FieldVar pointers) */
#define NUOSC_REG_STAT 0
#define NUOSC_REG_RHS 1
#define NUOSC_REG_PRE 2
#define NUOSC_REG_COR 3

/* fields: 0..7 are the state (FieldVar order); 8..15 are derived per point
 * from the current v_stat as eval_conserved does (nuosc_ana.cpp:8-28) */
#define NUOSC_EE 0
#define NUOSC_MM 1
#define NUOSC_EMR 2
#define NUOSC_EMI 3
#define NUOSC_BEE 4
#define NUOSC_BMM 5
#define NUOSC_BEMR 6
#define NUOSC_BEMI 7
#define NUOSC_P1 8
#define NUOSC_P2 9
#define NUOSC_P3 10
#define NUOSC_P1B 11
#define NUOSC_P2B 12
#define NUOSC_P3B 13
#define NUOSC_DP 14
#define NUOSC_DPB 15

/* host array layouts for state transfer */
#define NUOSC_LAYOUT_COMPACT 0 /* [x][z][v], nx*nz*nv doubles, no ghosts */
#define NUOSC_LAYOUT_GHOSTED 1 /* the reference's array: [(i+gx)*(nz+2gz)+j+gz]*nv+v (CartGrid.h:91) */

/* stage-kernel selection (nuosc_set_kernel) */
#define NUOSC_KERNEL_AUTO 0   /* the TMA x-march kernel when the geometry allows, else the cp.async one */
#define NUOSC_KERNEL_DIRECT 1 /* one thread per (cell, velocity), separate moment pass */
#define NUOSC_KERNEL_XMARCH 2 /* cp.async-staged x-march with fused moments (any geometry) */
#define NUOSC_KERNEL_XTMA 3   /* TMA-fed x-march with mbarrier ring, fused moments (nz % tz == 0) */

typedef struct nuosc_handle nuosc_handle;

/* Constructor arguments of NuOsc::NuOsc (nuosc_class.cpp:454-457). */
typedef struct nuosc_params {
    int px, pz;    /* process grid; must be 1, 1: one solve lives on one GPU */
    int nv;        /* icosahedron subdivision count nn: 10*nn*nn+2 velocities (the reference's --nv) */
    int nphi;      /* unused (polar velocity grid, IM_V2D_POLAR_GRID, is not built) */
    int gx, gz;    /* ghost width: 3 selects the 6th-difference KO (KO_ORD_3 undefined), 2 the 4th-difference KO */
    double x0, x1; /* box [x0, x1) */
    double z0, z1; /* box [z0, z1) */
    double dx, dz; /* nx = int((x1-x0)/dx), nz = int((z1-z0)/dz) (CartGrid.cpp:196-197) */
    double cfl;    /* dt = dz*cfl (nuosc_class.cpp:464) */
    double ko;     /* Kreiss-Oliger strength */
    int precision; /* NUOSC_FP64 or NUOSC_FP32 */
    int device;    /* CUDA device ordinal */
} nuosc_params;

typedef struct nuosc_geometry {
    int nx, nz, nv;     /* interior cells and velocities */
    int nv_stride;      /* velocities per (x,z) row in device memory (nv padded to a 16-byte row) */
    int gx, gz;         /* ghost width given at creation (selects the KO order) */
    int precision;
    double dt, ds_L, phy_time;
    double x0, x1, z0, z1, dx, dz;
    double n_nue0[2];   /* initial number densities (nuosc_init.cpp:129-130) */
    size_t device_bytes; /* device memory held by the handle */
} nuosc_geometry;

/* One analysis() record: the analysis.dat columns (nuosc_ana.cpp:126-129). */
typedef struct nuosc_diag {
    double phy_time, maxdP, surv, survb, avgP, avgPb, aM0, Lex, ELNe;
    long long nonfinite; /* count of non-finite state values seen by the reduction */
    /* the advection test's integrals (printed by the reference when built
     * with ADV_TEST, nuosc_ana.cpp:58-61,121): I1 = sum w ee / nor,
     * I2 = sum w ee^2 / nor, nor = sum w G0 over all cells */
    double I1, I2;
} nuosc_diag;

/* gen_v2d_icosahedron (CartGrid.cpp:46-61, icosahedron.h:36-171): the velocity
 * quadrature for subdivision nn, host only (no GPU needed); arrays hold
 * 10*nn*nn+2 entries.  Returns the count in *n_out when n_out is not null. */
int nuosc_velocity_quadrature(int nn, double *vx, double *vy, double *vz, double *vw, int *n_out);

/* NuOsc::NuOsc (nuosc_class.cpp:454-576) and CartGrid::CartGrid (CartGrid.cpp:122-247) */
int nuosc_create(const nuosc_params *params, nuosc_handle **out);
/* NuOsc::~NuOsc (nuosc_class.h:136-146) */
int nuosc_destroy(nuosc_handle *h);
/* message of the last failed call on this thread ("" if none) */
const char *nuosc_last_error(void);

/* NuOsc::set_mu / set_pmo / set_renorm (nuosc_class.h:148-159) */
int nuosc_set_mu(nuosc_handle *h, double mu);
int nuosc_set_pmo(nuosc_handle *h, double pmo);
int nuosc_set_renorm(nuosc_handle *h, int renorm);
/* stage-kernel choice (NUOSC_KERNEL_*); no counterpart in the reference */
int nuosc_set_kernel(nuosc_handle *h, int kind);
/* x-march tile: tz z-rows per CTA (4, 8 or 16) and lx x-planes marched per CTA.
 * The default comes from the autotuner's table (tiles.txt beside the
 * library, keyed on velocity count and precision).  No reference counterpart. */
int nuosc_set_tile(nuosc_handle *h, int tz, int lx);
int nuosc_get_tile(const nuosc_handle *h, int *tz, int *lx);
/* How the FP32 TMA kernel sums the velocity-moment partials of a 64-velocity
 * block: 1 in FP64 (products of the float state with double weights, double
 * sums; the default, and always so for FP64 state), 0 in float.  The tile
 * table's sixth column holds the autotuner's choice per (nv, precision).
 * No reference counterpart (the reference sums in FP64, nuosc_class.cpp:62-82). */
int nuosc_set_moment_sum(nuosc_handle *h, int msum);
int nuosc_get_moment_sum(const nuosc_handle *h, int *msum);
/* Summation error of the handle's fused cell moments (the ones the last
 * stage's kernel accumulated for v_stat) against an FP64 recomputation from
 * the same stored state: max |fused - FP64| / max |FP64| over all cells and
 * the 12 moments.  The autotuner's accuracy test of the moment summation.
 * Synchronises; needs a step run since the state was last set. */
int nuosc_moment_error(nuosc_handle *h, double *err);

/* grid geometry (CartGrid members) and the velocity quadrature (CartGrid::vx,vy,vz,vw) */
int nuosc_get_geometry(const nuosc_handle *h, nuosc_geometry *out);
int nuosc_get_velocities(const nuosc_handle *h, double *vx, double *vy, double *vz, double *vw);
/* the angular spectra G0, G0b per velocity (NuOsc::G0, G0b; nuosc_init.cpp:95-96) */
int nuosc_get_spectra(const nuosc_handle *h, double *G0, double *G0b);
/* set G0/G0b and n_nue0 directly (for a state supplied with nuosc_set_state) */
int nuosc_set_spectra(nuosc_handle *h, const double *G0, const double *G0b, double n_nue0, double n_nueb0);
/* physical time (NuOsc::phy_time) */
int nuosc_set_time(nuosc_handle *h, double phy_time);

/* NuOsc::fillInitValue (nuosc_init.cpp:17-137), generic branch.  ipt 0: Gaussian
 * eps in z; 1: eps0*U(-1,1) per (x,z) cell from `seed` (replaces rand());
 * 2: eps_p profile; 3: constant eps0.  lnuex/lnuebx <= 0 mean unbounded
 * (the reference default DBL_MAX). */
int nuosc_fill_init(nuosc_handle *h, int ipt, double alpha, double eps0, double sigma, double lnue,
                    double lnueb, double lnuex, double lnuebx, uint64_t seed);

/* direct access to FieldVar arrays (callers of the reference read and write
 * v_stat->ee[...] in place); host arrays of double in the given layout */
int nuosc_set_state(nuosc_handle *h, int reg, int field, const double *host, int layout);
int nuosc_get_state(nuosc_handle *h, int reg, int field, double *host, int layout);

/* NuOsc::updatePeriodicBoundary (nuosc_boundary.cpp:4-52).  The stencil
 * kernels wrap indices periodically, so no ghost cells exist on the device;
 * this validates `reg` and returns. */
int nuosc_update_periodic_boundary(nuosc_handle *h, int reg);

/* NuOsc::calRHS (nuosc_class.cpp:11-307): register out = L(register in) */
int nuosc_calrhs(nuosc_handle *h, int out_reg, int in_reg);
/* NuOsc::vectorize (nuosc_class.cpp:313-351): dst = a1 + a*a2, dst = a1 + a*(a2 + a3) */
int nuosc_vectorize(nuosc_handle *h, int dst, int src1, double a, int src2);
int nuosc_vectorize2(nuosc_handle *h, int dst, int src1, double a, int src2, int src3);
/* NuOsc::step_rk4 (nuosc_class.cpp:374-427), nsteps times; v_stat holds the
 * new state afterwards (the other registers hold stage scratch) */
int nuosc_step_rk4(nuosc_handle *h, int nsteps);

/* NuOsc::analysis (nuosc_ana.cpp:34-137); appends a line to the analysis file
 * when one is open (nuosc_open_analysis_file) */
int nuosc_analysis(nuosc_handle *h, nuosc_diag *out);
/* opens the analysis.dat writer the NuOsc constructor opens (nuosc_class.cpp:536-540) */
int nuosc_open_analysis_file(nuosc_handle *h, const char *path);

/* NuOsc::addSnapShotAtV / addSnapShotAtXV / checkSnapShot (nuosc_snapshot.cpp:13-122).
 * `fields` are NUOSC_* field ids of the current v_stat (0..15).  `fntpl` is a
 * printf format given the step number alone: at most one integer conversion
 * (e.g. "ee%06d.bin"; flags, width and precision allowed, no '*' or length
 * modifier), '%' written as "%%" elsewhere; any other template is refused
 * with NUOSC_ERR_INVALID. */
int nuosc_add_snapshot_at_v(nuosc_handle *h, const int *fields, int nfields, const char *fntpl, int every,
                            const int *vidx, int n_vidx);
int nuosc_add_snapshot_at_xv(nuosc_handle *h, const int *fields, int nfields, const char *fntpl, int every,
                             const int *xidx, int n_xidx, const int *vidx, int n_vidx);
int nuosc_check_snapshot(nuosc_handle *h, int t);

/* ---- spatial domain decomposition: x-slabs ------------------------------
 * Replaces the reference's CartGrid decomposition and halo exchange
 * (CartGrid.cpp:130-200, 330-440; nuosc_boundary.cpp:64-208) for a split in x
 * only (the reference's --np px 1).  nuosc_create_slab makes the handle of
 * slab `rank` of params->px (params->pz must be 1): global box and spacing as
 * in nuosc_create, the handle owns planes [xoff, xoff + nx) of the global nx
 * (nx/px each, the first nx%px slabs one more; at least R = gx planes each),
 * periodic in x across the slabs and in z inside each.  Its stage kernels
 * read the R planes beyond each side from a halo buffer instead of wrapping,
 * so before every RK stage k the buffer must hold the neighbours' planes of
 * stage k's input: nuosc_halo_info lists the 32 pieces (per field, the R
 * planes to send to each neighbour and where each neighbour's arrive), and
 * either the caller moves them (NCCL send/recv between processes, one per
 * GPU) or nuosc_halo_exchange_local copies them between slabs held by one
 * process on one device.  nuosc_stage runs one stage; a step is stages 0..3,
 * each preceded by an exchange.  With px = 1 nuosc_step_rk4 does the
 * exchange itself (the slab is its own neighbour).  Slabs run the TMA stage
 * kernel only (nz % 8 == 0), cannot join a batch, and their analysis is over
 * their own cells: reduce nuosc_analysis_sums over the slabs (sum; max for
 * entry 0) and convert with nuosc_diag_from_sums.  Seeded initial data use
 * the global x index, so every decomposition gives the same solve. */
typedef struct nuosc_halo {
    void *send_lo[8], *send_hi[8]; /* device: the slab's first / last R planes of each field of stage k's input */
    void *recv_lo[8], *recv_hi[8]; /* device: where the left / right neighbour's last / first R planes go */
    size_t bytes;                  /* bytes of each piece (R contiguous planes of one field) */
    int left, right;               /* ranks of the neighbour slabs (periodic in x) */
} nuosc_halo;
int nuosc_create_slab(const nuosc_params *params, int rank, nuosc_handle **out);
int nuosc_get_slab(const nuosc_handle *h, int *px, int *rank, int *xoff, int *nx_global);
int nuosc_stage(nuosc_handle *h, int k);
int nuosc_halo_info(const nuosc_handle *h, int k, nuosc_halo *out);
int nuosc_halo_exchange_local(nuosc_handle *const *slabs, int n, int k);
/* the raw analysis sums of the handle's cells (12 doubles: 0 max |P|-1 over
 * both flavours, 1 sum w ee, 2 sum w bee, 3 sum w G dP, 4 sum w Gb dPb,
 * 5..7 the ELN moments, 8 sum w G, 9 sum w Gb, 10 non-finite count,
 * 11 sum w ee^2), and the diagnostics record of (reduced) sums */
int nuosc_analysis_sums(nuosc_handle *h, double *sums);
int nuosc_diag_from_sums(const nuosc_handle *h, const double *sums, nuosc_diag *out);
/* initial number densities n_nue0 (NuOsc::n_nue0) -- of the whole solve, for slabs */
int nuosc_set_n_nue0(nuosc_handle *h, double n0, double n1);

/* Checkpoint and restart of a solve (no counterpart in the reference, which
 * only writes slices).  save writes v_stat (raw, in the handle's precision),
 * the spectra G0/G0b, time, step count, n_nue0, mu, pmo, renorm and the cell
 * moments held for v_stat; load restores them into a handle created with
 * the same grid, velocity count, precision, ghost width, dt and ko (else
 * NUOSC_ERR_INVALID; a file of another grid or of the wrong size is refused
 * before the handle is changed).  A run stopped after step n, saved, loaded into a new
 * handle and continued is bit-identical to the uninterrupted run.  Both
 * synchronise the handle's stream and stage the state through 256 MB of
 * page-locked host memory. */
int nuosc_save_checkpoint(nuosc_handle *h, const char *path);
int nuosc_load_checkpoint(nuosc_handle *h, const char *path);
/* gather one snapshot block (sx * nz * sv doubles, (i,j,v) order) into host memory */
int nuosc_gather(nuosc_handle *h, int field, const int *xidx, int n_xidx, const int *vidx, int n_vidx,
                 double *host);

/* wait for all work queued on the handle's stream */
int nuosc_synchronize(nuosc_handle *h);
/* the handle's cudaStream_t (as void*), for callers that order their own work after it */
void *nuosc_stream(nuosc_handle *h);
/* number of kernel launches issued by step_rk4/calrhs of this handle so far */
long long nuosc_kernel_launches(const nuosc_handle *h);
/* RK4 steps taken since the initial data (fill_init resets it; -1 for NULL) */
long long nuosc_step_count(const nuosc_handle *h);

/* Device memory of handles and batches comes from the device's default
 * stream-ordered memory pool (cudaMallocAsync), and blocks freed by
 * nuosc_destroy / nuosc_batch_destroy stay in that pool for the next handle
 * (the library raises the pool's release threshold), so that creating and
 * destroying solves neither re-allocates nor stalls the device.  This call
 * waits for the device and returns the pool's unused blocks to it, for
 * callers that need the memory for something else.  No reference
 * counterpart (the reference allocates with new[] once per run). */
int nuosc_release_cached_memory(int device);

/* Self-test of the in-kernel bounded waits (no reference counterpart): one
 * warp waits on an mbarrier that nothing completes, gives up after `spins`
 * polls, records the timeout in a status word and returns, as the stage
 * kernels do when a copy never lands.  Returns NUOSC_ERR_TIMEOUT when the wait
 * expired and was reported (the expected outcome), with the kernel's time in
 * *ms (may be NULL); the device stays usable afterwards. */
int nuosc_selftest_wait_timeout(int device, unsigned spins, double *ms);

/* Self-test of the TMA stage kernels' own timeout path (no reference
 * counterpart).  While extra_bytes > 0 (a multiple of 16, at most 65536),
 * every TMA stage launch of this handle -- solo, or as a batch member --
 * declares extra_bytes more than its copies deliver for one box of the
 * handle's first tile (first z rows, velocity block, x segment and flavour
 * half).  All copies land; that box's full barrier never completes, so every
 * warp's bounded wait on it runs out (about 1 s), the tile stops, records
 * NUOSC_ERR_TIMEOUT in the handle's status word, waits (bounded) for the
 * copies it issued and returns; nothing faults.  nuosc_synchronize /
 * nuosc_batch_synchronize then return NUOSC_ERR_TIMEOUT and the handle's
 * state is undefined until it is set again.  0 switches the test off. */
int nuosc_selftest_overdeclare_tx(nuosc_handle *h, unsigned extra_bytes);

/* Per-kernel timing with CUDA events on the handle's stream (no counterpart
 * in the reference, which prints wall time per step, nuosc.cpp:222-235).
 * Kinds: 0 stage S1, 1 stage S2 (and S3 on the direct and cp.async paths),
 * 2 stage S4, 3 calRHS, 4 moments, 5 moment finalize, 6 stage S3 of the TMA
 * path.  A stage's time includes its tail-kernel launch.  nuosc_get_profile
 * synchronises, fills ms[k] (total milliseconds) and launches[k] for
 * k < nkinds, and resets the counters. */
#define NUOSC_PROF_KINDS 7
int nuosc_set_profiling(nuosc_handle *h, int on);
int nuosc_get_profile(nuosc_handle *h, double *ms, long long *launches, int nkinds);

/* ---- right-hand side without device allocation -------------------------
 * No counterpart in the reference.  For callers that may not call cudaMalloc:
 * host frameworks that reserve the device's memory for their own allocator
 * (a pool sized at start-up, a serving runtime with a fixed budget) and hand
 * a plugin only buffers they allocated; an allocation made behind their back
 * fails when the pool holds the memory, or breaks their accounting.
 * The caller passes everything in its own device memory: `in` and `out` are
 * states laid out like the library's registers, [8 fields][nx][nz][nv_stride]
 * of double (NUOSC_FP64) or float (NUOSC_FP32), padding velocities zero, and
 * the quadrature arrays (nv_stride doubles each, zero in the padding).  The
 * call computes out = L(in), the same right-hand side nuosc_calrhs computes
 * on a handle's registers, on `stream` and allocates nothing: the per-cell
 * velocity moments it needs go to a file-scope device array of
 * NUOSC_NOALLOC_MAX_CELLS * 12 doubles (6 MiB), which every GPU that loads
 * the library holds until the process exits.
 *   - grids with nx*nz > NUOSC_NOALLOC_MAX_CELLS, dx or dz <= 0 and
 *     non-finite coefficients are rejected (NUOSC_ERR_INVALID);
 *   - the first call in a CUDA context (the device's primary context, or a
 *     caller's own) looks up the array's device address in that context
 *     (cudaGetSymbolAddress) with its device current, and caches it per
 *     context; make that first call before any stream capture begins;
 *   - all calls share the one array and it keeps the last call's moments;
 *     each call rewrites every entry it reads, so nothing needs clearing, but
 *     calls that overlap on the GPU (e.g. on two streams at once) race on it.
 * Returns NUOSC_OK once the two kernels are queued; errors are reported by
 * nuosc_last_error(). */
#define NUOSC_NOALLOC_MAX_CELLS 65536
typedef struct nuosc_rhs_desc {
    int nx, nz, nv;     /* interior cells and velocities */
    int nv_stride;      /* velocities per (x,z) row of in/out (>= nv) */
    int precision;      /* NUOSC_FP64 or NUOSC_FP32: element type of in/out */
    int ko_order;       /* 6: 6th-difference KO (reference with KO_ORD_3 undefined), 4: 4th-difference KO */
    double dx, dz, ko, mu, pmo;
    const double *vx, *vy, *vz, *vw; /* device arrays of nv_stride entries */
} nuosc_rhs_desc;
int nuosc_calrhs_noalloc(const nuosc_rhs_desc *desc, const void *in, void *out, void *stream);

/* ---- batched stepping of many independent solves -----------------------
 * No counterpart in the reference, which runs one NuOsc per process
 * (nuosc.cpp:171-240).  A batch steps several handles (instances of possibly
 * different nx, nz, nv, mu, pmo, initial data) together: each RK stage is ONE
 * persistent kernel whose CTAs take tiles of all instances from a work-list
 * (largest instances first), then one moment-finalize kernel for all; the
 * whole step is captured once in a CUDA graph and replayed.  Every instance's
 * result is bit-for-bit the result of nuosc_step_rk4 on that handle alone.
 *   - members share device, precision and ghost width (KO order); every
 *     member needs nz % 8 == 0 and nz >= 14 (the TMA march kernel; nz % 16
 *     == 0 and nz >= 22 for all members selects 16-row tiles);
 *   - a handle belongs to at most one live batch and must outlive it;
 *     members stay usable alone (analysis, snapshots, set_state ...) between
 *     batch steps; nuosc_batch_step orders itself after work queued on the
 *     members' streams and the members' streams after it;
 *   - mu, pmo, renorm and tile changes on a member are picked up at the next
 *     nuosc_batch_step (the work-list is rebuilt). */
typedef struct nuosc_batch nuosc_batch;
typedef struct nuosc_batch_info {
    int n;                     /* instances */
    int tz;                    /* z rows per tile */
    int ctas;                  /* CTAs of each persistent stage launch */
    long long tiles;           /* tiles per stage launch, all instances */
    long long cells;           /* x-z cells, all instances */
    long long cell_velocities; /* sum of nx*nz*nv: the work unit of one step */
    size_t device_bytes;       /* sum of the members' device memory */
    long long graph_launches;  /* step graphs replayed so far */
    long long kernel_launches; /* kernels those replays ran (plus moment passes) */
} nuosc_batch_info;
int nuosc_batch_create(nuosc_handle *const *members, int n, nuosc_batch **out);
/* nsteps RK4 steps of every member (nuosc_step_rk4 on each); asynchronous */
int nuosc_batch_step(nuosc_batch *b, int nsteps);
/* Streamed diagnostics: as nuosc_batch_step, and whenever a member's step
 * count (nuosc_step_count) reaches a multiple of `every`, the analysis of
 * that member is queued on the batch stream right after that step and its raw
 * sums are copied into the next record of `out` -- no host synchronisation.
 * *n_out = records queued; a call whose records would not fit in max_out is
 * refused with NUOSC_ERR_INVALID before any member steps.  Records are
 * complete after nuosc_batch_synchronize.  `out` should be page-locked
 * (nuosc_host_alloc): a pageable buffer makes each copy synchronous.
 * nuosc_batch_record_diag turns a record into the nuosc_diag that
 * nuosc_analysis gives at that step (and its NUOSC_ERR_NUMERIC check). */
typedef struct nuosc_batch_record {
    int member;       /* index into the members array given to nuosc_batch_create */
    int reserved;
    long long step;   /* the member's step count after the step the record follows */
    double phy_time;
    double q[12];     /* raw analysis sums */
} nuosc_batch_record;
int nuosc_batch_step_stream(nuosc_batch *b, int nsteps, int every, nuosc_batch_record *out, int max_out,
                            int *n_out);
int nuosc_batch_record_diag(const nuosc_batch *b, const nuosc_batch_record *r, nuosc_diag *d);
/* Device-side stop of failed members.  The reference stops a run at the
 * analysis whose max||P|-1| reaches 10 (the assert in nuosc_ana.cpp:131);
 * this is that test inside a batch, without a host round trip.  With
 * check_every > 0, every check_every steps of a member -- and at every record
 * nuosc_batch_step_stream streams -- the member's analysis is evaluated on the
 * device, and a member with a non-finite value or max||P|-1| >= 10 stops: the
 * batch's later stage, tail and finalize work skips it, so its state stays as
 * it was at that step (its step counter keeps counting the batch's steps).
 * The other members' results do not change (bit for bit).  check_every 0 (the
 * default) turns the checks off; a member that stopped stays stopped.
 * nuosc_batch_halted synchronises the batch and writes steps[k] = the step at
 * which member k (the order given to nuosc_batch_create; n entries) stopped,
 * 0 while it runs. */
int nuosc_batch_set_halt(nuosc_batch *b, int check_every);
int nuosc_batch_halted(nuosc_batch *b, int *steps, int n);
/* page-locked host memory for record buffers (NULL on failure) */
void *nuosc_host_alloc(size_t bytes);
void nuosc_host_free(void *p);
/* wait for the batch and check every member's in-kernel status word */
int nuosc_batch_synchronize(nuosc_batch *b);
int nuosc_batch_get_info(const nuosc_batch *b, nuosc_batch_info *info);
void *nuosc_batch_stream(nuosc_batch *b);
int nuosc_batch_destroy(nuosc_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* NUOSC_B200_H */
