// xtma.cu -- TMA-fed x-march stage kernel (the fast path of the fused stage).
//
// Same arithmetic and per-thread structure as xmarch.cu (one (z, v) column per
// thread -- two adjacent velocities per thread in FP32 --, a (2R+1)-deep
// register queue in x, fused RK epilogue and moment partials), with
// Blackwell-native data movement:
//   * box ring: for every x plane the CTA touches, lane 0 of warp 0 issues one
//     TMA tensor load (cp.async.bulk.tensor.4d; 2-3 boxes where the periodic z
//     wrap cuts it) of the plane's [TZ+2R rows][4 fields][VB velocities] box
//     and a bulk copy of the TZ cells' moments into a ring slot whose
//     completion is tracked by a "full" mbarrier (expect_tx bytes).  A box is
//     used twice: first as the queue front (x+R), R planes later as the
//     centre plane of the z stencil, so each state value crosses HBM once;
//   * warps never exchange data and there is no CTA-wide barrier in the
//     march: a warp waits only on full barriers and releases a slot after its
//     last use by arriving on the slot's "empty" mbarrier; the issuing lane
//     waits on "empty" before refilling a slot;
//   * the pointwise inputs of the epilogue (U in S2 and S3, U and B in S4;
//     none in S1) are plain coalesced loads issued at the top of each plane,
//     before the waits and the stencil; the issuing lane prefetches their TZ
//     rows into L2 two planes ahead with a tensor prefetch
//     (cp.async.bulk.prefetch.tensor), so the loads find them in L2;
//   * moment partials (FP64 products and sums; FP32 state may sum in float
//     within the block, stored as double): each lane forms its 12 products
//     (3 combinations x 4 weights, the weights in a lane-permuted order set
//     once per tile) and the warp reduce-scatters them over its 32 lanes
//     with 13 shuffle-adds;
//   * a stopped instance of a batch (its halt flag set by the device-side
//     stop test) has its tiles skipped.
// All mbarrier waits are bounded: on expiry the kernel records the timeout in
// the status word, stops marching and, before returning, waits (again
// bounded) for the copies it issued.  Requires nz % TZ == 0.
//
// The march of one tile is a device function shared by two kernels: k_xtma
// (one tile per CTA, one instance per launch) and k_xtma_batch (a persistent
// grid whose CTAs take tiles of many instances from a work-list).
#include "internal.cuh"
#include "physics.cuh"

#include <cuda.h>

#include <cstring>
#include <type_traits>

namespace nuosc {

namespace {

// bounded mbarrier waits: a poll of a phase that has not completed suspends
// the thread for about 4 us on B200 (nuosc_selftest_wait_timeout), so 2^18
// polls give up after about 1 s
constexpr unsigned kWaitSpins = 1u << 18;

// velocities per thread and per CTA: FP32 threads take two adjacent velocities
template <typename T>
constexpr int vpt() {
    return sizeof(T) == 4 ? 2 : 1;
}
template <typename T>
constexpr int vblock() {
    return 32 * vpt<T>();
}

struct __align__(64) TmaMaps {
    CUtensorMap zr;   // box of TZ+2R rows (plane box with both halos)
    CUtensorMap tzr;  // TZ+R rows (a box cut by the wrap)
    CUtensorMap tz;   // TZ rows (middle piece of a box wrapped at both ends)
    CUtensorMap r;    // R rows (wrapped halo)
    CUtensorMap pu;   // TZ rows of the stage's U register (L2 prefetch of the pointwise input)
    CUtensorMap pa;   // TZ rows of the final stage's B input (acc_src; L2 prefetch)
    // the same four box shapes over a slab's halo buffer (planes right of the slab)
    CUtensorMap hzr, htzr, htz, hr;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned spins = kWaitSpins) {
    for (unsigned it = 0; it < spins; ++it) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
// make generic-proxy writes of a tensor map in global memory visible to the TMA
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(m) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
// L2 prefetch of one tensor box: no shared memory, no completion to wait for
__device__ __forceinline__ void tma_prefetch_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];\n" ::"l"(
                     (unsigned long long)map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// VPT consecutive values (8-byte vector access when VPT == 2)
template <typename T, int N>
__device__ __forceinline__ void ldv(const T *p, T (&o)[N]) {
    if constexpr (N == 2) {
        const float2 t = *reinterpret_cast<const float2 *>(p);
        o[0] = t.x;
        o[1] = t.y;
    } else {
        o[0] = *p;
    }
}
template <typename T, int N>
__device__ __forceinline__ void stv(T *p, const T (&o)[N]) {
    if constexpr (N == 2) *reinterpret_cast<float2 *>(p) = make_float2(o[0], o[1]);
    else *p = o[0];
}

constexpr int up128(int x) { return (x + 127) / 128 * 128; }

// one ring slot: box [ZR][4][VB] T | moments [TZ][12] double
template <typename T, int TZ, int R>
struct Slot {
    static constexpr int VB = vblock<T>();
    static constexpr int ZR = TZ + 2 * R;
    static constexpr int box = 0;
    static constexpr int mb = up128(box + (int)sizeof(T) * ZR * 4 * VB);
    static constexpr int bytes = up128(mb + 8 * TZ * NMOM);
    static constexpr unsigned tx = sizeof(T) * ZR * 4 * VB + 8 * TZ * NMOM;  // bytes landing per plane
};

// The stencil of one field at one point, eps_z KO_z + eps_x KO_x + fz ADV_z
// + fx ADV_x with
//   KO  (unit strength) 6th: s[0]+s[6] - 6 (s[1]+s[5]) + 15 (s[2]+s[4]) - 20 s[3]
//                       4th: s[0]+s[4] - 4 (s[1]+s[3]) + 6 s[2]
//   ADV = s[C-2] - s[C+2] - 8 (s[C-1] - s[C+1]) (the 4th-order central
//         difference before its factor f = -v/(12 dx)),
// is evaluated as one weighted sum per axis: the four neighbours at offsets
// -2, -1, +1, +2 carry per-velocity weights (KO and ADV coefficients folded
// together, StencilW), the pair at +-3 (6th difference only) the uniform
// eps, and the centre, shared by both axes, -20 (eps_z + eps_x) or
// 6 (eps_z + eps_x).  That is 14 (6th) or 10 (4th) FP64 operations per field
// instead of 22 (18) for the separate KO and ADV sums.
//   6th: w = {-6 eps + f, 15 eps - 8 f, 15 eps + 8 f, -6 eps - f}
//   4th: w = {eps + f, -4 eps - 8 f, -4 eps + 8 f, eps - f}
template <int R>
__host__ __device__ __forceinline__ void stencil_weights(double eps, double f, double (&w)[4]) {
    if (R == 3) {
        w[0] = -6 * eps + f;
        w[1] = 15 * eps - 8 * f;
        w[2] = 15 * eps + 8 * f;
        w[3] = -6 * eps - f;
    } else {
        w[0] = eps + f;
        w[1] = -4 * eps - 8 * f;
        w[2] = -4 * eps + 8 * f;
        w[3] = eps - f;
    }
}

// one axis's off-centre terms: s[C-2..C+2] without the centre with weights
// w[0..3], plus eps (s[0] + s[6]) in the 6th difference
template <typename T, int R>
__device__ __forceinline__ T axis_sum(const T (&s)[2 * R + 1], const T (&w)[4], T eps) {
    constexpr int C = R;
    T acc;
    if constexpr (R == 3) acc = eps * (s[0] + s[6]);
    else acc = T(0);
    acc = fma(w[0], s[C - 2], acc);
    acc = fma(w[1], s[C - 1], acc);
    acc = fma(w[2], s[C + 1], acc);
    return fma(w[3], s[C + 2], acc);
}

template <typename T, bool VAC>
__device__ __forceinline__ void rhs_half(const T (&c)[4], T a, T b, T e, T mu, T p2s, T p2c, T ps, const T (&sten)[4],
                                         T (&out)[4], bool vac) {
    const T ee = c[0], mm = c[1], emr = c[2], emi = c[3];
    const T Iee = T(2) * mu * (emi * a + emr * b);
    const T Iemr = -mu * ((ee - mm) * b + e * emi);
    const T Iemi = mu * ((mm - ee) * a + e * emr);
    out[0] = Iee + sten[0];
    out[1] = -Iee + sten[1];
    out[2] = Iemr + sten[2];
    out[3] = Iemi + sten[3];
    if (VAC && vac) {  // pmo * [H_vac, rho] (nuosc_class.cpp:280-287); p2s = 2 pmo st, p2c = 2 pmo ct, ps = pmo st
        out[0] -= p2s * emi;
        out[1] += p2s * emi;
        out[2] -= p2c * emi;
        out[3] += p2c * emr + ps * (ee - mm);
    }
}

// the weights 2jj and 2jj + 1 of this lane's NP velocities (one 16-byte load)
template <typename T, int NP>
__device__ __forceinline__ void ldw(const T *p, T (&a)[NP], T (&b)[NP]) {
    if constexpr (NP == 2) {
        const float4 t = *reinterpret_cast<const float4 *>(p);
        a[0] = t.x;
        a[1] = t.y;
        b[0] = t.z;
        b[1] = t.w;
    } else {
        const double2 t = *reinterpret_cast<const double2 *>(p);
        a[0] = t.x;
        b[0] = t.y;
    }
}

// statically allocated per-CTA scratch of the march: the abort flag, the
// per-velocity stencil weights and, with two velocities per thread (FP32),
// the per-velocity constants of the commutator and the moments (the moment
// weights in double when the FP32 march sums its moment partials in FP64, M64)
template <typename T, bool M64>
struct MarchShared {
    static constexpr bool kShared = vpt<T>() == 2;
    static constexpr int NP = vpt<T>();
    // [component][lane] and [j][lane], the lane's two velocities side by side
    // (one 16-byte load, 8-byte for float weights); consecutive lanes read
    // consecutive vectors (a lane-major layout would put 16 lanes on one bank)
    double2 vq[kShared ? 3 : 1][kShared ? 32 : 1];                              // vx, vy, vz
    std::conditional_t<M64, double2, float2> wp[kShared ? 4 : 1][kShared ? 32 : 1];  // lane-permuted
    // stencil weights, z axis j = 0..3 then x axis j = 4..7, in pairs: sw[jj][lane]
    // holds weights 2jj (NP velocities) and 2jj + 1 (NP velocities), 16 bytes,
    // so a lane reads all eight with four conflict-free 16-byte loads
    __align__(16) T sw[4][32][2 * NP];
    int abort;
};

template <typename T, int TZ>
constexpr int tma_ctas_per_sm() {
    return TZ == 16 ? 1 : 2;
}

// Ring geometry of one march.  Boxes are issued D planes ahead of their
// front use: 3 with 16-row tiles (one CTA per SM, 8 slots of 24 KB at R = 3),
// 2 with 8-row tiles (two CTAs per SM share the 228 KB).  The pointwise
// inputs of the epilogue (U in S2/S3/S4, B in S4) stay plain
// per-thread loads, but thread 0 prefetches their TZ rows of plane x + PFD
// into L2 with one tensor prefetch each, so those loads hit L2: measured 3 %
// faster per step than without (PFD 1 and 3 equal within noise, 6 slower),
// and faster than staging them through shared memory, which costs ring depth.
template <typename T, int R, int MODE, int TZ>
struct MarchCfg {
    static constexpr int D = TZ == 16 ? 3 : 2;  // boxes issued ahead of their first use
    static constexpr int PFD = 2;                 // L2 prefetch distance of the pointwise inputs, planes
    static constexpr bool PU = MODE == MODE_SY || MODE == MODE_S2B;  // reads U pointwise
    static constexpr bool PA = MODE == MODE_S4B;                     // reads B pointwise
    static constexpr int NS = R + D + 2;  // a box lives from its front use to its centre use, plus slack
    static constexpr size_t ring = (size_t)NS * Slot<T, TZ, R>::bytes;
    static constexpr size_t smem = ring + 2 * NS * 8;  // box ring | mbarriers
};

}  // namespace

// value of x, re-read from (shared) memory at each use when V: keeps values
// that are loop-invariant but cheap to re-read out of the register file
template <bool V, typename P>
__device__ __forceinline__ P rd(const P &x) {
    if constexpr (V) return *(const volatile P *)&x;
    else return x;
}

// One tile of work: z rows z0..z0+TZ-1, velocity block vb (of nvb), x planes
// xs..xe-1, flavour half `half`, of the instance described by (*mp, a).
// Called by the single-instance kernel (one tile per CTA; a and *mp in kernel
// parameter space) and by the persistent batched kernel (many tiles per CTA,
// of many instances; SA: a and mp in shared memory); the arithmetic per
// (cell, velocity) does not depend on which.  VAC compiles the vacuum term in
// (it then runs where a.c.pmo != 0).  Returns true when a bounded wait
// expired (the status word is set and the tile is incomplete).
template <typename T, int R, int MODE, int TZ, bool VAC, bool SA, bool M64>
__device__ __forceinline__ bool xtma_march(const TmaMaps *const &mp, const StageArgs<T> &a, const int z0, const int vb,
                                           const int nvb, const int xs, const int xe, const int half,
                                           unsigned char *smem, MarchShared<T, M64> &sh) {
    using S = Slot<T, TZ, R>;
    using CF = MarchCfg<T, R, MODE, TZ>;
    constexpr int NP = vpt<T>();       // velocities per thread
    constexpr int VB = S::VB;          // velocities per CTA
    constexpr int W = 2 * R + 1;
    constexpr int ZR = S::ZR;
    constexpr int D = CF::D;
    constexpr int NS = CF::NS;
    unsigned long long *bars = (unsigned long long *)(smem + CF::ring);  // full[NS], empty[NS]
    int &s_abort = sh.abort;

    const Geom g = a.g;
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int v = vb * VB + NP * lane;  // first of this thread's NP velocities
    const bool vact = v < g.nvs;        // nvs is a multiple of NP, so all NP are active together
    const int nplanes = xe - xs;
    const int nboxes = nplanes + R;    // centres xs..xe-1 and fronts up to xe-1+R
    const int zr = z0 + r;             // < nz since nz % TZ == 0
    const long long fs = g.fs;
    const long long P = (long long)g.nz * g.nvs;
    const long long hoff = (long long)half * 4 * fs;
    const T *in = a.in + hoff;
    const int vc = vact ? v : 0;
    const long long own = (long long)zr * g.nvs + vc;
    // per-plane addressing in 32 bits: within one flavour half, a field's
    // offset f fs (f <= 3), a plane's x P and a cell's moment-partial index
    // all fit (xtma_supported requires 3 fs < 2^32); only the half's own
    // offset, hoff, needs 64 bits
    const unsigned fs32 = (unsigned)fs, P32 = (unsigned)P, own32 = (unsigned)own;

    __syncthreads();  // the previous tile of this CTA (batched kernel) is done with the ring
    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < 2 * NS; ++s) mbar_init(smem_u32(&bars[s]), s < NS ? 1u : (unsigned)TZ);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // lane 0 of warp 0: load box j (plane xs + j, periodic) into slot j % NS
    // (phase j / NS of its full barrier).  `issued` = last box issued + 1.
    // fault_tx (the self-test of the bounded waits) over-declares the bytes of
    // box R of the instance's first tile: all its copies land, its phase never
    // completes.
    int issued = 0;
    const unsigned fault_tx =
        (tid == 0 && z0 == 0 && vb == 0 && xs == 0 && half == 0) ? rd<SA>(a.fault_tx) : 0u;
    auto issue = [&](int j) -> bool {
        const int s = j % NS;
        if (j >= NS && !mbar_wait(smem_u32(&bars[NS + s]), (unsigned)((j / NS - 1) & 1))) return false;
        const unsigned full = smem_u32(&bars[s]);
        unsigned char *sp = smem + s * S::bytes;
        mbar_expect_tx(full, S::tx + (j == R ? fault_tx : 0u));
        // plane xs + j; past the last plane it wraps (periodic) or, in a slab,
        // comes from the halo buffer's right planes (box plane x - nx + R).
        // Boxes start at plane xs >= 0, so the left halo is never a box.
        const int nx = rd<SA>(a.g.nx), xl = xs + j;
        const bool hal = xl >= nx && rd<SA>(a.halo) != nullptr;
        const int x = hal ? xl - nx + R : xl % nx;
        const int nz = rd<SA>(a.g.nz);
        const TmaMaps &maps = *rd<SA>(mp);
        const int c1 = 4 * half, c0 = vb * VB;
        int zstart = z0 - R, dst = 0;
        while (dst < ZR) {
            const int zw = zstart < 0 ? zstart + nz : (zstart >= nz ? zstart - nz : zstart);
            int len = nz - zw;
            if (len > ZR - dst) len = ZR - dst;
            const CUtensorMap *m = len == ZR        ? (hal ? &maps.hzr : &maps.zr)
                                   : len == TZ + R ? (hal ? &maps.htzr : &maps.tzr)
                                   : len == TZ     ? (hal ? &maps.htz : &maps.tz)
                                                   : (hal ? &maps.hr : &maps.r);
            tma_load_4d(smem_u32(sp + S::box + dst * 4 * VB * sizeof(T)), m, c0, c1, zw, x, full);
            zstart += len;
            dst += len;
        }
        // the cell moments are read at a box's centre use, which is always an
        // interior plane; a halo box (front use only) loads plane nx-1's, unread
        const int xm = hal ? nx - 1 : x;
        bulk_load(smem_u32(sp + S::mb), rd<SA>(a.mom_in) + ((long long)xm * nz + z0) * NMOM, 8u * TZ * NMOM, full);
        issued = j + 1;
        return true;
    };

    // thread 0: L2 prefetch of the pointwise inputs of plane xs + i
    auto l2pref = [&](int i) {
        if ((CF::PU || CF::PA) && i < nplanes) {
            const TmaMaps &maps = *rd<SA>(mp);
            if (CF::PU) tma_prefetch_4d(&maps.pu, vb * VB, 4 * half, z0, xs + i);
            if (CF::PA) tma_prefetch_4d(&maps.pa, vb * VB, 4 * half, z0, xs + i);
        }
    };

    // per-velocity and uniform constants.  Lane-permuted moment weights: slot s
    // of this lane holds weight s ^ wq (weights w, w vx, w vy, w vz), wq = lane
    // bits 4..3, the order the moment reduce-scatter needs.  With two
    // velocities per thread (FP32) the per-velocity constants (FP64
    // velocities, float weights) live in shared memory and are read per plane,
    // which keeps the register queue clear of spills.
    const int wq = (lane >> 3) & 3;
    constexpr bool kShared = MarchShared<T, M64>::kShared;
    auto &s_vq = sh.vq;
    auto &s_wp = sh.wp;
    double vxd[NP], vyd[NP], vzd[NP], wperm[NP][4];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        vxd[p] = a.q.vx[vc + p];
        vyd[p] = a.q.vy[vc + p];
        vzd[p] = a.q.vz[vc + p];
        if (r == 0) {
            double wz[4], wx[4];
            stencil_weights<R>(a.c.kz, vzd[p] * a.c.fzs, wz);
            stencil_weights<R>(a.c.kx, vxd[p] * a.c.fxs, wx);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                sh.sw[j >> 1][lane][(j & 1) * NP + p] = T(wz[j]);
                sh.sw[2 + (j >> 1)][lane][(j & 1) * NP + p] = T(wx[j]);
            }
        }
        const double wd = vact ? a.q.vw[vc + p] : 0.0;
        const double v4w[4] = {wd, vxd[p] * wd, vyd[p] * wd, vzd[p] * wd};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = j ^ wq;
            wperm[p][j] = k == 0 ? v4w[0] : k == 1 ? v4w[1] : k == 2 ? v4w[2] : v4w[3];
        }
    }
    if constexpr (kShared) {
        if (r == 0) {
            s_vq[0][lane] = make_double2(vxd[0], vxd[NP - 1]);
            s_vq[1][lane] = make_double2(vyd[0], vyd[NP - 1]);
            s_vq[2][lane] = make_double2(vzd[0], vzd[NP - 1]);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if constexpr (M64) s_wp[j][lane] = make_double2(wperm[0][j], wperm[NP - 1][j]);
                else s_wp[j][lane] = make_float2((float)wperm[0][j], (float)wperm[NP - 1][j]);
            }
        }
    }
    __syncthreads();  // the per-velocity constants in shared memory are complete
    // uniform coefficients: hoisted (kernel parameters in the single-instance
    // kernel; FP32 values in registers), except for the FP64 batched kernel,
    // which re-reads them from shared memory at each use
    constexpr bool RR = SA && sizeof(T) == 8;
    const T kz = RR ? T(0) : T(a.c.kz), kx = RR ? T(0) : T(a.c.kx), mu = RR ? T(0) : T(a.c.mu);
    const T kc = T((R == 3 ? -20.0 : 6.0) * (a.c.kz + a.c.kx));  // centre weight of both axes
    const T cA0 = RR ? T(0) : T(a.cA), cY0 = RR ? T(0) : T(a.cY);
    auto K = [&](const double &x, T hoisted) -> T {
        if constexpr (RR) return T(rd<true>(x));
        else return hoisted;
    };
    const T p2s = T(2 * a.c.pmo * a.c.st), p2c = T(2 * a.c.pmo * a.c.ct), ps = T(a.c.pmo * a.c.st);
    const bool vac = VAC && a.c.pmo != 0.0;  // batched launches: instances without a vacuum term skip it

    // prime the register queue with planes xs-R .. xs+R-1 (periodic, or from
    // a slab's halo buffer outside [0, nx))
    T q[4][W][NP];
    const T *halo = rd<SA>(a.halo);
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) {
        const int pl = xs - R + k;
        const bool hal = halo != nullptr && (pl < 0 || pl >= g.nx);
        const long long o = (long long)wrap_index(pl, g.nx) * P + own;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T t[NP];
            const T *src = hal ? halo + halo_offset(4 * half + f, pl, g.nx, R, P) + own : in + f * fs + o;
            if (vact) ldv<T, NP>(src, t);
#pragma unroll
            for (int p = 0; p < NP; ++p) q[f][k][p] = vact ? t[p] : T(0);
        }
    }
    bool ok = true;
    if (tid == 0) {  // boxes j < R are only centres: skip those past a short segment's end
        for (int j = 0; j < R + D && j < nboxes; ++j)
            if (j >= R || j < nplanes) ok = ok && issue(j);
        for (int j = 1; j < CF::PFD; ++j) l2pref(j);
    }

    for (int i = 0; i < nplanes; ++i) {
        if (tid == 0) {
            if (ok && i + R + D < nboxes) ok = issue(i + R + D);
            if (!ok) s_abort = 1;
            l2pref(i + CF::PFD);
        }
        const int x = xs + i;
        const unsigned ox = (unsigned)x * P32 + own32;  // element offset of (x, zr, v) within a field
        T uin[4][NP], ain[4][NP];  // U, B
        {
            // pointwise epilogue inputs first (they are not in the ring; L2 hits
            // after the tensor prefetch PFD planes earlier)
            constexpr bool LU = CF::PU, LA = CF::PA;
            const T *up = LU ? rd<SA>(a.u) + hoff + ox : nullptr;
            const T *ap = LA ? rd<SA>(a.acc_src) + hoff + ox : nullptr;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
#pragma unroll
                for (int p = 0; p < NP; ++p) uin[f][p] = ain[f][p] = T(0);
                if (vact) {
                    if (LU) ldv<T, NP>(up + f * fs32, uin[f]);
                    if (LA) ldv<T, NP>(ap + f * fs32, ain[f]);
                }
            }
        }
        // the front box (plane i + R) has to be waited for; the centre box was
        // this warp's front box R planes ago (its slot is not refilled before
        // its centre use), except for the first R centres, which are never fronts
        const int jf = i + R, sf = jf % NS, sc = i % NS;
        if (!mbar_wait(smem_u32(&bars[sf]), (unsigned)((jf / NS) & 1)) ||
            (i < R && !mbar_wait(smem_u32(&bars[sc]), (unsigned)((i / NS) & 1))) ||
            ((i & 3) == 0 && *(volatile int *)&s_abort)) {  // another warp's abort, looked at every 4th plane
            s_abort = 1;
            break;
        }
        const T *fbox = (const T *)(smem + sf * S::bytes + S::box);
#pragma unroll
        for (int f = 0; f < 4; ++f) ldv<T, NP>(&fbox[((R + r) * 4 + f) * VB + NP * lane], q[f][2 * R]);
        if (jf >= nplanes) {  // this box is never a centre: its front use was the last
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bars[NS + sf]));
        }
        const unsigned char *sp = smem + sc * S::bytes;
        const T *zb = (const T *)(sp + S::box);
        const double *mb = (const double *)(sp + S::mb);

        T sten[4][NP];
        const T kzp = K(a.c.kz, kz), kxp = K(a.c.kx, kx);
        T swz[4][NP], swx[4][NP];  // this lane's stencil weights (shared memory, re-read per plane)
        ldw<T, NP>(&sh.sw[0][lane][0], swz[0], swz[1]);
        ldw<T, NP>(&sh.sw[1][lane][0], swz[2], swz[3]);
        ldw<T, NP>(&sh.sw[2][lane][0], swx[0], swx[1]);
        ldw<T, NP>(&sh.sw[3][lane][0], swx[2], swx[3]);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T zs[W][NP];
#pragma unroll
            for (int k = 0; k < W; ++k)  // the centre row is the x-queue's centre: not re-read
                if (k != R) ldv<T, NP>(&zb[((r + k) * 4 + f) * VB + NP * lane], zs[k]);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                T zsp[W], xsp[W], wzp[4], wxp[4];
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    zsp[k] = k == R ? q[f][R][p] : zs[k][p];
                    xsp[k] = q[f][k][p];
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    wzp[j] = swz[j][p];
                    wxp[j] = swx[j][p];
                }
                const T sz = axis_sum<T, R>(zsp, wzp, kzp), sx = axis_sum<T, R>(xsp, wxp, kxp);
                sten[f][p] = fma(kc, q[f][R][p], sz + sx);
            }
        }
        double m[NMOM];
        {
            const double2 *m2 = (const double2 *)(mb + r * NMOM);
#pragma unroll
            for (int k = 0; k < NMOM / 2; ++k) {
                const double2 t = m2[k];
                m[2 * k] = t.x;
                m[2 * k + 1] = t.y;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&bars[NS + sc]));  // centre use is the box's last use

        T outm[4][NP];
        double2 vq2[3];
        if constexpr (kShared) {
#pragma unroll
            for (int c = 0; c < 3; ++c) vq2[c] = s_vq[c][lane];
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const double ux = kShared ? (p ? vq2[0].y : vq2[0].x) : vxd[p];
            const double uy = kShared ? (p ? vq2[1].y : vq2[1].x) : vyd[p];
            const double uz = kShared ? (p ? vq2[2].y : vq2[2].x) : vzd[p];
            const T ia = T(inp(m, ux, uy, uz)), ib = T(inp(m + 4, ux, uy, uz)), ie = T(inp(m + 8, ux, uy, uz));
            const T cen[4] = {q[0][R][p], q[1][R][p], q[2][R][p], q[3][R][p]};
            const T st4[4] = {sten[0][p], sten[1][p], sten[2][p], sten[3][p]};
            T kk[4];
            rhs_half<T, VAC>(cen, ia, ib, ie, K(a.c.mu, mu), p2s, p2c, ps, st4, kk, vac);
            const T cA = K(a.cA, cA0), cY = K(a.cY, cY0);
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                if (MODE == MODE_S1Y) {
                    outm[f][p] = cen[f] + cY * kk[f];  // Y2
                } else if (MODE == MODE_SY) {
                    outm[f][p] = uin[f][p] + cY * kk[f];  // Y4
                } else if (MODE == MODE_S2B) {
                    const T u = uin[f][p];
                    ain[f][p] = (u + cen[f]) + cA * kk[f];  // B = U + Y2 + dt k2
                    outm[f][p] = u + cY * kk[f];            // Y3
                } else {
                    outm[f][p] = third_plus(ain[f][p] + cen[f], cA * kk[f]);  // (B + Y4)/3 + dt/6 k4
                }
            }
        }
        if (vact) {
            T *dp = (MODE == MODE_S4B ? rd<SA>(a.acc_dst) : rd<SA>(a.y_dst)) + hoff + ox;
#pragma unroll
            for (int f = 0; f < 4; ++f) stv<T, NP>(dp + f * fs32, outm[f]);
            if (MODE == MODE_S2B) {
                T *bp = rd<SA>(a.acc_dst) + hoff + ox;
#pragma unroll
                for (int f = 0; f < 4; ++f) stv<T, NP>(bp + f * fs32, ain[f]);
            }
        }
        // velocity-moment partials of the written state (nuosc_class.cpp:69-71):
        // moment 4c + j = sum over the block's velocities of weight j (w, w vx,
        // w vy, w vz) times combination c (emr, emi, ee - mm; the neutrino half
        // enters with sign -1 in combinations 0 and 2, applied to the final
        // sum, which is exact).
        // M64 (every FP64 march; the FP32 march when the tile table says so):
        // products and the warp's reduce-scatter in double -- the float state
        // converts exactly and each product with a double weight is a double
        // product, so the sums carry no error beyond the state's own rounding.
        // FP32 march without M64: in float -- the float state's products with
        // float-rounded weights, summed over the block's 64 velocities --, the
        // block's partial stored as double; the blocks and both halves are
        // summed in FP64 by the finalize either way.
        // Each lane forms its 12 products (weight slots in its order s ^ wq) and
        // the warp reduce-scatters them, pairing lanes over bits 4, 3, 2, 1, 0:
        // over bit 4 weight slots 2 and 3 go to the partner, over bit 3 slot 1,
        // which leaves every lane the three combinations of weight wq; over bit
        // 2 the lanes with the bit clear keep combinations 0 and 1, the others
        // combination 2; over bit 1 the former split 0 and 1 while the latter
        // sum 2; over bit 0 both sum.  13 shuffle-adds for the 12 sums.
        {
            using M = std::conditional_t<M64, double, float>;
            M acc[3][4];
            [[maybe_unused]] std::conditional_t<M64, double2, float2> wp2[kShared ? 4 : 1];
            if constexpr (kShared) {
#pragma unroll
                for (int j = 0; j < 4; ++j) wp2[j] = s_wp[j][lane];
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                const M ee = M(outm[0][p]), mm = M(outm[1][p]), emr = M(outm[2][p]), emi = M(outm[3][p]);
                const M d[3] = {emr, emi, ee - mm};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    M wj;
                    if constexpr (kShared) wj = p ? wp2[j].y : wp2[j].x;
                    else wj = wperm[p][j];
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[c][j] = p == 0 ? wj * d[c] : fma(wj, d[c], acc[c][j]);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                acc[c][0] += __shfl_xor_sync(0xffffffffu, acc[c][2], 16);
                acc[c][1] += __shfl_xor_sync(0xffffffffu, acc[c][3], 16);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c][0] += __shfl_xor_sync(0xffffffffu, acc[c][1], 8);
            const bool b2 = (lane >> 2) & 1, b1 = (lane >> 1) & 1;
            M k0 = b2 ? acc[2][0] : acc[0][0];
            k0 += __shfl_xor_sync(0xffffffffu, b2 ? acc[0][0] : acc[2][0], 4);
            const M k1 = acc[1][0] + __shfl_xor_sync(0xffffffffu, acc[1][0], 4);
            M kk = (!b2 && b1) ? k1 : k0;
            kk += __shfl_xor_sync(0xffffffffu, (b2 || b1) ? k0 : k1, 2);
            kk += __shfl_xor_sync(0xffffffffu, kk, 1);
            if ((lane & 1) == 0 && !(b2 && b1)) {  // lanes 0 mod 2 hold moment 4c + wq
                const int c = b2 ? 2 : (int)b1;
                const double v = (double)kk;
                const unsigned cell = (unsigned)x * (unsigned)rd<SA>(a.g.nz) + (unsigned)zr;
                rd<SA>(a.mom_part)[((cell * (unsigned)nvb + (unsigned)vb) * 2u + (unsigned)half) * NMOM + 4 * c + wq] =
                    (half || c == 1) ? v : -v;
            }
        }
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int k = 0; k < 2 * R; ++k)
#pragma unroll
                for (int p = 0; p < NP; ++p) q[f][k][p] = q[f][k + 1][p];
    }
    __syncthreads();
    const bool aborted = s_abort != 0;
    if (tid == 0) {
        if (aborted) {
            // a wait expired: report it, then wait (bounded) for the copies of
            // the last NS boxes issued -- the only ones that may still be in
            // flight: box j - NS of a slot was consumed (so had landed) before
            // box j was issued into it -- before the CTA's shared memory is
            // reused or released
            atomicExch(a.status, NUOSC_TIMEOUT_CODE);
            for (int j = issued > NS ? issued - NS : 0; j < issued; ++j)
                if (j >= R || j < nplanes) mbar_wait(smem_u32(&bars[j % NS]), (unsigned)((j / NS) & 1));
        }
        for (int s = 0; s < 2 * NS; ++s) mbar_inval(smem_u32(&bars[s]));
    }
    return aborted;
}

// grid (velocity blocks run by this kernel, z tiles, 2 x x-segments); nvb:
// velocity blocks of the moment partials (one more when a tail kernel runs
// the last block)
template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
__global__ void __launch_bounds__(32 * TZ, tma_ctas_per_sm<T, TZ>())
    k_xtma(const __grid_constant__ TmaMaps maps, const StageArgs<T> a, int LX, int nvb) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ MarchShared<T, M64> sh;
    const int xs = (blockIdx.z >> 1) * LX;
    if (xs >= a.g.nx) return;
    const TmaMaps *mp = &maps;
    xtma_march<T, R, MODE, TZ, VAC, false, M64>(mp, a, blockIdx.y * TZ, blockIdx.x, nvb, xs, min(xs + LX, a.g.nx),
                                           blockIdx.z & 1, smem, sh);
}

// One instance's stage in a batched launch: its tensor maps (over the stage's
// input register), stage arguments and tile counts.  Lives in device memory;
// the TMA reads the maps from there.
template <typename T>
struct __align__(64) BatchItem {
    TmaMaps maps;
    StageArgs<T> a;
    int ntz, nvb, lx, nseg;
    int nvbm;  // velocity blocks run by the march (nvb - 1 when a tail kernel runs the last)
};

// Persistent batched stage kernel.  The tiles of all instances form one list
// (instances in the order of the table -- largest first --, each instance's
// tiles in the single-instance kernel's CTA order: velocity block fastest,
// then z rows, then flavour half and x segment) that the CTAs take from an
// atomic cursor, so the tiles in flight stay a narrow window of the list, as
// in a hardware-scheduled grid (neighbouring tiles share halo rows in L2 and
// DRAM pages).  Tile k of instance i is the tile the single-instance kernel
// runs as its CTA k, so each instance's result is the same bits as its own
// launch.  The tile's StageArgs are copied to shared memory and re-read there at each use
// (the single-instance kernel reads them from the constant bank), which keeps
// them out of the register file that the march's x-queue fills.  VAC compiles
// the vacuum term in (for batches with any pmo != 0); it is then switched per
// instance at run time.
template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
__global__ void __launch_bounds__(32 * TZ, tma_ctas_per_sm<T, TZ>())
    k_xtma_batch(const BatchItem<T> *items, const long long *__restrict__ starts, int ninst, long long nitems,
                 unsigned long long *counter, const int *__restrict__ halt) {
    constexpr int NW = (int)(sizeof(StageArgs<T>) / 8);
    static_assert(sizeof(StageArgs<T>) % 8 == 0 && NW <= 32 * TZ, "StageArgs copy: one 8-byte word per thread");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ MarchShared<T, M64> sh;
    __shared__ __align__(16) StageArgs<T> s_a;
    __shared__ const TmaMaps *s_mp;
    __shared__ int s_t[6];  // instance (-1: no tiles left, -2: a stopped instance's tile), z0, vb, xs, xe, half
    for (;;) {
        __syncthreads();  // every thread is done with the previous tile's arguments
        if (threadIdx.x == 0) {
            const long long it = (long long)atomicAdd(counter, 1ull);
            s_t[0] = -1;
            if (it < nitems) {
                int lo = 0, hi = ninst - 1;  // last instance whose first tile is <= it
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (starts[mid] <= it) lo = mid;
                    else hi = mid - 1;
                }
                const BatchItem<T> &e = items[lo];
                long long loc = it - starts[lo];  // ((seg * 2 + half) * ntz + zt) * nvbm + vb
                s_t[0] = (halt && halt[lo]) ? -2 : lo;
                const int vb = (int)(loc % e.nvbm);
                loc /= e.nvbm;
                const int zt = (int)(loc % e.ntz);
                loc /= e.ntz;
                const int xs = (int)(loc >> 1) * e.lx;
                s_t[1] = zt * TZ;
                s_t[2] = vb;
                s_t[3] = xs;
                s_t[4] = min(xs + e.lx, e.a.g.nx);
                s_t[5] = (int)(loc & 1);
                s_mp = &e.maps;
                // thread 0 issues every TMA load of the tile; the maps were written
                // through the generic proxy (a host copy when the work-list was built)
                tensormap_acquire(&e.maps.zr);
                tensormap_acquire(&e.maps.tzr);
                tensormap_acquire(&e.maps.tz);
                tensormap_acquire(&e.maps.r);
                if (MarchCfg<T, R, MODE, TZ>::PU) tensormap_acquire(&e.maps.pu);
                if (MarchCfg<T, R, MODE, TZ>::PA) tensormap_acquire(&e.maps.pa);
            }
        }
        __syncthreads();
        const int lo = s_t[0];
        if (lo == -1) break;
        if (lo == -2) continue;  // every thread: the loop's first barrier comes next
        if (threadIdx.x < NW)
            reinterpret_cast<long long *>(&s_a)[threadIdx.x] =
                reinterpret_cast<const long long *>(&items[lo].a)[threadIdx.x];
        const int nvb = items[lo].nvb;
        const int z0 = s_t[1], vb = s_t[2], xs = s_t[3], xe = s_t[4], half = s_t[5];
        __syncthreads();  // s_a is complete
        if (xtma_march<T, R, MODE, TZ, VAC, true, M64>(s_mp, s_a, z0, vb, nvb, xs, xe, half, smem, sh)) break;
    }
}

// Self-test of the bounded wait that the march kernels use: one warp waits on
// an mbarrier that nothing completes (initialised for two arrivals, given
// one).  The wait gives up after `spins` polls; the kernel then records the
// timeout in the status word, as a march does, invalidates the barrier and
// returns.  Nothing else is touched, so the context stays usable.
__global__ void k_wait_selftest(int *status, unsigned spins) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 2u);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        mbar_arrive(smem_u32(&bar));  // one arrival of two: phase 0 never completes
        if (!mbar_wait(smem_u32(&bar), 0u, spins)) atomicExch(status, NUOSC_TIMEOUT_CODE);
        mbar_inval(smem_u32(&bar));
    }
}

cudaError_t launch_wait_selftest(int *status, unsigned spins, cudaStream_t s) {
    k_wait_selftest<<<1, 32, 0, s>>>(status, spins);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ host side
namespace {

bool tma_mode(int mode) { return mode == MODE_S1Y || mode == MODE_S2B || mode == MODE_SY || mode == MODE_S4B; }

using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeFn)p;
    }
    return fn;
}

// 4D view of one register: (v, field, z, x) with box {VB, 4, rows, 1}
template <typename T>
bool make_map(CUtensorMap *m, const T *base, const Geom &g, int rows) {
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nvs, 8, (cuuint64_t)g.nz, (cuuint64_t)g.nx};
    const cuuint64_t strides[3] = {(cuuint64_t)g.fs * sizeof(T), (cuuint64_t)g.nvs * sizeof(T),
                                   (cuuint64_t)g.nz * g.nvs * sizeof(T)};
    const cuuint32_t box[4] = {(cuuint32_t)vblock<T>(), 4, (cuuint32_t)rows, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return fn(m, dt, 4, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// velocity blocks the march runs: all of them, or all but the tail block
template <typename T>
int march_vblocks(const Geom &g) {
    const int v0 = xtma_tail_v0<T>(g);
    return v0 == g.nvs ? xtma_num_vblocks<T>(g) : v0 / vblock<T>();
}

// the stencil input's boxes, and the TZ-row boxes of the stage's pointwise
// inputs (U, A) where the stage has them (zeroed maps otherwise)
template <typename T>
bool make_maps(TmaMaps *m, const StageArgs<T> &a, int tz, int r) {
    memset((void *)&m->pu, 0, sizeof m->pu);
    memset((void *)&m->pa, 0, sizeof m->pa);
    memset((void *)&m->hzr, 0, 4 * sizeof m->hzr);
    // a slab's halo buffer as a register of 2R planes
    Geom h = a.g;
    h.nx = 2 * r;
    h.fs = (long long)h.nx * h.nz * h.nvs;
    return make_map<T>(&m->zr, a.in, a.g, tz + 2 * r) && make_map<T>(&m->tzr, a.in, a.g, tz + r) &&
           make_map<T>(&m->tz, a.in, a.g, tz) && make_map<T>(&m->r, a.in, a.g, r) &&
           (!a.u || make_map<T>(&m->pu, a.u, a.g, tz)) && (!a.acc_src || make_map<T>(&m->pa, a.acc_src, a.g, tz)) &&
           (!a.halo || (make_map<T>(&m->hzr, a.halo, h, tz + 2 * r) && make_map<T>(&m->htzr, a.halo, h, tz + r) &&
                        make_map<T>(&m->htz, a.halo, h, tz) && make_map<T>(&m->hr, a.halo, h, r)));
}

template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
cudaError_t launch_t(const StageArgs<T> &a, XTile t, cudaStream_t s) {
    using CF = MarchCfg<T, R, MODE, TZ>;
    static_assert(tma_ctas_per_sm<T, TZ>() * (CF::smem + sizeof(MarchShared<T, M64>) + 64 + 1024) <= 228 * 1024,
                  "ring exceeds shared memory");
    TmaMaps maps;
    if (!make_maps<T>(&maps, a, TZ, R)) return cudaErrorInvalidValue;
    const size_t smem = CF::smem;
    cudaError_t e = cudaFuncSetAttribute(k_xtma<T, R, MODE, TZ, VAC, M64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int nseg = (a.g.nx + t.lx - 1) / t.lx;
    const int nvb = xtma_num_vblocks<T>(a.g), nvbm = march_vblocks<T>(a.g);
    if (nvbm < 1) return cudaSuccess;  // the tail kernel runs every velocity
    // velocity blocks fastest: the CTAs resident at once read whole velocity
    // rows of a few z rows (DRAM page locality) rather than one block of many rows
    dim3 grid(nvbm, a.g.nz / TZ, nseg * 2);
    k_xtma<T, R, MODE, TZ, VAC, M64><<<grid, 32 * TZ, smem, s>>>(maps, a, t.lx, nvb);
    return cudaGetLastError();
}

template <typename T, int R, int TZ, bool VAC, bool M64>
cudaError_t launch_tm(const StageArgs<T> &a, int mode, XTile t, cudaStream_t s) {
    switch (mode) {
    case MODE_S1Y: return launch_t<T, R, MODE_S1Y, TZ, VAC, M64>(a, t, s);
    case MODE_S2B: return launch_t<T, R, MODE_S2B, TZ, VAC, M64>(a, t, s);
    case MODE_SY: return launch_t<T, R, MODE_SY, TZ, VAC, M64>(a, t, s);
    case MODE_S4B: return launch_t<T, R, MODE_S4B, TZ, VAC, M64>(a, t, s);
    default: return cudaErrorInvalidValue;
    }
}

template <typename T, int R, int TZ, bool M64>
cudaError_t launch_tv(const StageArgs<T> &a, int mode, XTile t, cudaStream_t s) {
    return a.c.pmo != 0.0 ? launch_tm<T, R, TZ, true, M64>(a, mode, t, s)
                          : launch_tm<T, R, TZ, false, M64>(a, mode, t, s);
}

// moment partials summed in FP64 (always for FP64 state; for FP32 state per
// the tile's msum) or in float within a velocity block
template <typename T, int R, int TZ>
cudaError_t launch_tms(const StageArgs<T> &a, int mode, XTile t, cudaStream_t s) {
    if constexpr (sizeof(T) == 8) return launch_tv<T, R, TZ, true>(a, mode, t, s);
    else return t.msum ? launch_tv<T, R, TZ, true>(a, mode, t, s) : launch_tv<T, R, TZ, false>(a, mode, t, s);
}

// ---- batched launch: one persistent grid per stage over many instances
template <typename T, int R, int MODE, int TZ>
constexpr size_t batch_smem() {
    return MarchCfg<T, R, MODE, TZ>::smem;
}

template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
int batch_grid_t(int device) {
    const size_t smem = batch_smem<T, R, MODE, TZ>();
    auto kern = k_xtma_batch<T, R, MODE, TZ, VAC, M64>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * TZ, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || per_sm < 1)
        return -1;
    return per_sm * sms;
}

template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
cudaError_t batch_launch_t(const void *items, const long long *starts, int n, long long ntiles,
                           unsigned long long *counter, const int *halt, int grid, cudaStream_t s) {
    k_xtma_batch<T, R, MODE, TZ, VAC, M64><<<grid, 32 * TZ, batch_smem<T, R, MODE, TZ>(), s>>>(
        (const BatchItem<T> *)items, starts, n, ntiles, counter, halt);
    return cudaGetLastError();
}

// dispatch of (mode, ko6, tz, vac) onto the template instances of F
template <typename T, bool M64, template <typename, int, int, int, bool, bool> class F, typename... Args>
auto batch_dispatch(int mode, bool ko6, int tz, bool vac, Args... args) {
#define NUOSC_BATCH_V(R, M, Z) \
    (vac ? F<T, R, M, Z, true, M64>::run(args...) : F<T, R, M, Z, false, M64>::run(args...))
#define NUOSC_BATCH_TZ(R, M) (tz == 16 ? NUOSC_BATCH_V(R, M, 16) : NUOSC_BATCH_V(R, M, 8))
#define NUOSC_BATCH_MODE(R)                                                                                   \
    (mode == MODE_S1Y   ? NUOSC_BATCH_TZ(R, MODE_S1Y)                                                         \
     : mode == MODE_S2B ? NUOSC_BATCH_TZ(R, MODE_S2B)                                                         \
     : mode == MODE_SY  ? NUOSC_BATCH_TZ(R, MODE_SY)                                                          \
                        : NUOSC_BATCH_TZ(R, MODE_S4B))
    return ko6 ? NUOSC_BATCH_MODE(3) : NUOSC_BATCH_MODE(2);
#undef NUOSC_BATCH_MODE
#undef NUOSC_BATCH_TZ
#undef NUOSC_BATCH_V
}

template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
struct BatchGrid {
    static int run(int device) { return batch_grid_t<T, R, MODE, TZ, VAC, M64>(device); }
};
template <typename T, int R, int MODE, int TZ, bool VAC, bool M64>
struct BatchLaunch {
    static cudaError_t run(const void *items, const long long *starts, int n, long long ntiles,
                           unsigned long long *counter, const int *halt, int grid, cudaStream_t s) {
        return batch_launch_t<T, R, MODE, TZ, VAC, M64>(items, starts, n, ntiles, counter, halt, grid, s);
    }
};

}  // namespace

template <typename T>
bool xtma_supported(const Geom &g, XTile t) {
    // nz >= tz + 6: the widest box (tz + 2R rows, R <= 3) fits in the z extent;
    // 3 fs < 2^32: the march's per-plane offsets within a flavour half are
    // 32-bit (registers of up to 91 GB in FP64, 45 GB in FP32: every state
    // whose four registers fit a B200)
    return (t.tz == 8 || t.tz == 16) && g.nz % t.tz == 0 && g.nz >= t.tz + 6 && g.nx >= 4 &&
           g.nvs % vpt<T>() == 0 && 3 * g.fs < (1ll << 32) && encode_fn() != nullptr;
}

template <typename T>
size_t xtma_batch_item_bytes() {
    return sizeof(BatchItem<T>);
}

template <typename T>
long long xtma_batch_fill(void *item, const StageArgs<T> &a, bool ko6, int tz, int lx) {
    if (!xtma_supported<T>(a.g, XTile{tz, lx, vblock<T>()}) || lx < 1 || !a.mom_part) return -1;
    BatchItem<T> e;
    memset((void *)&e, 0, sizeof e);
    if (!make_maps<T>(&e.maps, a, tz, ko6 ? 3 : 2)) return -1;
    e.a = a;
    e.ntz = a.g.nz / tz;
    e.nvb = xtma_num_vblocks<T>(a.g);
    e.nvbm = march_vblocks<T>(a.g);
    e.lx = lx;
    e.nseg = (a.g.nx + lx - 1) / lx;
    memcpy(item, (const void *)&e, sizeof e);
    return (long long)e.ntz * e.nvbm * 2 * e.nseg;
}

template <typename T>
int xtma_batch_grid(int mode, bool ko6, int tz, bool vac, bool m64, int device) {
    if ((tz != 8 && tz != 16) || !tma_mode(mode)) return -1;
    if constexpr (sizeof(T) == 8) return batch_dispatch<T, true, BatchGrid>(mode, ko6, tz, vac, device);
    else
        return m64 ? batch_dispatch<T, true, BatchGrid>(mode, ko6, tz, vac, device)
                   : batch_dispatch<T, false, BatchGrid>(mode, ko6, tz, vac, device);
}

template <typename T>
cudaError_t launch_stage_xtma_batch(const void *items, const long long *starts, int n, long long ntiles,
                                    unsigned long long *counter, const int *halt, int mode, bool ko6, int tz,
                                    bool vac, bool m64, int grid, cudaStream_t s) {
    if ((tz != 8 && tz != 16) || !tma_mode(mode) || n < 1 || grid < 1)
        return cudaErrorInvalidValue;
    if constexpr (sizeof(T) == 8)
        return batch_dispatch<T, true, BatchLaunch>(mode, ko6, tz, vac, items, starts, n, ntiles, counter, halt, grid,
                                                    s);
    else
        return m64 ? batch_dispatch<T, true, BatchLaunch>(mode, ko6, tz, vac, items, starts, n, ntiles, counter, halt,
                                                          grid, s)
                   : batch_dispatch<T, false, BatchLaunch>(mode, ko6, tz, vac, items, starts, n, ntiles, counter,
                                                           halt, grid, s);
}

template <typename T>
int xtma_num_vblocks(const Geom &g) {
    return (g.nvs + vblock<T>() - 1) / vblock<T>();
}

template <typename T>
int xtma_tail_v0(const Geom &g) {
    const int nvb = xtma_num_vblocks<T>(g), last = (nvb - 1) * vblock<T>();
    return 4 * (g.nvs - last) <= vblock<T>() ? last : g.nvs;
}

template <typename T>
cudaError_t launch_stage_xtma(const StageArgs<T> &a, int mode, bool ko6, XTile t, cudaStream_t s) {
    if (!a.mom_part || a.g.nz % t.tz) return cudaErrorInvalidValue;
    if (t.tz == 16) return ko6 ? launch_tms<T, 3, 16>(a, mode, t, s) : launch_tms<T, 2, 16>(a, mode, t, s);
    return ko6 ? launch_tms<T, 3, 8>(a, mode, t, s) : launch_tms<T, 2, 8>(a, mode, t, s);
}

template bool xtma_supported<double>(const Geom &, XTile);
template bool xtma_supported<float>(const Geom &, XTile);
template int xtma_num_vblocks<double>(const Geom &);
template int xtma_num_vblocks<float>(const Geom &);
template int xtma_tail_v0<double>(const Geom &);
template int xtma_tail_v0<float>(const Geom &);
template cudaError_t launch_stage_xtma<double>(const StageArgs<double> &, int, bool, XTile, cudaStream_t);
template cudaError_t launch_stage_xtma<float>(const StageArgs<float> &, int, bool, XTile, cudaStream_t);
template size_t xtma_batch_item_bytes<double>();
template size_t xtma_batch_item_bytes<float>();
template long long xtma_batch_fill<double>(void *, const StageArgs<double> &, bool, int, int);
template long long xtma_batch_fill<float>(void *, const StageArgs<float> &, bool, int, int);
template int xtma_batch_grid<double>(int, bool, int, bool, bool, int);
template int xtma_batch_grid<float>(int, bool, int, bool, bool, int);
template cudaError_t launch_stage_xtma_batch<double>(const void *, const long long *, int, long long,
                                                     unsigned long long *, const int *, int, bool, int, bool, bool,
                                                     int, cudaStream_t);
template cudaError_t launch_stage_xtma_batch<float>(const void *, const long long *, int, long long,
                                                    unsigned long long *, const int *, int, bool, int, bool, bool,
                                                    int, cudaStream_t);

}  // namespace nuosc
