// xmarch.cu -- fused RK4 stage kernel that marches along x.
//
// One CTA owns TZ consecutive z rows x 32 consecutive velocities x one flavour
// half (fields ee,mm,emr,emi or their barred partners) and walks a segment of
// LX x planes.  Per thread (one (z, v) column):
//   * a (2R+1)-deep register queue in x per field holds the x stencil, so each
//     state value is read from HBM once per stage (plus the z halo rows and
//     the 2R planes that prime each segment);
//   * the centre plane goes through shared memory for the z stencil;
//   * the inputs of the planes ahead (queue front, z-halo rows, the U and A
//     registers, cell moments) are staged by cp.async into an NS-deep
//     shared-memory ring, NS-1 planes ahead, with one barrier per plane;
//   * the epilogue applies the RK-stage update and accumulates the velocity
//     moments of the state it writes: a reduce-scatter over the 32
//     velocities of the warp gives one partial per (cell, velocity block,
//     half); moment_finalize sums the partials in a fixed order, so the next
//     stage needs no separate moment pass and results are deterministic.
// ADV and KO of one field are accumulated as one FMA chain over the symmetric
// sums x[-k]+x[+k] and differences x[-k]-x[+k]; this reassociates the
// reference's ADV_FD + KO_FD (nuosc_class.cpp:112-183) at the last-bit level.
// Periodic wrap in x and z is index arithmetic.
#include "internal.cuh"
#include "physics.cuh"

#include <dlfcn.h>

#include <array>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

namespace nuosc {

namespace {

constexpr int VB = 32;

__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// shared-memory layout of one pipeline stage (all offsets 16-byte aligned);
// S1 stages no U or A, S4 no U
template <typename T, int TZ, int R, int MODE>
struct Stage {
    static constexpr int ZR = TZ + 2 * R;
    static constexpr size_t plane = sizeof(T) * 4 * TZ * VB;
    static constexpr size_t zb = 0;                                        // [4][ZR][VB] centre plane + z halo
    static constexpr size_t fr = zb + sizeof(T) * 4 * ZR * VB;             // [4][TZ][VB] queue front
    static constexpr size_t ub = fr + plane;                               // [4][TZ][VB] U       (S2/S3)
    static constexpr size_t ab = ub + (MODE == MODE_S23 ? plane : 0);      // [4][TZ][VB] A       (S2/S3/S4)
    static constexpr size_t mb = ab + (MODE != MODE_S1 ? plane : 0);       // [TZ][12] double, cell moments
    static constexpr size_t bytes = mb + sizeof(double) * TZ * NMOM;
    static_assert(fr % 16 == 0 && mb % 16 == 0 && bytes % 16 == 0, "stage alignment");
};

// ADV + KO along one axis, accumulated into acc; s[0..2R] = x[-R..+R].
template <typename T, int R>
__device__ __forceinline__ T axis_terms(const T (&s)[2 * R + 1], T f, T k3, T k2, T k1, T acc) {
    constexpr int C = R;
    const T t2 = s[C - 2] + s[C + 2], t1 = s[C - 1] + s[C + 1];
    const T d2 = s[C - 2] - s[C + 2], d1 = s[C - 1] - s[C + 1];
    if (R == 3) acc = fma(k3, s[0] + s[6], acc);
    acc = fma(k2, t2, acc);
    acc = fma(k1, t1, acc);
    return fma(f, fma(T(-8), d1, d2), acc);
}

// commutator + vacuum terms of one flavour half on top of the stencil sum
template <typename T>
__device__ __forceinline__ void rhs_half(const T (&c)[4], T a, T b, T e, T mu, T pmo, T ct, T st, T (&sten)[4],
                                         T (&out)[4]) {
    const T ee = c[0], mm = c[1], emr = c[2], emi = c[3];
    const T Iee = T(2) * mu * (emi * a + emr * b);
    const T Iemr = -mu * ((ee - mm) * b + e * emi);
    const T Iemi = mu * ((mm - ee) * a + e * emr);
    out[0] = Iee + sten[0] - pmo * T(2) * st * emi;
    out[1] = -Iee + sten[1] + pmo * T(2) * st * emi;
    out[2] = Iemr + sten[2] - pmo * T(2) * ct * emi;
    out[3] = Iemi + sten[3] + pmo * (T(2) * ct * emr + st * (ee - mm));
}

// one reduce-scatter step over lane pairs (lane, lane^O): N values -> N/2
template <int N, int O>
__device__ __forceinline__ void rs_step(double (&m)[16], int lane) {
    const bool up = (lane & O) != 0;
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
        const double send = up ? m[i] : m[i + N / 2];
        const double keep = up ? m[i + N / 2] : m[i];
        m[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
}

}  // namespace

// CTAs per SM the tile is built for: 8-row tiles run two, 4-row tiles four
// independent CTAs per SM, so some compute while others wait at their
// per-plane barrier.
template <int TZ>
constexpr int ctas_per_sm() {
    return TZ == 4 ? 4 : TZ == 8 ? 2 : 1;
}

template <typename T, int R, int MODE, int TZ, int NS>
__global__ void __launch_bounds__(VB *TZ, ctas_per_sm<TZ>()) k_xmarch(StageArgs<T> a, int LX) {
    using S = Stage<T, TZ, R, MODE>;
    constexpr int W = 2 * R + 1;
    constexpr int ZR = S::ZR;
    constexpr int D = NS - 1;                 // planes staged ahead
    constexpr int NHR = 4 * 2 * R;            // z-halo rows per plane (4 fields)
    constexpr int NH = (NHR + TZ - 1) / TZ;   // halo rows per warp
    extern __shared__ __align__(16) unsigned char smem[];

    const Geom g = a.g;
    const int lane = threadIdx.x, r = threadIdx.y, tid = r * VB + lane;
    const int z0 = blockIdx.x * TZ;
    const int vb = blockIdx.y;
    const int v = vb * VB + lane;
    const bool vact = v < g.nvs;
    const int seg = blockIdx.z >> 1, half = blockIdx.z & 1;
    const int xs = seg * LX;
    if (xs >= g.nx) return;
    const int xe = min(xs + LX, g.nx);
    const int zr = z0 + r;
    const bool zact = zr < g.nz;
    const bool act = vact && zact;
    const long long fs = g.fs;
    const long long P = (long long)g.nz * g.nvs;  // elements per x plane of one field
    const long long hoff = (long long)half * 4 * fs;
    const T *in = a.in + hoff;
    const int vc = vact ? v : 0;
    const long long own_ld = (long long)wrap_index(zr, g.nz) * g.nvs + vc;  // this column (wrapped) for loads
    const long long own_st = (long long)(zact ? zr : 0) * g.nvs + vc;       // this column for U/A and stores
    const int nvb = gridDim.y;

    // z-halo rows staged by this warp (plane-independent part of the address)
    long long h_off[NH];
    int h_sm[NH];
    bool h_ok[NH];
#pragma unroll
    for (int k = 0; k < NH; ++k) {
        const int hrow = r + k * TZ;
        h_ok[k] = vact && hrow < NHR;
        const int f = hrow / (2 * R), hr = hrow - f * (2 * R);
        const int kb = hr < R ? hr : TZ + hr;
        h_off[k] = f * fs + (long long)wrap_index(z0 - R + kb, g.nz) * g.nvs + vc;
        h_sm[k] = (f * ZR + kb) * VB + lane;
    }
    // cell moments of the TZ rows: threads tid < TZ*6 copy 16 bytes each
    const bool m_ok = tid < TZ * NMOM / 2 && z0 + (2 * tid) / NMOM < g.nz;
    const long long m_off = (long long)z0 * NMOM + 2 * tid;

    // per-velocity constants (constant along the march)
    const double vxd = a.q.vx[vc], vyd = a.q.vy[vc], vzd = a.q.vz[vc], wd = vact ? a.q.vw[vc] : 0.0;
    const T fx = T(vxd * a.c.fxs), fz = T(vzd * a.c.fzs);
    const T kz3 = T(a.c.kz3), kz2 = T(a.c.kz2), kz1 = T(a.c.kz1);
    const T kx3 = T(a.c.kx3), kx2 = T(a.c.kx2), kx1 = T(a.c.kx1), kc = T(a.c.kc);
    const T mu = T(a.c.mu), pmo = T(a.c.pmo), ct = T(a.c.ct), st = T(a.c.st);
    const T cA = T(a.cA), cY = T(a.cY);

    auto issue = [&](int xn, int b) {
        unsigned char *sp = smem + (size_t)b * S::bytes;
        T *zb = (T *)(sp + S::zb);
        T *fr = (T *)(sp + S::fr);
        T *ubuf = (T *)(sp + S::ub);
        T *abuf = (T *)(sp + S::ab);
        double *mb = (double *)(sp + S::mb);
        const int xf = xn + R < g.nx ? xn + R : xn + R - g.nx;
        const long long xo = (long long)xn * P;
        if (vact) {
            const T *pf = in + (long long)xf * P + own_ld;
#pragma unroll
            for (int f = 0; f < 4; ++f) cp_async(&fr[(f * TZ + r) * VB + lane], pf + f * fs, sizeof(T));
            if (MODE != MODE_S1 && zact) {
                const long long oc = hoff + xo + own_st;
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    if (MODE == MODE_S23) cp_async(&ubuf[(f * TZ + r) * VB + lane], a.u + oc + f * fs, sizeof(T));
                    cp_async(&abuf[(f * TZ + r) * VB + lane], a.acc_src + oc + f * fs, sizeof(T));
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NH; ++k)
            if (h_ok[k]) cp_async(&zb[h_sm[k]], in + h_off[k] + xo, sizeof(T));
        if (m_ok) cp_async(&mb[2 * tid], a.mom_in + (long long)xn * g.nz * NMOM + m_off, 16);
    };

    // prime the queue with planes xs-R .. xs+R-1 and stage the first D planes
    T q[4][W];
#pragma unroll
    for (int p = 0; p < 2 * R; ++p) {
        const long long o = (long long)wrap_index(xs - R + p, g.nx) * P + own_ld;
#pragma unroll
        for (int f = 0; f < 4; ++f) q[f][p] = vact ? in[f * fs + o] : T(0);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        if (xs + d < xe) issue(xs + d, d);
        cp_async_commit();
    }

    int bi = 0;  // ring slot of plane x
    for (int x = xs; x < xe; ++x) {
        cp_async_wait<D - 1>();
        unsigned char *sp = smem + (size_t)bi * S::bytes;
        T *zb = (T *)(sp + S::zb);
        const T *fr = (const T *)(sp + S::fr);
        const T *ubuf = (const T *)(sp + S::ub);
        const T *abuf = (const T *)(sp + S::ab);
        const double *mb = (const double *)(sp + S::mb);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            q[f][2 * R] = vact ? fr[(f * TZ + r) * VB + lane] : T(0);
            zb[(f * ZR + R + r) * VB + lane] = q[f][R];
        }
        __syncthreads();
        {
            int bn = bi + D;
            if (bn >= NS) bn -= NS;
            if (x + D < xe) issue(x + D, bn);
            cp_async_commit();
        }

        // stencil sums: z from the shared centre plane, x from the register queue
        T sten[4], cen[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T zs[W];
#pragma unroll
            for (int k = 0; k < W; ++k) zs[k] = zb[(f * ZR + r + k) * VB + lane];
            cen[f] = q[f][R];
            T acc = kc * cen[f];
            acc = axis_terms<T, R>(zs, fz, kz3, kz2, kz1, acc);
            sten[f] = axis_terms<T, R>(q[f], fx, kx3, kx2, kx1, acc);
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
        const T ia = T(inp(m, vxd, vyd, vzd)), ib = T(inp(m + 4, vxd, vyd, vzd)), ie = T(inp(m + 8, vxd, vyd, vzd));
        T kk[4];
        rhs_half(cen, ia, ib, ie, mu, pmo, ct, st, sten, kk);

        // RK-stage epilogue
        T outm[4];
        const long long oc = hoff + (long long)x * P + own_st;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (MODE == MODE_S1) {
                const T A = cen[f] + cA * kk[f];
                const T Y = cen[f] + cY * kk[f];
                if (act) {
                    a.acc_dst[oc + f * fs] = A;
                    a.y_dst[oc + f * fs] = Y;
                }
                outm[f] = Y;
            } else if (MODE == MODE_S23) {
                const T A = abuf[(f * TZ + r) * VB + lane] + cA * kk[f];
                const T Y = ubuf[(f * TZ + r) * VB + lane] + cY * kk[f];
                if (act) {
                    a.acc_dst[oc + f * fs] = A;
                    a.y_dst[oc + f * fs] = Y;
                }
                outm[f] = Y;
            } else {
                const T A = abuf[(f * TZ + r) * VB + lane] + cA * kk[f];
                if (act) a.acc_dst[oc + f * fs] = A;
                outm[f] = A;
            }
        }

        // velocity-moment partials of the written state (nuosc_class.cpp:69-71)
        {
            double d0, d1, d2;
            if (half == 0) moment_terms<false>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
            else moment_terms<true>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
            if (!act) d0 = d1 = d2 = 0.0;
            const double v4w[4] = {wd, vxd * wd, vyd * wd, vzd * wd};
            double mp[16];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                mp[s] = v4w[s] * d0;
                mp[4 + s] = v4w[s] * d1;
                mp[8 + s] = v4w[s] * d2;
                mp[12 + s] = 0.0;
            }
            rs_step<16, 16>(mp, lane);
            rs_step<8, 8>(mp, lane);
            rs_step<4, 4>(mp, lane);
            rs_step<2, 2>(mp, lane);
            mp[0] += __shfl_xor_sync(0xffffffffu, mp[0], 1);
            const int idx = lane >> 1;  // lanes 2k, 2k+1 hold moment k
            if (zact && (lane & 1) == 0 && idx < NMOM) {
                const long long cell = (long long)x * g.nz + zr;
                a.mom_part[((cell * nvb + vb) * 2 + half) * NMOM + idx] = mp[0];
            }
        }

#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int k = 0; k < 2 * R; ++k) q[f][k] = q[f][k + 1];
        bi = bi + 1 == NS ? 0 : bi + 1;
    }
    cp_async_wait<0>();
}

// Sum the partial moments of each cell over velocity blocks and halves in a
// fixed order: one thread per (cell, moment).
__global__ void k_moment_finalize(const double *__restrict__ part, double *__restrict__ mom, long long ncell,
                                  int nvb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell * NMOM) return;
    const long long cell = t / NMOM;
    const int k = (int)(t - cell * NMOM);
    const double *p = part + cell * nvb * 2 * NMOM + k;
    double s = 0.0;
    for (int b = 0; b < 2 * nvb; ++b) s += p[(long long)b * NMOM];
    mom[t] = s;
}

int xmarch_num_vblocks(const Geom &g, XTile) { return (g.nvs + VB - 1) / VB; }

template <typename T>
bool xmarch_supported(const Geom &g, bool, XTile t) {
    return (t.tz == 4 || t.tz == 8 || t.tz == 16) && t.lx >= 1 && t.vb == VB && g.nx >= 4 && g.nz >= 1;
}

namespace {

// deepest ring (4, 3 or 2 planes) that lets ctas_per_sm CTAs share the SM's 228 KB
template <typename T, int TZ, int R, int MODE>
constexpr int ring_depth() {
    constexpr size_t b = Stage<T, TZ, R, MODE>::bytes, cap = 228 * 1024;
    return ctas_per_sm<TZ>() * (4 * b + 1024) <= cap ? 4 : ctas_per_sm<TZ>() * (3 * b + 1024) <= cap ? 3 : 2;
}

template <typename T, int R, int MODE, int TZ>
cudaError_t launch_x(const StageArgs<T> &a, XTile t, cudaStream_t s) {
    constexpr int NS = ring_depth<T, TZ, R, MODE>();
    const size_t smem = NS * Stage<T, TZ, R, MODE>::bytes;
    cudaError_t e = cudaFuncSetAttribute(k_xmarch<T, R, MODE, TZ, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int nseg = (a.g.nx + t.lx - 1) / t.lx;
    dim3 grid((a.g.nz + TZ - 1) / TZ, (a.g.nvs + VB - 1) / VB, nseg * 2);
    dim3 block(VB, TZ);
    k_xmarch<T, R, MODE, TZ, NS><<<grid, block, smem, s>>>(a, t.lx);
    return cudaGetLastError();
}

template <typename T, int R, int TZ>
cudaError_t launch_mode(const StageArgs<T> &a, int mode, XTile t, cudaStream_t s) {
    switch (mode) {
    case MODE_S1: return launch_x<T, R, MODE_S1, TZ>(a, t, s);
    case MODE_S23: return launch_x<T, R, MODE_S23, TZ>(a, t, s);
    case MODE_S4: return launch_x<T, R, MODE_S4, TZ>(a, t, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

template <typename T>
cudaError_t launch_stage_xmarch(const StageArgs<T> &a, int mode, bool ko6, XTile t, cudaStream_t s) {
    if (!a.mom_part) return cudaErrorInvalidValue;
    if (t.tz == 16) return ko6 ? launch_mode<T, 3, 16>(a, mode, t, s) : launch_mode<T, 2, 16>(a, mode, t, s);
    if (t.tz == 8) return ko6 ? launch_mode<T, 3, 8>(a, mode, t, s) : launch_mode<T, 2, 8>(a, mode, t, s);
    return ko6 ? launch_mode<T, 3, 4>(a, mode, t, s) : launch_mode<T, 2, 4>(a, mode, t, s);
}

cudaError_t launch_moment_finalize(const double *part, double *mom, Geom g, int nvb, cudaStream_t s) {
    const long long n = g.ncell * NMOM;
    k_moment_finalize<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, mom, g.ncell, nvb);
    return cudaGetLastError();
}

namespace {
// k_moment_finalize over the cells of many instances (same summation order)
__global__ void k_moment_finalize_batch(const FinalizeItem *__restrict__ items, const long long *__restrict__ starts,
                                        int n, long long total, const int *__restrict__ halt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    if (halt && halt[lo]) return;  // a stopped instance keeps its moments
    const FinalizeItem e = items[lo];
    const long long u = t - starts[lo];
    const long long cell = u / NMOM;
    const int k = (int)(u - cell * NMOM);
    const double *p = e.part + cell * e.nvb * 2 * NMOM + k;
    double s = 0.0;
    for (int b = 0; b < 2 * e.nvb; ++b) s += p[(long long)b * NMOM];
    e.mom[u] = s;
}
}  // namespace

cudaError_t launch_moment_finalize_batch(const FinalizeItem *items, const long long *starts, int n, long long total,
                                         const int *halt, cudaStream_t s) {
    if (n < 1 || total < 1) return cudaErrorInvalidValue;
    k_moment_finalize_batch<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(items, starts, n, total, halt);
    return cudaGetLastError();
}

template bool xmarch_supported<double>(const Geom &, bool, XTile);
template bool xmarch_supported<float>(const Geom &, bool, XTile);
template cudaError_t launch_stage_xmarch<double>(const StageArgs<double> &, int, bool, XTile, cudaStream_t);
template cudaError_t launch_stage_xmarch<float>(const StageArgs<float> &, int, bool, XTile, cudaStream_t);

// Tile table keyed on (velocity count, precision): lines "nv precision tz lx
// [kernel]" in tiles.txt beside the library (or the file named by
// NUOSC_TILES), written by the autotuner nuosc_b200/autotune.py; kernel 2 is
// the cp.async x-march, 3 the TMA one.  Shapes not listed use 16 x 128.
XTile autotune_lookup(int nv, int precision) {
    static std::vector<std::array<int, 6>> table;
    static std::once_flag once;
    std::call_once(once, [] {
        std::string path;
        if (const char *env = getenv("NUOSC_TILES")) {
            path = env;
        } else {
            Dl_info info;
            if (dladdr((void *)&autotune_lookup, &info) && info.dli_fname) {
                path = info.dli_fname;
                const size_t slash = path.rfind('/');
                path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/tiles.txt";
            }
        }
        FILE *f = path.empty() ? nullptr : fopen(path.c_str(), "r");
        if (!f) return;
        char line[256];
        while (fgets(line, sizeof line, f)) {
            // nv precision tz lx [kernel [msum]]; msum defaults to FP64 sums
            std::array<int, 6> e{0, 0, 0, 0, 0, 1};
            if (line[0] != '#' && sscanf(line, "%d %d %d %d %d %d", &e[0], &e[1], &e[2], &e[3], &e[4], &e[5]) >= 4)
                table.push_back(e);
        }
        fclose(f);
    });
    for (const auto &e : table)
        if (e[0] == nv && e[1] == precision && (e[2] == 4 || e[2] == 8 || e[2] == 16) && e[3] >= 1)
            return XTile{e[2], e[3], VB, e[4], e[5] != 0};
    return XTile{16, 128, VB, 0, 1};
}

}  // namespace nuosc
