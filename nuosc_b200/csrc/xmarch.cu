// xmarch.cu -- fused RK4 stage kernel that marches along x.
//
// One CTA owns TZ consecutive z rows x 32 consecutive velocities x one flavour
// half (fields ee,mm,emr,emi or their barred partners) and walks a segment
// of x planes.  Per thread (one (z, v) column):
//   * a (2R+1)-deep register queue in x per field holds the stencil in x, so
//     every state value is read from HBM once per stage (plus the z halo and
//     the 2R planes that prime each segment);
//   * the centre plane goes through shared memory for the z stencil;
//   * the inputs of the next plane (queue front, z-halo rows, U and A
//     registers, cell moments) are staged into a double-buffered shared
//     pipeline with cp.async while the current plane computes;
//   * the epilogue applies the RK-stage update and accumulates the velocity
//     moments of the state it writes (warp butterfly over the 32 velocities,
//     one partial per (cell, velocity block, half)); moment_finalize sums the
//     partials in a fixed order, so the next stage needs no moment pass.
// The physics is the same as k_stage_direct (physics.cuh); only the data
// movement differs.  Periodic wrap in x and z is index arithmetic.
#include "internal.cuh"
#include "physics.cuh"

namespace nuosc {

namespace {

constexpr int VB = 32;

__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem, int bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// shared-memory layout of one pipeline stage
template <typename T, int TZ, int R>
struct Stage {
    static constexpr int ZR = TZ + 2 * R;
    static constexpr size_t zb = 0;                                   // [4][ZR][VB]  centre plane + z halo
    static constexpr size_t fr = zb + sizeof(T) * 4 * ZR * VB;        // [4][TZ][VB]  queue front
    static constexpr size_t ub = fr + sizeof(T) * 4 * TZ * VB;        // [4][TZ][VB]  U
    static constexpr size_t ab = ub + sizeof(T) * 4 * TZ * VB;        // [4][TZ][VB]  A (accumulator)
    static constexpr size_t mb = ab + sizeof(T) * 4 * TZ * VB;        // [TZ][12] double, cell moments
    static constexpr size_t bytes = mb + sizeof(double) * TZ * NMOM;
};

template <typename T>
__device__ __forceinline__ long long off3(int x, int z, int v, const Geom &g) {
    return ((long long)x * g.nz + z) * g.nvs + v;
}

}  // namespace

template <typename T, int R, int MODE, int TZ>
__global__ void __launch_bounds__(VB *TZ, 1) k_xmarch(StageArgs<T> a, int LX) {
    using S = Stage<T, TZ, R>;
    constexpr int W = 2 * R + 1;
    constexpr int ZR = S::ZR;
    extern __shared__ __align__(16) unsigned char smem[];

    const Geom g = a.g;
    const int lane = threadIdx.x, r = threadIdx.y, tid = r * VB + lane;
    const int z0 = blockIdx.x * TZ;
    const int vb = blockIdx.y;
    const int v = vb * VB + lane;
    const bool vact = v < g.nvs;
    const int seg = blockIdx.z >> 1, half = blockIdx.z & 1;
    const int xs = seg * LX;
    const int xe = min(xs + LX, g.nx);
    if (xs >= g.nx) return;
    const int zr = z0 + r;
    const bool zact = zr < g.nz;
    const int zl = wrap_index(zr, g.nz);
    const long long fs = g.fs;
    const long long hoff = (long long)half * 4 * fs;
    const T *in = a.in + hoff;
    const T *u = a.u ? a.u + hoff : nullptr;
    const T *accs = a.acc_src ? a.acc_src + hoff : nullptr;
    T *accd = a.acc_dst + hoff;
    T *yd = a.y_dst ? a.y_dst + hoff : nullptr;
    const int nvb = gridDim.y;

    // per-velocity constants (constant along the march)
    const int vc = vact ? v : 0;
    const double vxd = a.q.vx[vc], vyd = a.q.vy[vc], vzd = a.q.vz[vc], wd = vact ? a.q.vw[vc] : 0.0;
    const T fx = T(vxd * a.c.fxs), fz = T(vzd * a.c.fzs);
    const T kx = T(a.c.kx), kz = T(a.c.kz);
    const double v4w[4] = {wd, vxd * wd, vyd * wd, vzd * wd};
    const T cA = T(a.cA), cY = T(a.cY);

    auto stage_ptr = [&](int b) { return smem + (size_t)b * S::bytes; };

    // issue the copies for the plane with centre xn into buffer b
    auto issue = [&](int xn, int b) {
        unsigned char *st = stage_ptr(b);
        T *zb = (T *)(st + S::zb);
        T *fr = (T *)(st + S::fr);
        T *ubuf = (T *)(st + S::ub);
        T *abuf = (T *)(st + S::ab);
        double *mb = (double *)(st + S::mb);
        const int xf = wrap_index(xn + R, g.nx);
        if (vact) {
            const long long of = off3<T>(xf, zl, v, g);
#pragma unroll
            for (int f = 0; f < 4; ++f) cp_async_elem(&fr[(f * TZ + r) * VB + lane], in + f * fs + of, sizeof(T));
            if (zact && MODE != MODE_S1) {
                const long long oc = off3<T>(xn, zr, v, g);
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    if (MODE == MODE_S23) cp_async_elem(&ubuf[(f * TZ + r) * VB + lane], u + f * fs + oc, sizeof(T));
                    cp_async_elem(&abuf[(f * TZ + r) * VB + lane], accs + f * fs + oc, sizeof(T));
                }
            }
        }
        // z-halo rows of plane xn: buffer rows [0,R) and [R+TZ, ZR)
        for (int h = tid; h < 4 * 2 * R * VB; h += VB * TZ) {
            const int f = h / (2 * R * VB), rem = h - f * (2 * R * VB);
            const int hr = rem / VB, hl = rem - hr * VB;
            const int k = hr < R ? hr : TZ + hr;
            const int vv = vb * VB + hl;
            if (vv < g.nvs) {
                const int zg = wrap_index(z0 - R + k, g.nz);
                cp_async_elem(&zb[(f * ZR + k) * VB + hl], in + f * fs + off3<T>(xn, zg, vv, g), sizeof(T));
            }
        }
        // moments of the TZ cells of plane xn
        for (int e = tid; e < TZ * NMOM; e += VB * TZ) {
            const int row = e / NMOM;
            if (z0 + row < g.nz)
                cp_async_elem(&mb[e], a.mom_in + ((long long)xn * g.nz + z0) * NMOM + e, 8);
        }
    };

    // prime the queue with planes xs-R .. xs+R-1 and stage the first plane
    T q[4][W];
#pragma unroll
    for (int p = 0; p < 2 * R; ++p) {
        const int xp = wrap_index(xs - R + p, g.nx);
        const long long o = off3<T>(xp, zl, v, g);
#pragma unroll
        for (int f = 0; f < 4; ++f) q[f][p] = vact ? in[f * fs + o] : T(0);
    }
    issue(xs, 0);
    cp_async_commit();

    for (int x = xs; x < xe; ++x) {
        const int b = (x - xs) & 1;
        if (x + 1 < xe) issue(x + 1, b ^ 1);
        cp_async_commit();
        cp_async_wait<1>();

        unsigned char *st = stage_ptr(b);
        T *zb = (T *)(st + S::zb);
        const T *fr = (const T *)(st + S::fr);
        const T *ubuf = (const T *)(st + S::ub);
        const T *abuf = (const T *)(st + S::ab);
        const double *mb = (const double *)(st + S::mb);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            q[f][2 * R] = vact ? fr[(f * TZ + r) * VB + lane] : T(0);
            zb[(f * ZR + R + r) * VB + lane] = q[f][R];
        }
        __syncthreads();

        // stencil: z from the shared centre plane, x from the register queue
        T cen[4], adv[4], ko[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T zs[7], xq[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                const int kk = k - 3;
                if (kk >= -R && kk <= R) {
                    zs[k] = zb[(f * ZR + r + R + kk) * VB + lane];
                    xq[k] = q[f][R + kk];
                } else {
                    zs[k] = T(0);
                    xq[k] = T(0);
                }
            }
            cen[f] = q[f][R];
            adv[f] = adv_axis(zs, fz) + adv_axis(xq, fx);
            ko[f] = ko_axis<T, R == 3>(zs, kz) + ko_axis<T, R == 3>(xq, kx);
        }
        const double *m = mb + r * NMOM;
        const T ia = T(inp(m, vxd, vyd, vzd)), ib = T(inp(m + 4, vxd, vyd, vzd)), ie = T(inp(m + 8, vxd, vyd, vzd));
        T kk4[4];
        commutator_half(cen, ia, ib, ie, a.c, kk4, adv, ko);

        // RK-stage epilogue
        T outm[4];
        const bool act = vact && zact;
        const long long oc = off3<T>(x, zact ? zr : 0, v, g);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (MODE == MODE_S1) {
                const T A = cen[f] + cA * kk4[f];
                const T Y = cen[f] + cY * kk4[f];
                if (act) {
                    accd[f * fs + oc] = A;
                    yd[f * fs + oc] = Y;
                }
                outm[f] = Y;
            } else if (MODE == MODE_S23) {
                const T A = abuf[(f * TZ + r) * VB + lane] + cA * kk4[f];
                const T Y = ubuf[(f * TZ + r) * VB + lane] + cY * kk4[f];
                if (act) {
                    accd[f * fs + oc] = A;
                    yd[f * fs + oc] = Y;
                }
                outm[f] = Y;
            } else {
                const T A = abuf[(f * TZ + r) * VB + lane] + cA * kk4[f];
                if (act) accd[f * fs + oc] = A;
                outm[f] = A;
            }
        }
        // velocity-moment partials of the written state (nuosc_class.cpp:69-71)
        double d0, d1, d2;
        if (half == 0) moment_terms<false>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
        else moment_terms<true>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
        double mp[NMOM];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            mp[s] = act ? v4w[s] * d0 : 0.0;
            mp[4 + s] = act ? v4w[s] * d1 : 0.0;
            mp[8 + s] = act ? v4w[s] * d2 : 0.0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < NMOM; ++k) mp[k] += __shfl_xor_sync(0xffffffffu, mp[k], o);
        if (zact && lane < NMOM) {
            double val = mp[0];
#pragma unroll
            for (int k = 1; k < NMOM; ++k)
                if (lane == k) val = mp[k];
            const long long cell = (long long)x * g.nz + zr;
            a.mom_part[((cell * nvb + vb) * 2 + half) * NMOM + lane] = val;
        }

#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int k = 0; k < 2 * R; ++k) q[f][k] = q[f][k + 1];
        __syncthreads();
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
    return (t.tz == 8 || t.tz == 16) && t.lx >= 1 && t.vb == VB && g.nx >= 1 && g.nz >= 1;
}

namespace {

template <typename T, int R, int MODE, int TZ>
cudaError_t launch_x(const StageArgs<T> &a, XTile t, cudaStream_t s) {
    using St = Stage<T, TZ, R>;
    const size_t smem = 2 * St::bytes;
    cudaError_t e = cudaFuncSetAttribute(k_xmarch<T, R, MODE, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int nseg = (a.g.nx + t.lx - 1) / t.lx;
    dim3 grid((a.g.nz + TZ - 1) / TZ, (a.g.nvs + VB - 1) / VB, nseg * 2);
    dim3 block(VB, TZ);
    k_xmarch<T, R, MODE, TZ><<<grid, block, smem, s>>>(a, t.lx);
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
    return ko6 ? launch_mode<T, 3, 8>(a, mode, t, s) : launch_mode<T, 2, 8>(a, mode, t, s);
}

cudaError_t launch_moment_finalize(const double *part, double *mom, Geom g, int nvb, cudaStream_t s) {
    const long long n = g.ncell * NMOM;
    k_moment_finalize<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, mom, g.ncell, nvb);
    return cudaGetLastError();
}

template bool xmarch_supported<double>(const Geom &, bool, XTile);
template bool xmarch_supported<float>(const Geom &, bool, XTile);
template cudaError_t launch_stage_xmarch<double>(const StageArgs<double> &, int, bool, XTile, cudaStream_t);
template cudaError_t launch_stage_xmarch<float>(const StageArgs<float> &, int, bool, XTile, cudaStream_t);

// Tile table keyed on (velocity count, precision), written by the autotuner
// (nuosc_b200/autotune.py); shapes not listed use the default.
XTile autotune_lookup(int nv, int precision) {
    (void)nv;
    (void)precision;
    return XTile{16, 128, VB};
}

}  // namespace nuosc
