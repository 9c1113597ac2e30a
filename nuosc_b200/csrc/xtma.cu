// xtma.cu -- TMA-fed x-march stage kernel (the fast path of the fused stage).
//
// Same arithmetic and per-thread structure as xmarch.cu (one (z, v) column per
// thread, (2R+1)-deep register queue in x, fused RK epilogue and moment
// partials), but the data movement is Blackwell-native:
//   * per x plane, lane 0 of warp 0 issues TMA tensor loads
//     (cp.async.bulk.tensor.4d) of the whole centre-plane box with its z halo
//     ([TZ+2R rows][4 fields][32 velocities], split into 2-3 boxes where the
//     periodic z wrap cuts it), of the queue front plane, and a bulk copy of
//     the TZ cells' moments, into an NS-deep shared ring; completion is
//     tracked by one "full" mbarrier per ring slot (expect_tx bytes);
//   * every consumer warp reads its z stencil straight from the box, so warps
//     never exchange data and there is no CTA-wide barrier in the march: a
//     warp waits only on the slot's full barrier and releases the slot by
//     arriving on its "empty" mbarrier; the issuing lane waits on "empty"
//     before refilling a slot;
//   * the pointwise U and A inputs of the epilogue are plain coalesced loads
//     issued before the stencil arithmetic, so the ring holds only what the
//     stencil needs and can be deep.
// All mbarrier waits are bounded: on expiry the kernel records
// NUOSC_ERR_TIMEOUT in the status word, stops marching and, before
// returning, waits (again bounded) for the copies it issued.
// Requires nz % TZ == 0; other geometries use the cp.async kernel.
#include "internal.cuh"
#include "physics.cuh"

#include <cuda.h>

namespace nuosc {

namespace {

constexpr int VB = 32;
constexpr unsigned kWaitSpins = 1u << 22;  // bounded mbarrier waits (seconds at most)

struct __align__(64) TmaMaps {
    CUtensorMap zr;   // box of TZ+2R rows (centre plane + both halos)
    CUtensorMap tzr;  // TZ+R rows (a halo cut by the wrap)
    CUtensorMap tz;   // TZ rows (front plane; middle piece of a fully wrapped box)
    CUtensorMap r;    // R rows (wrapped halo)
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
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    for (unsigned it = 0; it < kWaitSpins; ++it) {
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
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

constexpr int up128(int x) { return (x + 127) / 128 * 128; }

// shared layout of one ring slot: zb [ZR][4][VB] T | fr [TZ][4][VB] T | mb [TZ][12] double
template <typename T, int TZ, int R>
struct Slot {
    static constexpr int ZR = TZ + 2 * R;
    static constexpr int zb = 0;
    static constexpr int fr = up128(zb + (int)sizeof(T) * ZR * 4 * VB);
    static constexpr int mb = up128(fr + (int)sizeof(T) * TZ * 4 * VB);
    static constexpr int bytes = up128(mb + 8 * TZ * NMOM);
    static constexpr unsigned tx = sizeof(T) * (ZR + TZ) * 4 * VB + 8 * TZ * NMOM;  // bytes landing per plane
};

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

template <typename T>
__device__ __forceinline__ void rhs_half(const T (&c)[4], T a, T b, T e, T mu, T pmo, T ct, T st, const T (&sten)[4],
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

template <int TZ>
constexpr int tma_ctas_per_sm() {
    return TZ == 16 ? 1 : 2;
}

}  // namespace

template <typename T, int R, int MODE, int TZ, int NS>
__global__ void __launch_bounds__(VB *TZ, tma_ctas_per_sm<TZ>())
    k_xtma(const __grid_constant__ TmaMaps maps, const StageArgs<T> a, int LX) {
    using S = Slot<T, TZ, R>;
    constexpr int W = 2 * R + 1;
    constexpr int ZR = S::ZR;
    constexpr int D = NS - 2 > 0 ? NS - 2 : 1;  // planes issued ahead (slack of NS-D slots)
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned long long *bars = (unsigned long long *)(smem + NS * S::bytes);  // full[NS], empty[NS]
    __shared__ int s_abort;

    const Geom g = a.g;
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    const int z0 = blockIdx.x * TZ;
    const int vb = blockIdx.y;
    const int v = vb * VB + lane;
    const bool vact = v < g.nvs;
    const int seg = blockIdx.z >> 1, half = blockIdx.z & 1;
    const int xs = seg * LX;
    if (xs >= g.nx) return;
    const int xe = min(xs + LX, g.nx);
    const int nplanes = xe - xs;
    const int zr = z0 + r;  // always < nz (nz % TZ == 0)
    const long long fs = g.fs;
    const long long P = (long long)g.nz * g.nvs;
    const long long hoff = (long long)half * 4 * fs;
    const T *in = a.in + hoff;
    const int vc = vact ? v : 0;
    const long long own = (long long)zr * g.nvs + vc;
    const int nvb = gridDim.y;

    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < 2 * NS; ++s) mbar_init(smem_u32(&bars[s]), s < NS ? 1u : (unsigned)TZ);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // lane 0 of warp 0 issues the loads of plane index i (x = xs + i) into slot i % NS
    auto issue = [&](int i) -> bool {
        const int s = i % NS;
        if (i >= NS && !mbar_wait(smem_u32(&bars[NS + s]), (unsigned)((i / NS - 1) & 1))) return false;
        const unsigned full = smem_u32(&bars[s]);
        unsigned char *sp = smem + s * S::bytes;
        mbar_expect_tx(full, S::tx);
        const int x = xs + i;
        const int c1 = 4 * half, c0 = vb * VB;
        // centre box rows z0-R .. z0+TZ+R-1 (periodic), as 1-3 contiguous pieces
        int zstart = z0 - R, dst = 0;
        while (dst < ZR) {
            const int zw = zstart < 0 ? zstart + g.nz : (zstart >= g.nz ? zstart - g.nz : zstart);
            int len = g.nz - zw;
            if (len > ZR - dst) len = ZR - dst;
            const CUtensorMap *m = len == ZR ? &maps.zr : len == TZ + R ? &maps.tzr : len == TZ ? &maps.tz : &maps.r;
            tma_load_4d(smem_u32(sp + S::zb + dst * 4 * VB * sizeof(T)), m, c0, c1, zw, x, full);
            zstart += len;
            dst += len;
        }
        const int xf = x + R < g.nx ? x + R : x + R - g.nx;
        tma_load_4d(smem_u32(sp + S::fr), &maps.tz, c0, c1, z0, xf, full);
        bulk_load(smem_u32(sp + S::mb), a.mom_in + ((long long)x * g.nz + z0) * NMOM, 8u * TZ * NMOM, full);
        return true;
    };

    // per-velocity and uniform constants
    const double vxd = a.q.vx[vc], vyd = a.q.vy[vc], vzd = a.q.vz[vc], wd = vact ? a.q.vw[vc] : 0.0;
    const T fx = T(vxd * a.c.fxs), fz = T(vzd * a.c.fzs);
    const T kz3 = T(a.c.kz3), kz2 = T(a.c.kz2), kz1 = T(a.c.kz1);
    const T kx3 = T(a.c.kx3), kx2 = T(a.c.kx2), kx1 = T(a.c.kx1), kc = T(a.c.kc);
    const T mu = T(a.c.mu), pmo = T(a.c.pmo), ct = T(a.c.ct), st = T(a.c.st);
    const T cA = T(a.cA), cY = T(a.cY);

    // prime the register queue with planes xs-R .. xs+R-1
    T q[4][W];
#pragma unroll
    for (int p = 0; p < 2 * R; ++p) {
        const long long o = (long long)wrap_index(xs - R + p, g.nx) * P + own;
#pragma unroll
        for (int f = 0; f < 4; ++f) q[f][p] = vact ? in[f * fs + o] : T(0);
    }
    bool ok = true;
    if (tid == 0)
        for (int d = 0; d < D && d < nplanes; ++d) ok = ok && issue(d);

    int done = 0;
    for (int i = 0; i < nplanes; ++i) {
        if (tid == 0 && ok && i + D < nplanes) ok = issue(i + D);
        if (tid == 0 && !ok) s_abort = 1;
        const int s = i % NS;
        const int x = xs + i;
        // pointwise epilogue inputs first (they are not in the ring)
        const long long oc = hoff + (long long)x * P + own;
        T uin[4], ain[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            uin[f] = (MODE == MODE_S23 && vact) ? a.u[oc + f * fs] : T(0);
            ain[f] = (MODE != MODE_S1 && vact) ? a.acc_src[oc + f * fs] : T(0);
        }
        if (!mbar_wait(smem_u32(&bars[s]), (unsigned)((i / NS) & 1)) || *(volatile int *)&s_abort) {
            s_abort = 1;
            break;
        }
        const unsigned char *sp = smem + s * S::bytes;
        const T *zb = (const T *)(sp + S::zb);
        const T *fr = (const T *)(sp + S::fr);
        const double *mb = (const double *)(sp + S::mb);
#pragma unroll
        for (int f = 0; f < 4; ++f) q[f][2 * R] = vact ? fr[(r * 4 + f) * VB + lane] : T(0);

        T sten[4], cen[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            T zs[W];
#pragma unroll
            for (int k = 0; k < W; ++k) zs[k] = zb[((r + k) * 4 + f) * VB + lane];
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
        // the slot's shared data is consumed: release it
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&bars[NS + s]));

        const T ia = T(inp(m, vxd, vyd, vzd)), ib = T(inp(m + 4, vxd, vyd, vzd)), ie = T(inp(m + 8, vxd, vyd, vzd));
        T kk[4];
        rhs_half(cen, ia, ib, ie, mu, pmo, ct, st, sten, kk);

        T outm[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (MODE == MODE_S1) {
                const T A = cen[f] + cA * kk[f];
                const T Y = cen[f] + cY * kk[f];
                if (vact) {
                    a.acc_dst[oc + f * fs] = A;
                    a.y_dst[oc + f * fs] = Y;
                }
                outm[f] = Y;
            } else if (MODE == MODE_S23) {
                const T A = ain[f] + cA * kk[f];
                const T Y = uin[f] + cY * kk[f];
                if (vact) {
                    a.acc_dst[oc + f * fs] = A;
                    a.y_dst[oc + f * fs] = Y;
                }
                outm[f] = Y;
            } else {
                const T A = ain[f] + cA * kk[f];
                if (vact) a.acc_dst[oc + f * fs] = A;
                outm[f] = A;
            }
        }
        {
            double d0, d1, d2;
            if (half == 0) moment_terms<false>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
            else moment_terms<true>(outm[0], outm[1], outm[2], outm[3], d0, d1, d2);
            if (!vact) d0 = d1 = d2 = 0.0;
            const double v4w[4] = {wd, vxd * wd, vyd * wd, vzd * wd};
            double mp[16];
#pragma unroll
            for (int s4 = 0; s4 < 4; ++s4) {
                mp[s4] = v4w[s4] * d0;
                mp[4 + s4] = v4w[s4] * d1;
                mp[8 + s4] = v4w[s4] * d2;
                mp[12 + s4] = 0.0;
            }
            rs_step<16, 16>(mp, lane);
            rs_step<8, 8>(mp, lane);
            rs_step<4, 4>(mp, lane);
            rs_step<2, 2>(mp, lane);
            mp[0] += __shfl_xor_sync(0xffffffffu, mp[0], 1);
            const int idx = lane >> 1;
            if ((lane & 1) == 0 && idx < NMOM) {
                const long long cell = (long long)x * g.nz + zr;
                a.mom_part[((cell * nvb + vb) * 2 + half) * NMOM + idx] = mp[0];
            }
        }
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int k = 0; k < 2 * R; ++k) q[f][k] = q[f][k + 1];
        done = i + 1;
    }
    (void)done;
    __syncthreads();
    if (tid == 0 && s_abort) {
        // a wait expired: report it, then drain (bounded) every slot that may
        // still receive a copy before the CTA's shared memory is released
        atomicExch(a.status, NUOSC_TIMEOUT_CODE);
        for (int s = 0; s < NS; ++s) {
            mbar_wait(smem_u32(&bars[s]), 0);
            mbar_wait(smem_u32(&bars[s]), 1);
        }
    }
}

// ------------------------------------------------------------------ host side
namespace {

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

// 4D view of one register: (v, field, z, x) with box {32, 4, rows, 1}
template <typename T>
bool make_map(CUtensorMap *m, const T *base, const Geom &g, int rows) {
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nvs, 8, (cuuint64_t)g.nz, (cuuint64_t)g.nx};
    const cuuint64_t strides[3] = {(cuuint64_t)g.fs * sizeof(T), (cuuint64_t)g.nvs * sizeof(T),
                                   (cuuint64_t)g.nz * g.nvs * sizeof(T)};
    const cuuint32_t box[4] = {(cuuint32_t)VB, 4, (cuuint32_t)rows, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return fn(m, dt, 4, (void *)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int TZ, int R>
constexpr int tma_ring() {
    constexpr int b = Slot<T, TZ, R>::bytes + 16;
    constexpr int cap = 227 * 1024 / tma_ctas_per_sm<TZ>() - 1024;
    return cap / b >= 6 ? 6 : cap / b >= 5 ? 5 : cap / b >= 4 ? 4 : 3;
}

template <typename T, int R, int MODE, int TZ>
cudaError_t launch_t(const StageArgs<T> &a, XTile t, cudaStream_t s) {
    constexpr int NS = tma_ring<T, TZ, R>();
    using Sl = Slot<T, TZ, R>;
    TmaMaps maps;
    if (!make_map<T>(&maps.zr, a.in, a.g, TZ + 2 * R) || !make_map<T>(&maps.tzr, a.in, a.g, TZ + R) ||
        !make_map<T>(&maps.tz, a.in, a.g, TZ) || !make_map<T>(&maps.r, a.in, a.g, R))
        return cudaErrorInvalidValue;
    const size_t smem = (size_t)NS * Sl::bytes + 2 * NS * 8;
    cudaError_t e =
        cudaFuncSetAttribute(k_xtma<T, R, MODE, TZ, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int nseg = (a.g.nx + t.lx - 1) / t.lx;
    dim3 grid(a.g.nz / TZ, (a.g.nvs + VB - 1) / VB, nseg * 2);
    k_xtma<T, R, MODE, TZ, NS><<<grid, VB * TZ, smem, s>>>(maps, a, t.lx);
    return cudaGetLastError();
}

template <typename T, int R, int TZ>
cudaError_t launch_tm(const StageArgs<T> &a, int mode, XTile t, cudaStream_t s) {
    switch (mode) {
    case MODE_S1: return launch_t<T, R, MODE_S1, TZ>(a, t, s);
    case MODE_S23: return launch_t<T, R, MODE_S23, TZ>(a, t, s);
    case MODE_S4: return launch_t<T, R, MODE_S4, TZ>(a, t, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

template <typename T>
bool xtma_supported(const Geom &g, XTile t) {
    return (t.tz == 8 || t.tz == 16) && g.nz % t.tz == 0 && g.nx >= 4 && encode_fn() != nullptr;
}

template <typename T>
cudaError_t launch_stage_xtma(const StageArgs<T> &a, int mode, bool ko6, XTile t, cudaStream_t s) {
    if (!a.mom_part || a.g.nz % t.tz) return cudaErrorInvalidValue;
    if (t.tz == 16) return ko6 ? launch_tm<T, 3, 16>(a, mode, t, s) : launch_tm<T, 2, 16>(a, mode, t, s);
    return ko6 ? launch_tm<T, 3, 8>(a, mode, t, s) : launch_tm<T, 2, 8>(a, mode, t, s);
}

template bool xtma_supported<double>(const Geom &, XTile);
template bool xtma_supported<float>(const Geom &, XTile);
template cudaError_t launch_stage_xtma<double>(const StageArgs<double> &, int, bool, XTile, cudaStream_t);
template cudaError_t launch_stage_xtma<float>(const StageArgs<float> &, int, bool, XTile, cudaStream_t);

}  // namespace nuosc
