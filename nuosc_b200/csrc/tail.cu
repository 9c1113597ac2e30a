// tail.cu -- the last, nearly empty velocity block of an x-march stage.
//
// The TMA x-march kernel runs 32 (FP64) or 64 (FP32) velocities per CTA, one
// or two per lane.  When nv leaves only a few velocities in the last block
// (642 = 20 x 32 + 2 in FP64, 644 = 10 x 64 + 4 in FP32), a CTA for that
// block would issue a full block's instructions for a handful of active
// lanes -- up to a tenth of the stage's issue slots.  Those tail velocities
// are computed here instead, one thread per (cell, tail velocity, flavour
// half) with 4 fields, the stencil read through the read-only cache (the
// tail columns of a few planes stay in L2), the same fused RK epilogue, and
// the velocity-moment partials of the written state summed over the tail
// lanes of the (cell, half) into the last block's slots of the partial
// array, so the fixed-order moment_finalize is unchanged.
#include "internal.cuh"
#include "physics.cuh"

namespace nuosc {

namespace {

// One (cell, velocity, flavour half) of the tail; every lane of the warp
// calls it (the moment reduction shuffles across the twp lanes of a cell and
// half), act says whether the lane holds a real point.  twp: lanes per
// (cell, half) (power of 2).  The commutator couples the four fields of a
// half only to each other once the moments are known, so a half is a
// complete unit of work.
template <typename T, bool KO6, int MODE>
__device__ __forceinline__ void tail_point(const StageArgs<T> &a, const long long cell, const int half, const int v,
                                           const bool act, const int twp, const int nvb, const int lane_in_cell) {
    const Geom g = a.g;
    double mom[NMOM];
#pragma unroll
    for (int k = 0; k < NMOM; ++k) mom[k] = 0.0;
    if (act) {
        const int i = (int)(cell / g.nz), j = (int)(cell - (long long)i * g.nz);
        constexpr int R = KO6 ? 3 : 2;
        const long long hoff = (long long)half * 4 * g.fs;
        const long long P = (long long)g.nz * g.nvs;
        // x neighbours: field-0 pointer of this half and field stride per
        // offset -- inside the register (periodic), or a slab's halo buffer
        long long oz[7];
        const T *xp[7];
        long long xfs[7];
#pragma unroll
        for (int k = -3; k <= 3; ++k) {
            const int kk = (k < -R || k > R) ? 0 : k;
            oz[k + 3] = ((long long)i * g.nz + wrap_index(j + kk, g.nz)) * g.nvs + v;
            const int pl = i + kk;
            if (a.halo && (pl < 0 || pl >= g.nx)) {
                xp[k + 3] = a.halo + halo_offset(4 * half, pl, g.nx, R, P) + (long long)j * g.nvs + v;
                xfs[k + 3] = 2 * R * P;
            } else {
                xp[k + 3] = a.in + hoff + ((long long)wrap_index(pl, g.nx) * g.nz + j) * g.nvs + v;
                xfs[k + 3] = g.fs;
            }
        }
        const double vxd = a.q.vx[v], vyd = a.q.vy[v], vzd = a.q.vz[v], wd = a.q.vw[v];
        const T fx = T(vxd * a.c.fxs), fz = T(vzd * a.c.fzs);
        const T kx = T(a.c.kx), kz = T(a.c.kz);
        const double *m = a.mom_in + cell * NMOM;
        const T ia = T(inp(m, vxd, vyd, vzd)), ib = T(inp(m + 4, vxd, vyd, vzd)), ie = T(inp(m + 8, vxd, vyd, vzd));
        T c4[4], a4[4], k4[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const T *F = a.in + hoff + f * g.fs;
            T zs[7], xs[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                zs[k] = __ldg(F + oz[k]);
                xs[k] = __ldg(xp[k] + f * xfs[k]);
            }
            c4[f] = zs[3];
            a4[f] = adv_axis(zs, fz) + adv_axis(xs, fx);
            k4[f] = ko_axis<T, KO6>(zs, kz) + ko_axis<T, KO6>(xs, kx);
        }
        T kv[4];
        commutator_half(c4, ia, ib, ie, a.c, kv, a4, k4);
        const long long o = oz[3] + hoff;
        const T cA = T(a.cA), cY = T(a.cY);
        T outm[4];  // the written state whose moments the next stage needs
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const long long idx = o + f * g.fs;
            if (MODE == MODE_S1Y) {
                outm[f] = c4[f] + cY * kv[f];  // Y2
                a.y_dst[idx] = outm[f];
            } else if (MODE == MODE_SY) {
                outm[f] = a.u[idx] + cY * kv[f];  // Y4
                a.y_dst[idx] = outm[f];
            } else if (MODE == MODE_S2B) {
                const T u = a.u[idx];
                a.acc_dst[idx] = (u + c4[f]) + cA * kv[f];  // B = U + Y2 + dt k2
                outm[f] = u + cY * kv[f];                   // Y3
                a.y_dst[idx] = outm[f];
            } else {
                outm[f] = third_plus(a.acc_src[idx] + c4[f], cA * kv[f]);  // (B + Y4)/3 + dt/6 k4
                a.acc_dst[idx] = outm[f];
            }
        }
        // velocity-moment contributions (nuosc_class.cpp:69-71): moment 4c + j
        // = weight j (w, w vx, w vy, w vz) x combination c of the half
        const double w4[4] = {wd, vxd * wd, vyd * wd, vzd * wd};
        double d[3];
        if (half == 0) moment_terms<false>(outm[0], outm[1], outm[2], outm[3], d[0], d[1], d[2]);
        else moment_terms<true>(outm[0], outm[1], outm[2], outm[3], d[0], d[1], d[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int jw = 0; jw < 4; ++jw) mom[4 * c + jw] = w4[jw] * d[c];
    }
    // sum over the lanes of the (cell, half) (xor offsets below twp stay inside its group)
    for (int off = twp >> 1; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < NMOM; ++k) mom[k] += __shfl_xor_sync(0xffffffffu, mom[k], off);
    if (lane_in_cell == 0 && cell < g.ncell) {
        double *p = a.mom_part + ((cell * nvb + (nvb - 1)) * 2 + half) * NMOM;
#pragma unroll
        for (int k = 0; k < NMOM; ++k) p[k] = mom[k];
    }
}

constexpr int TAIL_BLOCK = 256;

// thread t: lane l = t % twp of (cell, half) = (t / twp) / 2, (t / twp) % 2
template <typename T, bool KO6, int MODE>
__global__ void __launch_bounds__(TAIL_BLOCK, 3) k_stage_tail(const StageArgs<T> a, int v0, int twp, int nvb) {
    const long long t = (long long)blockIdx.x * TAIL_BLOCK + threadIdx.x;
    const int l = (int)(t & (twp - 1));
    const long long ch = t / twp, cell = ch >> 1;
    const int v = v0 + l;
    tail_point<T, KO6, MODE>(a, cell, (int)(ch & 1), v, cell < a.g.ncell && v < a.g.nvs, twp, nvb, l);
}

// many instances' tails in one launch: item i covers threads [starts[i],
// starts[i] + 2 ncell_i twp_i), each range a multiple of 32 threads so that
// no warp spans two instances
template <typename T, bool KO6, int MODE>
__global__ void __launch_bounds__(TAIL_BLOCK, 2) k_stage_tail_batch(const TailItem<T> *__restrict__ items,
                                                                 const long long *__restrict__ starts, int n,
                                                                 long long total, const int *__restrict__ halt) {
    const long long t = (long long)blockIdx.x * TAIL_BLOCK + threadIdx.x;
    if (t - (threadIdx.x & 31) >= total) return;  // whole warps past the end
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const TailItem<T> &e = items[lo];
    if (halt && halt[e.member]) return;  // a stopped instance: no work (whole warps: one item per warp)
    const long long u = t - starts[lo];
    const int l = (int)(u & (e.twp - 1));
    const long long ch = u / e.twp, cell = ch >> 1;
    const int v = e.v0 + l;
    tail_point<T, KO6, MODE>(e.a, cell, (int)(ch & 1), v, cell < e.a.g.ncell && v < e.a.g.nvs, e.twp, e.nvb, l);
}

template <typename T, bool KO6>
cudaError_t launch_tail_ko(const StageArgs<T> &a, int mode, int v0, int twp, int nvb, cudaStream_t s) {
    const long long threads = a.g.ncell * 2 * twp;
    const unsigned blocks = (unsigned)((threads + TAIL_BLOCK - 1) / TAIL_BLOCK);
    switch (mode) {
    case MODE_S1Y: k_stage_tail<T, KO6, MODE_S1Y><<<blocks, TAIL_BLOCK, 0, s>>>(a, v0, twp, nvb); break;
    case MODE_S2B: k_stage_tail<T, KO6, MODE_S2B><<<blocks, TAIL_BLOCK, 0, s>>>(a, v0, twp, nvb); break;
    case MODE_SY: k_stage_tail<T, KO6, MODE_SY><<<blocks, TAIL_BLOCK, 0, s>>>(a, v0, twp, nvb); break;
    case MODE_S4B: k_stage_tail<T, KO6, MODE_S4B><<<blocks, TAIL_BLOCK, 0, s>>>(a, v0, twp, nvb); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, bool KO6>
cudaError_t launch_tail_batch_ko(const TailItem<T> *items, const long long *starts, int n, long long total,
                                 const int *halt, int mode, cudaStream_t s) {
    const unsigned blocks = (unsigned)((total + TAIL_BLOCK - 1) / TAIL_BLOCK);
    switch (mode) {
    case MODE_S1Y: k_stage_tail_batch<T, KO6, MODE_S1Y><<<blocks, TAIL_BLOCK, 0, s>>>(items, starts, n, total, halt); break;
    case MODE_S2B: k_stage_tail_batch<T, KO6, MODE_S2B><<<blocks, TAIL_BLOCK, 0, s>>>(items, starts, n, total, halt); break;
    case MODE_SY: k_stage_tail_batch<T, KO6, MODE_SY><<<blocks, TAIL_BLOCK, 0, s>>>(items, starts, n, total, halt); break;
    case MODE_S4B: k_stage_tail_batch<T, KO6, MODE_S4B><<<blocks, TAIL_BLOCK, 0, s>>>(items, starts, n, total, halt); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

int tail_lanes(int width) {
    int twp = 1;
    while (twp < width) twp *= 2;
    return twp;
}

template <typename T>
cudaError_t launch_stage_tail(const StageArgs<T> &a, int mode, bool ko6, int v0, int nvb, cudaStream_t s) {
    const int width = a.g.nvs - v0;
    if (width < 1 || width > 32 || !a.mom_part || nvb < 1) return cudaErrorInvalidValue;
    const int twp = tail_lanes(width);
    return ko6 ? launch_tail_ko<T, true>(a, mode, v0, twp, nvb, s) : launch_tail_ko<T, false>(a, mode, v0, twp, nvb, s);
}

template <typename T>
cudaError_t launch_stage_tail_batch(const TailItem<T> *items, const long long *starts, int n, long long total,
                                    const int *halt, int mode, bool ko6, cudaStream_t s) {
    if (n < 1 || total < 1) return cudaErrorInvalidValue;
    return ko6 ? launch_tail_batch_ko<T, true>(items, starts, n, total, halt, mode, s)
               : launch_tail_batch_ko<T, false>(items, starts, n, total, halt, mode, s);
}

template cudaError_t launch_stage_tail<double>(const StageArgs<double> &, int, bool, int, int, cudaStream_t);
template cudaError_t launch_stage_tail<float>(const StageArgs<float> &, int, bool, int, int, cudaStream_t);
template cudaError_t launch_stage_tail_batch<double>(const TailItem<double> *, const long long *, int, long long,
                                                     const int *, int, bool, cudaStream_t);
template cudaError_t launch_stage_tail_batch<float>(const TailItem<float> *, const long long *, int, long long,
                                                    const int *, int, bool, cudaStream_t);

}  // namespace nuosc
