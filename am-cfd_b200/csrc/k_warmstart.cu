// Solver side of the learned warm start (no counterpart in the reference).
//
// Features of a cell (FP32, channels last over the unpadded node grid,
// cell = (k*nj + j)*ni + i), at the start of a time step after the laser has
// moved:  T, u, v, w, p, f_l, the cell's offset from the beam centre in x and
// y, the beam power, and the previous step's scaled enthalpy and pressure
// increments.  Targets: the increments of enthalpy and pressure over the step.
// All are scaled to O(1) by fixed constants (WsScale).
//
// A prediction is applied as h += a dh (and p += a dp unless the enthalpy-only
// mode is chosen) on interior cells (a = 1,
// then 1/2), with T and f_l re-derived from h by convertEnthalpyToTemp
// (CFDSolverManager.cpp:2531-2571); the host keeps the first that lowers the
// energy residual of calculateResiduals(5) (:2073-2101) evaluated at the start
// of the step, and otherwise restores the snapshot taken before it.
#include "kernels.cuh"

namespace amcfd {

struct WsScale {
    double t0 = 300.0, t = 2000.0;  // T -> (T - t0) / t
    double vel = 1.0;               // m/s
    double pres = 1e4;              // Pa
    double pos = 0.0;               // beam-offset length (4 x beam radius), m
    double pow = 500.0;             // W
    double dh = 0.0;                // enthalpy increment scale: 0.1 hlcal
    double dp = 1e4;                // pressure increment scale, Pa
};

__device__ __forceinline__ bool ws_interior(const Params &p, int i, int j, int k)
{
    return i >= 1 && i <= p.nim2 && j >= 1 && j <= p.njm2 && k >= 1 && k <= p.nkm2;
}

template <typename T>
__global__ void ws_features_kernel(Params p, Fields<T> g, float *feat, const float *prev, WsScale s,
                                   double beamx, double beamy, double power)
{
    const long long n = (long long)p.ni * p.nj * p.nk;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % p.ni);
        const long long r = q / p.ni;
        const int j = (int)(r % p.nj), k = (int)(r / p.nj);
        const size_t c = cidx(i, j, k, p.nj, p.nip);
        float *f = feat + q * 11;
        f[0] = (float)(((double)g.temp[c] - s.t0) / s.t);
        f[1] = (float)((double)g.uvel[c] / s.vel);
        f[2] = (float)((double)g.vvel[c] / s.vel);
        f[3] = (float)((double)g.wvel[c] / s.vel);
        f[4] = (float)((double)g.pressure[c] / s.pres);
        f[5] = (float)g.fracl[c];
        f[6] = (float)fmin(fmax((g.x[i] - beamx) / s.pos, -8.0), 8.0);
        f[7] = (float)fmin(fmax((g.y[j] - beamy) / s.pos, -8.0), 8.0);
        f[8] = (float)(power / s.pow);
        f[9] = prev[q * 2];
        f[10] = prev[q * 2 + 1];
    }
}

// save[0..3] <- h, p, T, f_l (dir = 0) or back (dir = 1)
template <typename T>
__global__ void ws_copy_kernel(Params p, Fields<T> g, T *h0, T *p0, T *t0, T *f0, int dir)
{
    const size_t total = (size_t)p.nk * p.nj * p.nip;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (size_t)gridDim.x * blockDim.x) {
        if (dir == 0) {
            h0[c] = g.h[c]; p0[c] = g.pressure[c]; t0[c] = g.temp[c]; f0[c] = g.fracl[c];
        } else {
            g.h[c] = h0[c]; g.pressure[c] = p0[c]; g.temp[c] = t0[c]; g.fracl[c] = f0[c];
        }
    }
}

template <typename T>
__global__ void ws_apply_kernel(Params p, Fields<T> g, const float *y, WsScale s, double alpha, int with_p)
{
    const long long n = (long long)p.ni * p.nj * p.nk;
    const double deltemp = p.tliquid - p.tsolid;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % p.ni);
        const long long r = q / p.ni;
        const int j = (int)(r % p.nj), k = (int)(r / p.nj);
        if (!ws_interior(p, i, j, k)) continue;
        const size_t c = cidx(i, j, k, p.nj, p.nip);
        const double h = (double)g.h[c] + alpha * s.dh * (double)y[q * 2];
        g.h[c] = (T)h;
        if (with_p) g.pressure[c] = (T)((double)g.pressure[c] + alpha * s.dp * (double)y[q * 2 + 1]);
        // convertEnthalpyToTemp of the new enthalpy
        double fl, t;
        if (h >= p.hlcal) {
            fl = 1.0;
            t = (h - p.hlcal) / p.acpl + p.tliquid;
        } else if (h <= p.hsmelt) {
            fl = 0.0;
            t = (sqrt(p.acpb * p.acpb + 2 * p.acpa * h) - p.acpb) / p.acpa;
        } else {
            fl = (h - p.hsmelt) / (p.hlcal - p.hsmelt);
            t = deltemp * fl + p.tsolid;
        }
        g.fracl[c] = (T)fl;
        g.temp[c] = (T)t;
    }
}

// realised increments of the step, scaled: target[q] = ((h - h0)/dh, (p - p0)/dp)
template <typename T>
__global__ void ws_target_kernel(Params p, Fields<T> g, const T *h0, const T *p0, float *target, WsScale s)
{
    const long long n = (long long)p.ni * p.nj * p.nk;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % p.ni);
        const long long r = q / p.ni;
        const int j = (int)(r % p.nj), k = (int)(r / p.nj);
        const size_t c = cidx(i, j, k, p.nj, p.nip);
        target[q * 2] = (float)(((double)g.h[c] - (double)h0[c]) / s.dh);
        target[q * 2 + 1] = (float)(((double)g.pressure[c] - (double)p0[c]) / s.dp);
    }
}

static WsScale ws_scale(const Params &p)
{
    WsScale s;
    s.pos = 4.0 * p.alasrb;
    s.dh = 0.1 * p.hlcal;
    return s;
}

template <typename T> void ws_features(Inst<T> &I, float *feat, const float *prev, double bx, double by,
                                       double power)
{
    ws_features_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g, feat, prev, ws_scale(I.p), bx, by, power);
}
template <typename T> void ws_copy(Inst<T> &I, T *const *save, int dir)
{
    ws_copy_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g, save[0], save[1], save[2], save[3], dir);
}
template <typename T> void ws_apply(Inst<T> &I, const float *y, double alpha, int with_p)
{
    ws_apply_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g, y, ws_scale(I.p), alpha, with_p);
}
template <typename T> void ws_target(Inst<T> &I, T *const *save, float *target)
{
    ws_target_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g, save[0], save[1], target, ws_scale(I.p));
}

#define AMCFD_INST(T)                                                                  \
    template void ws_features<T>(Inst<T> &, float *, const float *, double, double, double); \
    template void ws_copy<T>(Inst<T> &, T *const *, int);                              \
    template void ws_apply<T>(Inst<T> &, const float *, double, int);                  \
    template void ws_target<T>(Inst<T> &, T *const *, float *);
AMCFD_INST(double)
AMCFD_INST(float)
#undef AMCFD_INST

}  // namespace amcfd
