// Energy-equation kernels of one SIMPLE outer iteration, plus the per-step
// laser and push-back kernels.  Each kernel names the reference routine it
// replaces; arithmetic follows the reference expression by expression so that
// the FP64 build matches the CPU solve to rounding.
#include "kernels.cuh"

namespace amcfd {

// ---------------------------------------------------------------------------
// updateLaser heat flux (BoundCondManager.cpp:128-159): Gaussian surface flux
// heatin[j][i] and the partial sums of areaij*heatin (heatinlaser).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void laser_kernel(Params p, Fields<T> g, double *red)
{
    pdl_enter();
    const Status *st = g.st;
    double acc = 0.0;
    const double rb2 = p.alasrb * p.alasrb;
    const double varlas = p.alaspow * p.alaseta;
    const double peakhin = p.alasfact * varlas / (M_PI * rb2);
    const double pw = (double)st->powerindicator;
    const int n = p.ni * p.nj;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        int j = q / p.ni, i = q - j * p.ni;
        double ydist = st->beamposy - g.y[j];
        double xdist = st->beamposx - g.x[i];
        double dist2 = (xdist * xdist) + (ydist * ydist);
        double hin = peakhin * exp(-p.alasfact * dist2 / rb2) * pw;
        if (p.alasfact < 1.0e-6 && dist2 < rb2) hin = varlas / (M_PI * rb2) * pw;
        g.heatin[(size_t)j * p.nip + i] = hin;
        acc += area_ij(p, g, i, j) * hin;
    }
    double v[1] = {acc};
    const int s[1] = {R_HEATIN};
    const bool m[1] = {false};
    block_reduce_store<1>(v, s, m, red, blockIdx.x);
}

// ---------------------------------------------------------------------------
// applyBCs(5) (BoundCondManager.cpp:565-654): top-surface flux balance and
// convective side planes.  Also advances the volumetric heat-source table the
// way calculateSource(5) does at the start of each outer iteration
// (CFDSolverManager.cpp:1707-1717).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void energy_bc_kernel(Params p, Fields<T> g, double *red)
{
    pdl_enter();
    Status *st = g.st;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (p.nheattable > 0) {
            int it = st->heat_iter;
            if (st->timet > g.heattable[6 * it] && it < p.nheattable - 1) it += 1;
            st->heat_iter = it;
            const double *row = &g.heattable[6 * it];
            st->avolpow = row[1];
            st->apowseta = row[2];
            st->heatthick = row[3];
            st->heatrb = row[4];
            st->avolfact = row[5];
        }
    }
    const int ni = p.ni, nj = p.nj, nip = p.nip;
    const int nim1 = p.nim1, njm1 = p.njm1, nkm1 = p.nkm1, nim2 = p.nim2, njm2 = p.njm2,
              nkm2 = p.nkm2;
    const int ntop = (nim1 - 1) * (njm1 - 1);
    const int new_ = (nkm1 - 1) * (njm1 - 1);
    const int nns = (nkm1 - 1) * (nim1 - 1);
    double ahtop = 0.0;
    double a4 = p.tempamb;
    for (int q = 1; q < 4; q++) a4 *= p.tempamb;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ntop + new_ + nns;
         q += gridDim.x * blockDim.x) {
        if (q < ntop) {
            int j = 1 + q / (nim1 - 1), i = 1 + q % (nim1 - 1);
            double t = (double)g.temp[cidx(i, j, nkm1, nj, nip)];
            double hlossevap = 0.0;
            if (p.isevap) {
                double psat = p.pressamb * exp(-p.evaplatent * p.molarmass / p.gasconst *
                                               (1.0 / t - 1.0 / p.evaptemp));
                double mdot = p.evapfact * psat * sqrt(p.molarmass / (2.0 * M_PI * p.gasconst * t));
                hlossevap = mdot * p.evaplatent;
            }
            double t4 = t;
            for (int r = 1; r < 4; r++) t4 *= t;
            double hlossradia = p.emiss * p.sigm * (t4 - a4);
            double ctmp1 = (double)g.diff_cur[cidx(i, j, nkm2, nj, nip)] * g.dzpbinv[nkm1];
            double hb = (double)g.h[cidx(i, j, nkm2, nj, nip)];
            g.h[cidx(i, j, nkm1, nj, nip)] =
                (T)(hb + (g.heatin[(size_t)j * nip + i] - hlossradia - hlossradia - hlossevap) / ctmp1);
            ahtop += (hlossradia + hlossradia + hlossevap) * area_ij(p, g, i, j);
        } else if (q < ntop + new_) {
            int r = q - ntop;
            int k = 1 + r / (njm1 - 1), j = 1 + r % (njm1 - 1);
            double hc = p.htci * ((double)g.temp[cidx(0, j, k, nj, nip)] - p.tempamb);
            double ctmp1 = (double)g.diff_cur[cidx(1, j, k, nj, nip)] * g.dxpwinv[1];
            g.h[cidx(0, j, k, nj, nip)] = (T)((double)g.h[cidx(1, j, k, nj, nip)] - hc / ctmp1);
            hc = p.htci * ((double)g.temp[cidx(nim1, j, k, nj, nip)] - p.tempamb);
            ctmp1 = (double)g.diff_cur[cidx(nim2, j, k, nj, nip)] * g.dxpwinv[nim2];
            g.h[cidx(nim1, j, k, nj, nip)] = (T)((double)g.h[cidx(nim2, j, k, nj, nip)] - hc / ctmp1);
        } else {
            int r = q - ntop - new_;
            int k = 1 + r / (nim1 - 1), i = 1 + r % (nim1 - 1);
            double hc = p.htcj * ((double)g.temp[cidx(i, 0, k, nj, nip)] - p.tempamb);
            double ctmp1 = (double)g.diff_cur[cidx(i, 1, k, nj, nip)] * g.dypsinv[1];
            g.h[cidx(i, 0, k, nj, nip)] = (T)((double)g.h[cidx(i, 1, k, nj, nip)] - hc / ctmp1);
            hc = p.htcj * ((double)g.temp[cidx(i, njm1, k, nj, nip)] - p.tempamb);
            ctmp1 = (double)g.diff_cur[cidx(i, njm2, k, nj, nip)] * g.dypsinv[njm2];
            g.h[cidx(i, njm1, k, nj, nip)] = (T)((double)g.h[cidx(i, njm2, k, nj, nip)] - hc / ctmp1);
        }
    }
    (void)ni;
    double v[1] = {ahtop};
    const int s[1] = {R_AHTOP};
    const bool m[1] = {false};
    block_reduce_store<1>(v, s, m, red, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Block correction solve (enhanceConvergenceSpeed(5), CFDSolverManager.cpp:2334-2349)
// and the energy residual resorh (:2099).  One CTA.
// ---------------------------------------------------------------------------
// Per-i sums of the block-correction partial rows in a fixed order: CTA (32 i x
// 8 part-strides) per i-chunk and quantity.
template <typename T>
__global__ void __launch_bounds__(256) bc_reduce_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    __shared__ double sh[8][33];
    const int i = blockIdx.x * 32 + threadIdx.x, w = blockIdx.y, nip = p.nip;
    double s = 0.0;
    for (int part = threadIdx.y; part < g.npart; part += 8)
        s += g.bc[((size_t)part * 4 + w) * nip + i];
    sh[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0) {
        double t = 0.0;
        for (int y = 0; y < 8; ++y) t += sh[y][threadIdx.x];
        g.bcsum[(size_t)w * nip + i] = t;
    }
}

// 1-D TDMA of the block correction (enhanceConvergenceSpeed(5),
// CFDSolverManager.cpp:2334-2349) for cells i0..i1 by one warp:
//   den_i = bl_i - blm_i pib_{i-1},  pib_i = blp_i / den_i,
//   qib_i = (blc_i + blm_i qib_{i-1}) / den_i,  delphi_i = pib_i delphi_{i+1} + qib_i,
// with pib_{i0-1} = qib_{i0-1} = 0 and delphi_{i1+1} = 0.  Each lane owns a
// contiguous chunk.  pib follows x -> blp / (bl - blm x), a Moebius map: the
// chunks' 2x2 matrices (rescaled as they are multiplied; the map ignores
// scale) are combined by a warp scan to give each chunk its entry value, and
// the chunk then runs the reference recurrence.  qib and delphi are affine in
// their predecessor and use warp scans of affine maps.  All in FP64.  On
// return bl holds den, blm holds pib and blp holds qib.
__device__ __forceinline__ double moebius_scale(double a, double b, double c, double d)
{
    const double mx = fmax(fmax(fabs(a), fabs(b)), fmax(fabs(c), fabs(d)));
    return mx > 0.0 ? 1.0 / mx : 1.0;
}

__device__ void block_tdma_warp(double *bl, double *blp, double *blm, const double *blc, int i0, int i1,
                                double *delphi)
{
    const int lane = threadIdx.x & 31;
    const int n = i1 - i0 + 1;
    if (n <= 0) return;
    const int L = (n + 31) >> 5;
    const int a = i0 + min(lane * L, n), e = i0 + min(lane * L + L, n);
    // chunk product of the Moebius matrices [[0, blp], [-blm, bl]] (later cells on the left)
    double m00 = 1.0, m01 = 0.0, m10 = 0.0, m11 = 1.0;
    for (int i = a; i < e; ++i) {
        const double n00 = blp[i] * m10, n01 = blp[i] * m11;
        const double n10 = -blm[i] * m00 + bl[i] * m10, n11 = -blm[i] * m01 + bl[i] * m11;
        const double sc = moebius_scale(n00, n01, n10, n11);
        m00 = n00 * sc; m01 = n01 * sc; m10 = n10 * sc; m11 = n11 * sc;
    }
    // inclusive scan: M_lane <- M_lane * M_{lane-o}
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double p00 = __shfl_up_sync(0xffffffffu, m00, o), p01 = __shfl_up_sync(0xffffffffu, m01, o);
        const double p10 = __shfl_up_sync(0xffffffffu, m10, o), p11 = __shfl_up_sync(0xffffffffu, m11, o);
        if (lane >= o) {
            const double n00 = m00 * p00 + m01 * p10, n01 = m00 * p01 + m01 * p11;
            const double n10 = m10 * p00 + m11 * p10, n11 = m10 * p01 + m11 * p11;
            const double sc = moebius_scale(n00, n01, n10, n11);
            m00 = n00 * sc; m01 = n01 * sc; m10 = n10 * sc; m11 = n11 * sc;
        }
    }
    // entry value pib_{a-1}: the exclusive prefix applied to x = 0
    double e01 = __shfl_up_sync(0xffffffffu, m01, 1), e11 = __shfl_up_sync(0xffffffffu, m11, 1);
    double pib = (lane == 0) ? 0.0 : e01 / e11;
    // the chunk runs the reference recurrence for den and pib; qib's affine maps
    double A = 1.0, B = 0.0;
    for (int i = a; i < e; ++i) {
        const double den = bl[i] - blm[i] * pib;
        const double pv = blp[i] / den;
        const double ca = blm[i] / den, cb = blc[i] / den;  // qib_i = ca qib_{i-1} + cb
        bl[i] = den;
        blm[i] = pv;
        blp[i] = cb;  // temporarily the affine offset
        pib = pv;
        B = ca * B + cb;
        A = ca * A;
        delphi[i] = ca;  // temporarily the affine slope
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double A2 = __shfl_up_sync(0xffffffffu, A, o), B2 = __shfl_up_sync(0xffffffffu, B, o);
        if (lane >= o) { B = A * B2 + B; A = A * A2; }
    }
    double Be = __shfl_up_sync(0xffffffffu, B, 1);
    double q = (lane == 0) ? 0.0 : Be;  // qib_{a-1} (qib_{i0-1} = 0)
    for (int i = a; i < e; ++i) {
        q = delphi[i] * q + blp[i];
        blp[i] = q;
    }
    // back substitution delphi_i = pib_i delphi_{i+1} + qib_i, delphi_{i1+1} = 0
    A = 1.0;
    B = 0.0;
    for (int i = e - 1; i >= a; --i) {
        B = blm[i] * B + blp[i];
        A = blm[i] * A;
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double A2 = __shfl_down_sync(0xffffffffu, A, o), B2 = __shfl_down_sync(0xffffffffu, B, o);
        if (lane + o < 32) { B = A * B2 + B; A = A * A2; }
    }
    Be = __shfl_down_sync(0xffffffffu, B, 1);
    double d = (lane == 31) ? 0.0 : Be;
    for (int i = e - 1; i >= a; --i) {
        d = blm[i] * d + blp[i];
        delphi[i] = d;
    }
}

template <typename T>
__global__ void block_correct_kernel(Params p, Fields<T> gd, double *red_asm, int nblk_asm,
                                     int check_finite, int ivar)
{
    pdl_enter();
    extern __shared__ double sm[];  // 4 * nip
    const int nip = p.nip, nim2 = p.nim2;
    double *bl = sm, *blp = sm + nip, *blm = sm + 2 * nip, *blc = sm + 3 * nip;
    for (int q = threadIdx.x; q < 4 * nip; q += blockDim.x) sm[q] = gd.bcsum[q];
    double sd = 0.0, sh = 0.0;
    for (int b = threadIdx.x; b < nblk_asm; b += blockDim.x) {
        sd += red_asm[(size_t)b * R_NSLOTS + R_SUMD];
        sh += red_asm[(size_t)b * R_NSLOTS + R_SUMH];
    }
    __syncthreads();
    double v[2] = {sd, sh};
    const int sl[2] = {0, 1};
    const bool mx[2] = {false, false};
    __shared__ double tot[R_NSLOTS];
    block_reduce_store<2>(v, sl, mx, tot, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
        Status *st = gd.st;
        // resorh (calculateResiduals(5)) or resorc (calculateResiduals(6))
        double res = tot[0] / (tot[1] + kSmall);
        if (ivar == 6) st->resorc = res; else st->resorh = res;
        if (check_finite && !isfinite(res)) st->nonfinite = 1;
    }
    if (threadIdx.x < 32) block_tdma_warp(bl, blp, blm, blc, 1, nim2, gd.delphi);
}
// ---------------------------------------------------------------------------
// convertEnthalpyToTemp (CFDSolverManager.cpp:2531-2571), fused with the
// peak-temperature maximum (BoundCondManager.cpp:301) and the reductions of
// calculateFluxes (BoundCondManager.cpp:778-843): boundary conduction fluxes,
// heat accumulation and volumetric heat input.  H->T is evaluated in FP64.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 4) h2t_kernel(Params p, Fields<T> g, double *red)
{
    pdl_enter();
    const Status *st = g.st;
    const int ni = p.ni, nj = p.nj, nk = p.nk, nip = p.nip;
    const int nim1 = p.nim1, njm1 = p.njm1, nkm1 = p.nkm1, nim2 = p.nim2, njm2 = p.njm2,
              nkm2 = p.nkm2;
    const double deltemp = p.tliquid - p.tsolid;
    const double delt = st->delt;
    // The FP64 build divides exactly as the reference; the FP32 build keeps the
    // inversion in FP64 but multiplies by reciprocals formed once per launch.
    constexpr bool kExact = sizeof(T) == sizeof(double);
    const double inv_acpl = 1.0 / p.acpl, inv_acpa = 1.0 / p.acpa,
                 inv_mush = 1.0 / (p.hlcal - p.hsmelt), inv_delt = 1.0 / delt;
    double tmax = -INFINITY, accul = 0.0, heatvol = 0.0;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const int js = st->jstart, is0 = st->istart;
    const double ts = p.tsolid;
    const bool steady = p.steady != 0;
    const bool volsrc = p.volsrc != 0;
    const int lane = threadIdx.x & 31;
    // Work unit: a chunk of 32 V cells of one x-line, V = 16 bytes per element;
    // lane l holds the 16-byte vector of cells base = chunk start + V l (the pitch
    // nip is a multiple of 32, so a vector lies wholly inside or wholly past the
    // padded row).  Chunk indices are 32-bit (the chunk count is bounded at
    // context creation): a 64-bit division per chunk costs more than the
    // chunk's enthalpy inversions.
    constexpr int V = 16 / (int)sizeof(T);
    constexpr int RC = 32 * V;
    const unsigned cpr = ((unsigned)nip + RC - 1) / RC;  // chunks per row
    const unsigned unj = (unsigned)nj;
    const unsigned nchunks = (unsigned)nk * unj * cpr;
    const unsigned W = gridDim.x * (blockDim.x >> 5);
    const unsigned w0 = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const double *dxw = g.dxpwinv, *dys = g.dypsinv, *dzb = g.dzpbinv;
    for (unsigned q = w0; q < nchunks; q += W) {
        const unsigned r = q / cpr;
        const int base = (int)(q - r * cpr) * RC + V * lane;
        const int k = (int)(r / unj), j = (int)(r - (unsigned)k * unj);
        const bool inrow = base < nip;
        const size_t c0 = (size_t)r * nip + (inrow ? base : 0);
        T hv[V], hn[V], fln[V], rn[V], sv[V];
        ld16(g.h + c0, hv); ld16(g.hnot + c0, hn); ld16(g.fraclnot + c0, fln);
        ld16(g.rho_nxt + c0, rn);
        // the volumetric source input is zero everywhere without a volumetric source
        if (volsrc) ld16(g.sourceinput + c0, sv);
        const bool rowint = !steady && j >= 1 && j <= njm2 && k >= 1 && k <= nkm2;
        T tout[V], fout[V];
        int cmaxl = INT_MAX, cminl = INT_MIN;  // beam-row length candidates of this lane
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int i = base + v;
            tout[v] = fout[v] = T(0);
            if (!inrow || i >= ni) continue;
            const double h = (double)hv[v];
            double fl, t;
            if (h >= p.hlcal) {
                fl = 1.0;
                t = (kExact ? (h - p.hlcal) / p.acpl : (h - p.hlcal) * inv_acpl) + p.tliquid;
            } else if (h <= p.hsmelt) {
                fl = 0.0;
                const double root = sqrt(p.acpb * p.acpb + 2 * p.acpa * h) - p.acpb;
                t = kExact ? root / p.acpa : root * inv_acpa;
            } else {
                fl = kExact ? (h - p.hsmelt) / (p.hlcal - p.hsmelt) : (h - p.hsmelt) * inv_mush;
                t = deltemp * fl + p.tsolid;
            }
            fout[v] = (T)fl;
            tout[v] = (T)t;
            const double tt = (double)(T)t;
            if (tt > tmax) tmax = tt;
            // melt-pool scan candidates (BoundCondManager.cpp:318-417).  Most cells
            // are solid, so each atomic is issued only when it can still change the
            // value (candidates only move one way); the beam-row scalars are
            // warp-reduced below.
            if (j == js && k >= 1 && k <= nkm2 && tt < ts && k > *(volatile int *)&g.mp_kb[i])
                atomicMax(&g.mp_kb[i], k);
            if (k == nkm1) {
                if (j >= js && j <= njm2 && tt < ts && j < *(volatile int *)&g.mp_jup[i])
                    atomicMin(&g.mp_jup[i], j);
                if (j >= 1 && j <= js && tt < ts && j > *(volatile int *)&g.mp_jdn[i])
                    atomicMax(&g.mp_jdn[i], j);
                if (j == js) {
                    if (i >= is0 && i < nim1 && tt <= ts) cmaxl = min(cmaxl, i);
                    if (i >= 1 && i <= is0 && tt < ts) cminl = max(cminl, i);
                }
            }
            if (!rowint || i < 1 || i > nim2) continue;
            const double dh1 = h - (double)hn[v] + ((double)(T)fl - (double)fln[v]) * p.hlatnt;
            const double vol = volume_p(p, g, i, j, k);
            accul += kExact ? vol * (double)rn[v] * dh1 / delt : vol * (double)rn[v] * dh1 * inv_delt;
            if (volsrc) heatvol += (double)sv[v] * vol;
        }
        if (inrow) {
            if (base + V <= ni) {
                typename Vec16<T>::type w;
                memcpy(&w, tout, 16);
                *reinterpret_cast<typename Vec16<T>::type *>(g.temp + c0) = w;
                memcpy(&w, fout, 16);
                *reinterpret_cast<typename Vec16<T>::type *>(g.fracl + c0) = w;
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (base + v < ni) {
                        g.temp[c0 + v] = tout[v];
                        g.fracl[c0 + v] = fout[v];
                    }
            }
        }
        if (k == nkm1 && j == js) {  // chunk-uniform: every lane takes part
            const int wmin = __reduce_min_sync(0xffffffffu, cmaxl);
            const int wmax = __reduce_max_sync(0xffffffffu, cminl);
            if (lane == 0) {
                if (wmin != INT_MAX) atomicMin(&g.st->mp_imax, wmin);
                if (wmax != INT_MIN) atomicMax(&g.st->mp_imin, wmax);
            }
        }
    }
    // Boundary conduction fluxes (BoundCondManager.cpp:778-843): a second pass
    // over the six interior boundary layers only, so that the bulk loop above
    // carries no flux accumulators.  Face f's layer is a 2-D index set.
    double fw = 0.0, fe = 0.0, fb = 0.0, ft = 0.0, fs = 0.0, fn = 0.0;
    {
        const int I = nim2, J = njm2, K = nkm2;  // interior extents
        const long long nx = (long long)J * K, ny = (long long)I * K, nz = (long long)I * J;
        const long long nall = 2 * (nx + ny + nz);
        const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const long long nthr = (long long)gridDim.x * blockDim.x;
        for (long long q = tid; q < nall; q += nthr) {
            long long r = q;
            int face, a, b;  // face 0..5 = W E B T S N
            if (r < 2 * nx) { face = (int)(r / nx); r %= nx; a = (int)(r % J); b = (int)(r / J); }
            else if ((r -= 2 * nx) < 2 * nz) { face = 2 + (int)(r / nz); r %= nz; a = (int)(r % I); b = (int)(r / I); }
            else { r -= 2 * nz; face = 4 + (int)(r / ny); r %= ny; a = (int)(r % I); b = (int)(r / I); }
            int i, j, k;
            if (face < 2) { i = face == 0 ? 1 : nim2; j = 1 + a; k = 1 + b; }
            else if (face < 4) { k = face == 2 ? 1 : nkm2; i = 1 + a; j = 1 + b; }
            else { j = face == 4 ? 1 : njm2; i = 1 + a; k = 1 + b; }
            const size_t c = cidx(i, j, k, nj, nip);
            const double h = (double)g.h[c];
            const double dn = (double)g.diff_nxt[c];
            switch (face) {
            case 0: fw += area_jk(p, g, j, k) * (dn * ((double)g.h[c - 1] - h) * dxw[1]); break;
            case 1: fe += area_jk(p, g, j, k) * (dn * ((double)g.h[c + 1] - h) * dxw[nim1]); break;
            case 2: fb += area_ij(p, g, i, j) * (dn * ((double)g.h[c - sk] - h) * dzb[1]); break;
            case 3: ft += area_ij(p, g, i, j) * (dn * ((double)g.h[c + sk] - h) * dzb[nkm1]); break;
            case 4: fs += area_ik(p, g, i, k) * (dn * ((double)g.h[c - sj] - h) * dys[1]); break;
            default: fn += area_ik(p, g, i, k) * (dn * ((double)g.h[c + sj] - h) * dys[njm1]); break;
            }
        }
    }
    double v[8] = {tmax, accul, heatvol, fw, fe, fb, ft, fs};
    const int s[8] = {R_TPEAK, R_ACCUL, R_HEATVOL, R_FW, R_FE, R_FB, R_FT, R_FS};
    const bool m[8] = {true, false, false, false, false, false, false, false};
    block_reduce_store<8>(v, s, m, red, blockIdx.x);
    __syncthreads();
    double v2[1] = {fn};
    const int s2[1] = {R_FN};
    const bool m2[1] = {false};
    block_reduce_store<1>(v2, s2, m2, red, blockIdx.x);
}

// Fixed-order block reduction of one slot over `nb` per-CTA partials.
__device__ double reduce_slot(const double *red, int nb, int slot, bool is_max, double *scratch)
{
    double acc = is_max ? -INFINITY : 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        double x = red[(size_t)b * R_NSLOTS + slot];
        acc = is_max ? fmax(acc, x) : acc + x;
    }
    acc = is_max ? warp_max(acc) : warp_sum(acc);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = acc;
    __syncthreads();
    double r = is_max ? -INFINITY : 0.0;
    if (warp == 0) {
        r = (lane < (int)(blockDim.x >> 5)) ? scratch[lane] : (is_max ? -INFINITY : 0.0);
        r = is_max ? warp_max(r) : warp_sum(r);
        if (lane == 0) scratch[32] = r;
    }
    __syncthreads();
    r = scratch[32];
    __syncthreads();
    return r;
}

// Sentinels of the melt-pool scan candidates for the next outer iteration.
template <typename T>
__device__ void reset_scan_candidates(const Params &p, Fields<T> &g)
{
    for (int i = threadIdx.x; i < p.nip; i += blockDim.x) {
        g.mp_kb[i] = 0;
        g.mp_jup[i] = p.njm1;
        g.mp_jdn[i] = 0;
    }
    if (threadIdx.x == 0) {
        g.st->mp_imax = INT_MAX;
        g.st->mp_imin = INT_MIN;
    }
}

// ---------------------------------------------------------------------------
// getMeltPoolShape (BoundCondManager.cpp:280-447), one CTA.  The scans along
// i/j/k are evaluated per column in parallel; the folds whose result depends on
// order (the NaN behaviour of std::max/min) run sequentially in thread 0.
// Also activates the momentum box and builds its exact-order ticket list.
// ---------------------------------------------------------------------------
// acc = f(x_i, acc) in ascending i over the flagged i of [lo, hi), from init,
// with f = std::max or std::min as the reference folds (maxd/mind): a NaN element
// makes acc NaN and the next element replaces it.  The fold therefore equals the
// extreme of the flagged elements after the last NaN, NaN when that NaN is the
// last flagged element, and includes init only when no NaN occurs -- which a
// block can compute in two passes.  Every thread of the block calls it.
__device__ double ordered_fold(const double *x, const int *fl, int bit, int lo, int hi, double init,
                               bool is_max, int *si, double *sd)
{
    const int tid = threadIdx.x, nth = blockDim.x;
    if (tid == 0) { si[0] = -1; si[1] = -1; }
    __syncthreads();
    int lastf = -1, lastn = -1;  // per thread, indices ascend
    for (int i = lo + tid; i < hi; i += nth)
        if (fl[i] & bit) {
            lastf = i;
            if (isnan(x[i])) lastn = i;
        }
    if (lastf >= 0) atomicMax(&si[0], lastf);
    if (lastn >= 0) atomicMax(&si[1], lastn);
    __syncthreads();
    const int L = si[0], P = si[1];
    double v = is_max ? -INFINITY : INFINITY;
    for (int i = max(lo, P + 1) + tid; i < hi; i += nth)
        if (fl[i] & bit) v = is_max ? fmax(v, x[i]) : fmin(v, x[i]);
    v = is_max ? warp_max(v) : -warp_max(-v);
    if ((tid & 31) == 0) sd[tid >> 5] = v;
    __syncthreads();
    double r = is_max ? -INFINITY : INFINITY;
    for (int w = 0; w < (nth + 31) / 32; ++w) r = is_max ? fmax(r, sd[w]) : fmin(r, sd[w]);
    __syncthreads();
    if (L < 0) return init;
    if (P >= 0) return P == L ? (double)NAN : r;
    return is_max ? ((r < init) ? init : r) : ((init < r) ? init : r);
}

template <typename T>
__global__ void __launch_bounds__(1024) meltpool_kernel(Params p, Fields<T> g, const double *red_h2t,
                                                        int nblk_h2t)
{
    pdl_enter();
    Status *st = g.st;
    __shared__ double scratch[40];
    extern __shared__ double colv[];  // 3 * nip doubles + nip ints
    const int nj = p.nj, nip = p.nip;
    const int nim1 = p.nim1, nkm1 = p.nkm1, nim2 = p.nim2, njm2 = p.njm2, nkm2 = p.nkm2;
    const double ts = p.tsolid;
    double tp = reduce_slot(red_h2t, nblk_h2t, R_TPEAK, true, scratch);
    double t0 = (double)g.temp[0];
    if (isnan(t0)) tp = t0;  // std::max_element keeps a leading NaN
    if (threadIdx.x == 0) st->tpeak = tp;
    if (!(tp > ts)) {
        if (threadIdx.x == 0) {
            st->alen = 0.0;
            st->depth = 0.0;
            st->width = 0.0;
            st->momentum_active = 0;
        }
        reset_scan_candidates(p, g);
        return;
    }
    const int js = st->jstart, is0 = st->istart;
    // Reads outside the node range (the reference reads past its arrays when the
    // pool touches the north/south boundary rows) return NaN instead.
    auto TT = [&](int i, int j, int k) {
        if (i < 0 || i >= p.ni || j < 0 || j >= nj || k < 0 || k >= p.nk) return (double)NAN;
        return (double)g.temp[cidx(i, j, k, nj, nip)];
    };
    auto YY = [&](int j) { return (j < 0 || j >= nj) ? (double)NAN : g.y[j]; };
    double *depv = colv, *wmax = colv + nip, *wmin = colv + 2 * nip;
    int *imaxc = (int *)(colv + 3 * nip);
    // length: first i >= istart on the top row with T <= Ts; last i <= istart with T < Ts
    // (candidates gathered by h2t_kernel with integer atomics, read and reset here)
    // depth: per column i, mp_kb = the largest k in 1..nkm2 with T < Ts on the beam
    // plane (0 if none) -- the scan from nkm2 down visits nkm2..mp_kb+1.
    // width: mp_jup = first j >= jstart with T < Ts (njm1 if none), mp_jdn = first
    // j <= jstart going down with T < Ts (0 if none).
    int kmin_c = INT_MAX, jmax_c = INT_MIN, jmin_c = INT_MAX;
    for (int i = 1 + (int)threadIdx.x; i < nim1; i += blockDim.x) {
        const int kb = g.mp_kb[i], ju = g.mp_jup[i], jd = g.mp_jdn[i];
        if (kb < nkm2) kmin_c = min(kmin_c, kb + 1);
        if (ju > js) jmax_c = max(jmax_c, ju - 1);
        if (jd < js) jmin_c = min(jmin_c, jd + 1);
    }
    // block min/max of the integer candidates
    __shared__ int red_i[6];
    if (threadIdx.x == 0) {
        red_i[0] = st->mp_imax; red_i[1] = st->mp_imin; red_i[2] = INT_MAX; red_i[3] = INT_MIN;
        red_i[4] = INT_MAX;
    }
    __syncthreads();
    atomicMin(&red_i[2], kmin_c);
    atomicMax(&red_i[3], jmax_c);
    atomicMin(&red_i[4], jmin_c);
    __syncthreads();
    int imax = (is0 < nim1) ? (red_i[0] == INT_MAX ? nim1 - 1 : red_i[0]) : is0;
    int imin = (is0 > 0) ? (red_i[1] == INT_MIN ? 1 : red_i[1]) : is0;
    int kmin = min(nkm2, red_i[2]) - 1;
    int jmax = max(js, red_i[3]) + 1;
    int jmin = min(js, red_i[4]) - 1;
    // per-column interpolated values for the order-dependent folds
    // imaxc[i] bits: 1 = column enters the depth fold, 2 = the max-width fold,
    // 4 = the min-width fold (the reference's `continue` tests), so that the
    // sequential folds below read shared memory only.
    for (int i = 1 + (int)threadIdx.x; i < nim1; i += blockDim.x) {
        int fl = 0;
        if (kmin != 0 && !(TT(i, js, kmin + 1) < ts)) {
            fl |= 1;
            double dtdzzinv = (g.z[kmin] - g.z[kmin - 1]) / (TT(i, js, kmin) - TT(i, js, kmin - 1));
            depv[i] = g.z[nkm1] - g.z[kmin] + (TT(i, js, kmin) - ts) * dtdzzinv;
        }
        if (jmax != js && !(TT(i, jmax - 1, nkm1) < ts)) {
            fl |= 2;
            double dtdyyinv = (YY(jmax) - YY(jmax + 1)) / (TT(i, jmax, nkm1) - TT(i, jmax + 1, nkm1));
            wmax[i] = YY(jmax) + (ts - TT(i, jmax, nkm1)) * dtdyyinv;
        }
        if (jmin != js && !(TT(i, jmin + 1, nkm1) < ts)) {
            fl |= 4;
            double dtdyyinv = (YY(jmin) - YY(jmin - 1)) / (TT(i, jmin, nkm1) - TT(i, jmin - 1, nkm1));
            wmin[i] = YY(jmin) + (ts - TT(i, jmin, nkm1)) * dtdyyinv;
        }
        imaxc[i] = fl;
    }
    __syncthreads();
    // the reference's three folds over the columns (BoundCondManager.cpp:360-417),
    // in parallel with the same NaN behaviour
    __shared__ int fsi[2];
    __shared__ double fsd[32];
    const double depth_f = ordered_fold(depv, imaxc, 1, 1, nim1, 0.0, true, fsi, fsd);
    const double ymax_f = ordered_fold(wmax, imaxc, 2, 1, nim1, g.y[0], true, fsi, fsd);
    const double ymin_f = ordered_fold(wmin, imaxc, 4, 1, nim1, YY(js), false, fsi, fsd);
    if (threadIdx.x == 0) {
        auto XX = [&](int i) { return (i < 0 || i >= p.ni) ? (double)NAN : g.x[i]; };
        double dtdxxinv = (XX(imax) - XX(imax + 1)) / (TT(imax, js, nkm1) - TT(imax + 1, js, nkm1));
        double xxmax = XX(imax) + (ts - TT(imax, js, nkm1)) * dtdxxinv;
        dtdxxinv = (XX(imin) - XX(imin - 1)) / (TT(imin, js, nkm1) - TT(imin - 1, js, nkm1));
        double xxmin = XX(imin) + (ts - TT(imin, js, nkm1)) * dtdxxinv;
        st->alen = xxmax - xxmin;
        st->depth = kmin == 0 ? g.z[nkm1] - g.z[0] : depth_f;
        const double yymax = jmax != js ? ymax_f : g.y[0];
        const double yymin = jmin != js ? ymin_f : YY(js);
        st->width = yymax - yymin;
        st->imax = imax; st->imin = imin; st->kmin = kmin; st->kmax = nkm2;
        st->jmax = jmax; st->jmin = jmin;
        st->istat = max(imin - 3, 1);
        st->iend = min(imax + 3, nim2);
        st->jstat = max(jmin - 3, 1);
        st->jend = min(jmax + 2, njm2);
        st->kstat = max(kmin - 2, 2);
        st->istatp1 = st->istat + 1;
        st->iendm1 = st->iend - 1;
        st->momentum_active = p.navierstokes ? 1 : 0;
        st->box_cells = st->momentum_active
            ? max(0, st->iendm1 - st->istatp1 + 1) * max(0, st->jend - st->jstat + 1) * max(0, nkm1 - st->kstat)
            : 0;
    }
    reset_scan_candidates(p, g);  // every reader passed the __syncthreads above
}

// ---------------------------------------------------------------------------
// End of an outer iteration: calculateFluxes ratio (BoundCondManager.cpp:846-857),
// amaxres and the convergence test (CFDSolverManager.cpp:689-716).  One CTA.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void converge_kernel(Params p, Fields<T> gd, const double *red_h2t, int nb_h2t,
                                const double *red_bc, int nb_bc, const double *red_las, int nb_las,
                                const double *red_mom, int nb_mom, double tol, int check_finite,
                                LoopCtl lc)
{
    pdl_enter();
    __shared__ double scratch[40];
    __shared__ double scr8[8 * 33];
    Status *st = gd.st;
    const double *hb[8] = {red_h2t, red_h2t, red_h2t, red_h2t, red_h2t, red_h2t, red_h2t, red_h2t};
    const int hs[8] = {R_ACCUL, R_HEATVOL, R_FW, R_FE, R_FB, R_FT, R_FS, R_FN};
    double hv[8];
    reduce_sums<8>(hb, hs, nb_h2t, hv, scr8);
    const double accul = hv[0], heatvol = hv[1], fw = hv[2], fe = hv[3], fb = hv[4], ft = hv[5],
                 fs = hv[6], fn = hv[7];
    double ahtop = reduce_slot(red_bc, nb_bc, R_AHTOP, false, scratch);
    double heatin = reduce_slot(red_las, nb_las, R_HEATIN, false, scratch);
    if (threadIdx.x == 0) {
        st->accul = p.steady ? 0.0 : accul;
        st->heatvol = p.steady ? 0.0 : heatvol;
        st->fluxwest = fw; st->fluxeast = fe; st->fluxbottom = fb; st->fluxtop = ft;
        st->fluxsouth = fs; st->fluxnorth = fn;
        st->ahtoploss = ahtop;
        st->heatinlaser = heatin;
        st->heatout = (fn + fb + fw + fe + fs) - ahtop;
        double ratio = p.steady ? -st->heatout / heatin : (st->heatvol + heatin) / (st->accul - st->heatout);
        st->ratio = ratio;
        double list[5] = {st->resorm, st->resoru, st->resorv, st->resorw, st->resorc};
        double amaxres = list[0];
        for (int q = 1; q < 5; q++)
            if (amaxres < list[q]) amaxres = list[q];
        int conv;
        if (p.steady)
            conv = (ratio <= 1.001 && ratio >= 0.999 && amaxres < tol);
        else if (st->powerindicator == 1)
            conv = (ratio <= 1.01 && ratio >= 0.99 && amaxres < tol);
        else
            conv = (st->resorh < 1e-6 && amaxres < tol);
        st->converged = conv;
        if (check_finite && (!isfinite(st->tpeak) || !isfinite(ratio) || !isfinite(st->resorh)))
            st->nonfinite = 1;
        if (lc.active) {
            // the host loop's bookkeeping: count the iteration, remember its box, and
            // continue unless converged, failed or out of iterations
            const int it = st->lp_niter + 1;
            st->lp_niter = it;
            st->lp_small += st->lp_mode;
            const int box = st->momentum_active ? st->box_cells : 0;
            st->lp_box = box;
            const int mode = lc.cap >= 0 && box <= lc.cap;
            st->lp_mode = mode;
            const int cont = !conv && !st->nonfinite && !*(volatile int *)&st->error && it < lc.maxit;
            if (lc.has_next) {
                cudaGraphSetConditional(lc.mode_next, (unsigned)mode);
                cudaGraphSetConditional(lc.cont, (unsigned)cont);
            }
        }
    }
    (void)red_mom; (void)nb_mom;
}

// Head of a step captured as one graph: the momentum path of its first outer
// iteration, from the box of the last iteration before it.
__global__ void loop_init_kernel(Status *st, LoopCtl lc)
{
    const int mode = lc.cap >= 0 && st->lp_box >= 0 && st->lp_box <= lc.cap;
    st->lp_mode = mode;
    cudaGraphSetConditional(lc.mode_next, (unsigned)mode);
}
void launch_loop_init(Status *st, const LoopCtl &lc, cudaStream_t s)
{
    loop_init_kernel<<<1, 1, 0, s>>>(st, lc);
}

// ---------------------------------------------------------------------------
// updateSolutions (CFDSolverManager.cpp:2625-2687): solid velocities to zero and
// the previous-step copies.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void update_solutions_kernel(Params p, Fields<T> g, double trackindx, int trackid)
{
    pdl_enter();
    const size_t total = (size_t)p.nk * p.nj * p.nip;
    const T ts = (T)p.tsolid;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (size_t)gridDim.x * blockDim.x) {
        if (g.temp[c] <= ts) {
            g.uvel[c] = T(0);
            g.vvel[c] = T(0);
            g.wvel[c] = T(0);
        }
        g.unot[c] = g.uvel[c];
        g.vnot[c] = g.vvel[c];
        g.wnot[c] = g.wvel[c];
        g.hnot[c] = g.h[c];
        g.fraclnot[c] = g.fracl[c];
        if (p.powder) {  // CFDSolverManager.cpp:2666-2678
            const T fl = g.fracl[c];
            g.csfrac[c] = maxd(g.csfrac[c], fl);
            g.solfrac[c] = maxd(g.solfrac[c], (T)((double)fl * trackindx));
            if (g.temp[c] > ts) g.mpphase[c] = (T)trackid;
            if (g.temp[c] > (T)p.tliquid) g.mpliq[c] = (T)trackid;
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T> void launch_laser(Inst<T> &I)
{
    launch_k(I.pdl, laser_kernel<T>, I.nb_las, 256, 0, I.stream, I.p, I.g, I.red_las);
}
template <typename T> void launch_energy_bc(Inst<T> &I)
{
    launch_k(I.pdl, energy_bc_kernel<T>, I.nb_bc, 256, 0, I.stream, I.p, I.g, I.red_bc);
}
template <typename T> void launch_block_correct(Inst<T> &I, int ivar)
{
    launch_k(I.pdl, bc_reduce_kernel<T>, dim3(I.p.nip / 32, 4), dim3(32, 8), 0, I.stream, I.p, I.g);
    launch_k(I.pdl, block_correct_kernel<T>, 1, 1024, 4 * I.p.nip * sizeof(double), I.stream, I.p, I.g, I.red_asm, I.nb_asm, I.check_finite, ivar);
}
// Field read-out: the padded [k][j][nip] array widened to FP64 and packed to
// the reference's unpadded [k][j][ni] layout (CFDSolverManager.cpp:249), so
// that a single contiguous copy moves it to the host.
template <typename T>
__global__ void pack_field_kernel(const T *src, double *dst, int ni, int nip, long long rows)
{
    const long long n = rows * ni;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / ni;
        const int i = (int)(q - r * ni);
        dst[q] = (double)src[r * nip + i];
    }
}
template <typename T> void launch_pack_field(const T *src, double *dst, int ni, int nip,
                                             long long rows, int sm_count, cudaStream_t s)
{
    pack_field_kernel<T><<<sm_count * 4, 256, 0, s>>>(src, dst, ni, nip, rows);
}

// Cell-centred velocity for output (vtsBinWriter::transferVelNodes,
// vtsBinWriter.cpp:497-522): the mean of the two faces of component `comp`
// (0 u, 1 v, 2 w) on interior nodes of the active domain, zero where T <= T_solidus,
// on the boundary nodes and on inactive powder layers, packed to FP64 [k][j][ni].
template <typename T>
__global__ void centre_velocity_kernel(Params p, Fields<T> g, int comp, double *dst)
{
    const long long n = (long long)p.ni * p.nj * p.nk_alloc;  // every allocated plane
    const T *f = comp == 0 ? g.uvel : comp == 1 ? g.vvel : g.wvel;
    const size_t step = comp == 0 ? 1 : comp == 1 ? (size_t)p.nip : (size_t)p.nj * p.nip;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % p.ni);
        const long long r = q / p.ni;
        const int j = (int)(r % p.nj), k = (int)(r / p.nj);
        double v = 0.0;
        if (i >= 1 && i < p.nim1 && j >= 1 && j < p.njm1 && k >= 1 && k < p.nkm1) {
            const size_t c = cidx(i, j, k, p.nj, p.nip);
            v = ((double)f[c] + (double)f[c + step]) * 0.5;
            if ((double)g.temp[c] <= p.tsolid) v = 0.0;
        }
        dst[q] = v;
    }
}
template <typename T> void launch_centre_velocity(Inst<T> &I, int comp, double *dst)
{
    centre_velocity_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g, comp, dst);
}

// Resident 256-thread CTAs of h2t_kernel per SM (its grid is one full wave).
template <typename T> int h2t_blocks_per_sm()
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, h2t_kernel<T>, 256, 0);
    return nb > 0 ? nb : 1;
}
template <typename T> void launch_h2t(Inst<T> &I)
{
    launch_k(I.pdl, h2t_kernel<T>, I.nb_h2t, 256, 0, I.stream, I.p, I.g, I.red_h2t);
}
template <typename T> void launch_meltpool(Inst<T> &I)
{
    size_t smem = 3 * (size_t)I.p.nip * sizeof(double) + (size_t)I.p.nip * sizeof(int);
    launch_k(I.pdl, meltpool_kernel<T>, 1, 1024, smem, I.stream, I.p, I.g, I.red_h2t, I.nb_h2t);
}
template <typename T> void launch_converge(Inst<T> &I, double tol, const LoopCtl &lc)
{
    launch_k(I.pdl, converge_kernel<T>, 1, 1024, 0, I.stream, I.p, I.g, I.red_h2t, I.nb_h2t, I.red_bc, I.nb_bc,
                                                  I.red_las, I.nb_las, I.red_mom, I.nb_mom, tol,
                                                  I.check_finite, lc);
}
template <typename T> void launch_update_solutions(Inst<T> &I)
{
    launch_k(I.pdl, update_solutions_kernel<T>, I.grid_1d, 256, 0, I.stream, I.p, I.g, I.trackindx, I.trackid);
}

#define AMCFD_INST(T)                                        \
    template void launch_laser<T>(Inst<T> &);               \
    template void launch_energy_bc<T>(Inst<T> &);           \
    template void launch_block_correct<T>(Inst<T> &, int);  \
    template void launch_h2t<T>(Inst<T> &);                 \
    template int h2t_blocks_per_sm<T>();                    \
    template void launch_pack_field<T>(const T *, double *, int, int, long long, int, cudaStream_t); \
    template void launch_centre_velocity<T>(Inst<T> &, int, double *);                                \
    template void launch_meltpool<T>(Inst<T> &);            \
    template void launch_converge<T>(Inst<T> &, double, const LoopCtl &); \
    template void launch_update_solutions<T>(Inst<T> &);
AMCFD_INST(double)
AMCFD_INST(float)
#undef AMCFD_INST

}  // namespace amcfd
