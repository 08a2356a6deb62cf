// Fused energy assembly: discretizeEquations(5) (CFDSolverManager.cpp:1157-1264),
// calculateSource(5) (:1677-1843), calculateResiduals(5) (:2073-2101), the
// coefficient/residual sums of enhanceConvergenceSpeed(5) (:2310-2332) and
// bareplateMaterialProps (:2137-2189, written to the *_nxt buffers so that the
// old properties stay readable by neighbouring cells).
//
// 2.5-D stencil fed by TMA.  A CTA owns a 32 (i) x 8 (j) tile and walks a
// segment of k planes.  The ten input fields arrive in shared memory as 3-D
// tensor tiles (the tile plus a one-cell j halo and an i halo widened to 16
// bytes on each side, so every box starts on a 16-byte boundary) through two
// rings completing on mbarriers:
//   ring A (diff, h, f_l, rho, w): planes k-1, k, k+1 resident, k+2 in flight;
//   ring B (u, v, T, hnot, f_l,not): plane k resident, k+1 in flight.
// There is no CTA-wide barrier per plane: each warp counts itself done with a
// plane in a shared counter, and the last warp to finish plane k refills the
// slots that held planes k-1 (ring A) and k (ring B).  Warps therefore drift up
// to one plane apart instead of waiting for the slowest, and no thread waits on
// a global load.
// Face areas and volumes are products of per-column (x, y) and per-plane (z)
// widths, formed in FP64 in the reference's order.  The FP64 build's arithmetic
// is the reference's expression by expression; the FP32 build evaluates
// properties and divisions in FP32, and it and the defect-correction build form
// each face's conductance and Peclet number from one reciprocal.
#include <algorithm>

#include "kernels.cuh"
#include "async.cuh"

namespace amcfd {

constexpr int kTX = 32, kTY = 8, kKSEG = 16;

// Box geometry of the staged tiles, per element type.
template <typename T> struct AsmBox {
    static constexpr int OX = 16 / (int)sizeof(T);  // i halo: one 16-byte unit
    static constexpr int BX = kTX + 2 * OX;         // box width (elements)
    static constexpr int BY = kTY + 2;              // box height (rows)
    static constexpr int BYTES = BX * BY * (int)sizeof(T);
    static constexpr int FE = ((BYTES + 127) / 128 * 128) / (int)sizeof(T);  // 128-B aligned stride
    // fields per ring and ring slots (planes): FP32 rings take 50 KB, FP64 88 KB.
    // Deeper FP32 rings (5 + 3 planes, 67 KB) measured slower on the 400x200x100
    // deck: 328 against 286 us a launch.
    static constexpr int NA = 5, NB = 5, SA = 4, SB = 2;
    // rings + mbarriers + slack to align the dynamic region to 128 bytes
    static constexpr size_t SMEM = (size_t)(SA * NA + SB * NB) * FE * sizeof(T) + 8 * (SA + SB) + 128;
    // resident CTAs per SM: three in FP32 (80 registers a thread still hold the
    // whole stencil), two in FP64
    static constexpr int MINB = sizeof(T) == 4 ? 3 : 2;
};
// Warps of a CTA, and the plane-completion counters (a warp is at most one
// plane ahead of the slowest, so four counters never mix two planes).
constexpr int kAsmWarps = kTX * kTY / 32, kAsmCounters = 4;
enum { FA_D = 0, FA_H, FA_F, FA_R, FA_W };
enum { FB_U = 0, FB_V, FB_T, FB_HN, FB_FN };

// A face of the fast builds: conductance d = num / den (den = 1 on a boundary face,
// else the harmonic-mean denominator) and the pair D A(|F|/D) + max(0, -+F), with
// one reciprocal r = 1 / (num den): d = num^2 r and |F| / d = |F| den^2 r.
__device__ __forceinline__ float rcp_fast(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double rcp_fast(double x) { return 1.0 / x; }
template <typename R>
__device__ __forceinline__ void face_fast(int sch, R num, R den, R f, R &plus, R &minus)
{
    const R r = rcp_fast(num * den);
    const R d = num * num * r;
    const R a = d * scheme_fn<R>(sch, fabs(f) * (den * den * r));
    plus = a + maxd(R(0), -f);
    minus = a + maxd(R(0), f);
}

// SCH: the discretisation scheme as a compile-time constant (one instantiation per
// scheme), so that the six face coefficients carry no untaken scheme branches.
// DC (FP64 only, defect correction): the coefficients are formed in FP64 (with
// the fast builds' one reciprocal per face), stored rounded to FP32 in `dco`, and
// the FP32 `su` slot receives the FP64 defect su + sum a_nb h_nb - ap h of the
// current enthalpy; the FP64 coefficient arrays are not written.
template <typename T, int SCH, bool DC>
__global__ void __launch_bounds__(256, AsmBox<T>::MINB)
energy_assemble_kernel(Params p, Fields<T> g, double *red, const __grid_constant__ AsmMaps mp, DcBuf dco)
{
    pdl_enter();
    using R = T;
    using B = AsmBox<T>;
    constexpr int OX = B::OX, BX = B::BX, FE = B::FE;
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned char *base = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u);
    T *bufA = reinterpret_cast<T *>(base);
    T *bufB = bufA + B::SA * B::NA * FE;
    uint64_t *barA = reinterpret_cast<uint64_t *>(bufB + B::SB * B::NB * FE);
    uint64_t *barB = barA + B::SA;
    __shared__ uint32_t done_cnt[kAsmCounters];  // warps done, per plane (k - kb) mod 4
    __shared__ int lastA[B::SA], lastB[B::SB];  // last plane issued into each slot

    Status *st = g.st;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx, lane = tid & 31;
    const int i = blockIdx.x * kTX + tx, j = blockIdx.y * kTY + ty;
    const int x0 = blockIdx.x * kTX - OX, y0 = blockIdx.y * kTY - 1;
    const int ni = p.ni, nj = p.nj, nk = p.nk, nip = p.nip;
    const int nim1 = p.nim1, njm1 = p.njm1, nkm1 = p.nkm1, nim2 = p.nim2, njm2 = p.njm2,
              nkm2 = p.nkm2;
    const int kseg = (nk + gridDim.z - 1) / gridDim.z;
    const int kb = blockIdx.z * kseg, ke = min(kb + kseg, nk);
    const bool in = (i < ni && j < nj);
    const bool colint = in && i >= 1 && i <= nim2 && j >= 1 && j <= njm2;
    const size_t sk = (size_t)nj * nip;
    const size_t col = in ? cidx(i, j, 0, nj, nip) : 0;
    constexpr int sch = SCH;
    const double delt = st->delt;
    const bool volsrc = p.volsrc != 0;
    const bool powder = p.powder != 0;

    // ---- copy pipeline ----
    // Slots are filled in plane order (ring A from plane kb-1, ring B from kb),
    // so the n-th fill of a slot completes its barrier's phase of parity n & 1.
    auto slotA = [&](int q) { return (q - kb + 1) % B::SA; };
    auto parA = [&](int q) { return (uint32_t)(((q - kb + 1) / B::SA) & 1); };
    auto slotB = [&](int q) { return (q - kb) % B::SB; };
    auto parB = [&](int q) { return (uint32_t)(((q - kb) / B::SB) & 1); };
    auto issueA = [&](int q) {
        const int s = slotA(q);
        T *dst = bufA + s * B::NA * FE;
        lastA[s] = q;
        fence_proxy_async();
        mbar_expect_tx(&barA[s], B::NA * B::BYTES);
        tma_load_3d(dst + FA_D * FE, &mp.diff, x0, y0, q, &barA[s]);
        tma_load_3d(dst + FA_H * FE, &mp.h, x0, y0, q, &barA[s]);
        tma_load_3d(dst + FA_F * FE, &mp.fracl, x0, y0, q, &barA[s]);
        tma_load_3d(dst + FA_R * FE, &mp.rho, x0, y0, q, &barA[s]);
        tma_load_3d(dst + FA_W * FE, &mp.w, x0, y0, q, &barA[s]);
    };
    auto issueB = [&](int q) {
        const int s = slotB(q);
        T *dst = bufB + s * B::NB * FE;
        lastB[s] = q;
        fence_proxy_async();
        mbar_expect_tx(&barB[s], B::NB * B::BYTES);
        tma_load_3d(dst + FB_U * FE, &mp.u, x0, y0, q, &barB[s]);
        tma_load_3d(dst + FB_V * FE, &mp.v, x0, y0, q, &barB[s]);
        tma_load_3d(dst + FB_T * FE, &mp.temp, x0, y0, q, &barB[s]);
        tma_load_3d(dst + FB_HN * FE, &mp.hnot, x0, y0, q, &barB[s]);
        tma_load_3d(dst + FB_FN * FE, &mp.flnot, x0, y0, q, &barB[s]);
    };
    constexpr int kNone = -(1 << 30);
    // per-plane metrics of this segment, converted once for the CTA (the same
    // values every thread would form)
    __shared__ double pl_dz[kKSEG];
    __shared__ T pl_m[5][kKSEG];  // fracz[k], fracz[k-1], dzpbinv[k], dzpbinv[k+1], dz
    if (tid < ke - kb) {
        const int k = kb + tid;
        if (k >= 1 && k <= nkm2) {
            pl_dz[tid] = g.zw[k + 1] - g.zw[k];
            pl_m[0][tid] = (T)g.fracz[k];
            pl_m[1][tid] = (T)g.fracz[k - 1];
            pl_m[2][tid] = (T)g.dzpbinv[k];
            pl_m[3][tid] = (T)g.dzpbinv[k + 1];
            pl_m[4][tid] = (T)pl_dz[tid];
        }
    }

    if (tid == 0) {
        for (int s = 0; s < B::SA; ++s) { mbar_init(&barA[s]); lastA[s] = kNone; }
        for (int s = 0; s < B::SB; ++s) { mbar_init(&barB[s]); lastB[s] = kNone; }
        for (int s = 0; s < kAsmCounters; ++s) done_cnt[s] = 0u;
    }
    __syncthreads();
    if (kb >= ke) return;
    if (tid == 0) {
        for (int q = kb - 1; q <= min(kb - 2 + B::SA, ke); ++q) issueA(q);
        for (int q = kb; q <= min(kb - 1 + B::SB, ke - 1); ++q) issueB(q);
    }
    bool ok = mbar_wait(&barA[slotA(kb - 1)], parA(kb - 1), st, 1);
    if (ok) ok = mbar_wait(&barA[slotA(kb)], parA(kb), st, 1);

    // per-column metrics (interior columns only)
    double dx = 0.0, dy = 0.0;
    R fx_i = 0, fx_m = 0, dxp_i = 0, dxp_p = 0, fy_j = 0, fy_m = 0, dyp_j = 0, dyp_p = 0;
    if (colint) {
        dx = g.xu[i + 1] - g.xu[i];
        dy = g.yv[j + 1] - g.yv[j];
        fx_i = (R)g.fracx[i]; fx_m = (R)g.fracx[i - 1];
        dxp_i = (R)g.dxpwinv[i]; dxp_p = (R)g.dxpwinv[i + 1];
        fy_j = (R)g.fracy[j]; fy_m = (R)g.fracy[j - 1];
        dyp_j = (R)g.dypsinv[j]; dyp_p = (R)g.dypsinv[j + 1];
    }
    const R aij = (R)(dx * dy);
    // FP32: column widths rounded once, face areas and volumes as FP32 products; the
    // divisions by per-launch constants become multiplications by their reciprocals
    // (the FP64 build keeps the reference's FP64 products and exact divisions)
    constexpr bool kF32 = sizeof(R) == 4;
    // FAST (FP32 bulk, or FP64 under defect correction; neither is compared bit for
    // bit with the reference): one reciprocal per face instead of two divisions,
    // and the divisions by per-launch constants as multiplications
    constexpr bool FAST = kF32 || DC;
    const R fdx = (R)dx, fdy = (R)dy;
    const R inv_acpl = (R)(1.0 / p.acpl), inv_delt = (R)(1.0 / delt), inv_urfh = (R)(1.0 / p.urfh);
    const R dxp_e = (R)g.dxpwinv[nim1], dxp_w = (R)g.dxpwinv[1];
    const R dyp_n = (R)g.dypsinv[njm1], dyp_s = (R)g.dypsinv[1];
    const R dzp_t = (R)g.dzpbinv[nkm1], dzp_b = (R)g.dzpbinv[1];
    const R thla = (R)p.thconla, thlb = (R)p.thconlb, acpl = (R)p.acpl, thsa = (R)p.thconsa,
            thsb = (R)p.thconsb, thsc = (R)p.thconsc, acpa = (R)p.acpa, acpb = (R)p.acpb,
            tliq = (R)p.tliquid, tsol = (R)p.tsolid, denl = (R)p.denl, dens = (R)p.dens,
            visc = (R)p.viscos;
    double sumd = 0.0, sumh = 0.0;
    double bl = 0.0, blp = 0.0, blm = 0.0, blc = 0.0;
    const int o = (ty + 1) * BX + tx + OX;  // this thread's cell inside a box
    // the top face's coefficient as seen from the cell above (its bottom face),
    // carried from one plane to the next
    R ab_bottom = R(0);

    for (int k = kb; k < ke; ++k) {
        if (ok) ok = mbar_wait(&barA[slotA(k + 1)], parA(k + 1), st, 2);
        if (ok) ok = mbar_wait(&barB[slotB(k)], parB(k), st, 3);
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        const T *Am = bufA + slotA(k - 1) * B::NA * FE + o;  // plane k-1
        const T *Ac = bufA + slotA(k) * B::NA * FE + o;      // plane k
        const T *Ap = bufA + slotA(k + 1) * B::NA * FE + o;  // plane k+1
        const T *Bc = bufB + slotB(k) * B::NB * FE + o;      // plane k
        const size_t c = col + (size_t)k * sk;
        if (in) {
            const R d_c = Ac[FA_D * FE], f_c = Ac[FA_F * FE], t_c = Bc[FB_T * FE];
            // ---- material properties (every node) ----
            {
                const R t = t_c, fl = f_c;
                const R diffl = FAST ? (thla * t + thlb) * inv_acpl : bdiv(thla * t + thlb, acpl);
                R dn = diffl, rn = denl, vn = visc;
                if (!(t >= tliq)) {
                    R diffs, rs = dens;
                    if (!powder) {
                        diffs = bdiv(thsa * (t * t) + thsb * t + thsc, acpa * t + acpb);
                    } else {
                        // powderMaterialProps (CFDSolverManager.cpp:2236-2252): solid and
                        // powder mixed by the consolidated fraction
                        const R cs = g.csfrac[c];
                        const R cps = acpa * t + acpb;
                        const R conds = thsa * (t * t) + thsb * t + thsc;
                        const R diffp = bdiv((R)p.powderthcona * t + (R)p.powderthconb,
                                             (R)p.powdercpa * t + (R)p.powdercpb);
                        diffs = (R(1) - cs) * diffp + bdiv(cs * conds, cps);
                        rs = (R(1) - cs) * (R)p.powderden + cs * dens;
                    }
                    dn = diffs; rn = rs; vn = R(1e10);
                    if (!(t <= tsol)) {
                        dn = fl * diffl + (R(1) - fl) * diffs;
                        rn = fl * denl + (R(1) - fl) * rs;
                        vn = visc;
                    }
                }
                g.diff_nxt[c] = dn;
                g.rho_nxt[c] = rn;
                g.vis_nxt[c] = vn;
            }
            if (colint && k >= 1 && k <= nkm2) {
                const int kl = k - kb;
                const double dz = pl_dz[kl];
                const R fdz = pl_m[4][kl];
                const R aik = kF32 ? fdx * fdz : (R)(dx * dz), ajk = kF32 ? fdy * fdz : (R)(dy * dz);
                const R vol = kF32 ? aij * fdz : (R)(dx * dy * dz);
                const R fz_k = pl_m[0][kl], fz_m = pl_m[1][kl];
                const R dzp_k = pl_m[2][kl], dzp_p = pl_m[3][kl];
                const R dcc = d_c, rhc = Ac[FA_R * FE];
                const R d_e = Ac[FA_D * FE + 1], d_w = Ac[FA_D * FE - 1], d_nn = Ac[FA_D * FE + BX],
                        d_s = Ac[FA_D * FE - BX], d_m = Am[FA_D * FE], d_p = Ap[FA_D * FE];
                R an, as_, ae, aw, at, ab, tmp, ab_up;
                const R u_c = Bc[FB_U * FE], u_e = Bc[FB_U * FE + 1];
                const R v_c = Bc[FB_V * FE], v_n = Bc[FB_V * FE + BX];
                const R w_c = Ac[FA_W * FE], w_p = Ap[FA_W * FE];
                // north face
                {
                    R fn = Ac[FA_R * FE + BX] * v_n * aik;
                    if constexpr (FAST) {
                        const bool bnd = j == njm2;
                        const R num = bnd ? dcc * aik * dyp_n : dcc * d_nn * aik * dyp_p;
                        const R den = bnd ? R(1) : (R(1) - fy_j) * d_nn + fy_j * dcc;
                        face_fast<R>(sch, num, den, fn, an, tmp);
                    } else {
                        R dn;
                        if (j == njm2) {
                            dn = dcc * aik * dyp_n;
                        } else {
                            R difn = bdiv(dcc * d_nn, (R(1) - fy_j) * d_nn + fy_j * dcc);
                            dn = difn * aik * dyp_p;
                        }
                        face_coef<R>(sch, dn, fn, an, tmp);
                    }
                }
                // south face
                {
                    R fs = rhc * v_c * aik;
                    if constexpr (FAST) {
                        const bool bnd = j == 1;
                        const R num = bnd ? dcc * aik * dyp_s : d_s * dcc * aik * dyp_j;
                        const R den = bnd ? R(1) : (R(1) - fy_m) * dcc + fy_m * d_s;
                        face_fast<R>(sch, num, den, fs, tmp, as_);
                    } else {
                        R ds;
                        if (j == 1) {
                            ds = dcc * aik * dyp_s;
                        } else {
                            R difs = bdiv(d_s * dcc, (R(1) - fy_m) * dcc + fy_m * d_s);
                            ds = difs * aik * dyp_j;
                        }
                        face_coef<R>(sch, ds, fs, tmp, as_);
                    }
                }
                // east face
                {
                    R fe = Ac[FA_R * FE + 1] * u_e * ajk;
                    if constexpr (FAST) {
                        const bool bnd = i == nim2;
                        const R num = bnd ? dcc * ajk * dxp_e : dcc * d_e * ajk * dxp_p;
                        const R den = bnd ? R(1) : (R(1) - fx_i) * d_e + fx_i * dcc;
                        face_fast<R>(sch, num, den, fe, ae, tmp);
                    } else {
                        R de;
                        if (i == nim2) {
                            de = dcc * ajk * dxp_e;
                        } else {
                            R dife = bdiv(dcc * d_e, (R(1) - fx_i) * d_e + fx_i * dcc);
                            de = dife * ajk * dxp_p;
                        }
                        face_coef<R>(sch, de, fe, ae, tmp);
                    }
                }
                // west face
                {
                    R fw = rhc * u_c * ajk;
                    if constexpr (FAST) {
                        const bool bnd = i == 1;
                        const R num = bnd ? dcc * ajk * dxp_w : d_w * dcc * ajk * dxp_i;
                        const R den = bnd ? R(1) : (R(1) - fx_m) * dcc + fx_m * d_w;
                        face_fast<R>(sch, num, den, fw, tmp, aw);
                    } else {
                        R dw;
                        if (i == 1) {
                            dw = dcc * ajk * dxp_w;
                        } else {
                            R difw = bdiv(d_w * dcc, (R(1) - fx_m) * dcc + fx_m * d_w);
                            dw = difw * ajk * dxp_i;
                        }
                        face_coef<R>(sch, dw, fw, tmp, aw);
                    }
                }
                // top face
                {
                    R ft = Ap[FA_R * FE] * w_p * aij;
                    if constexpr (FAST) {
                        const bool bnd = k == nkm2;
                        const R num = bnd ? dcc * aij * dzp_t : dcc * d_p * aij * dzp_p;
                        const R den = bnd ? R(1) : (R(1) - fz_k) * d_p + fz_k * dcc;
                        face_fast<R>(sch, num, den, ft, at, ab_up);
                    } else {
                        R dt;
                        if (k == nkm2) {
                            dt = dcc * aij * dzp_t;
                        } else {
                            R dift = bdiv(dcc * d_p, (R(1) - fz_k) * d_p + fz_k * dcc);
                            dt = dift * aij * dzp_p;
                        }
                        face_coef<R>(sch, dt, ft, at, ab_up);
                    }
                }
                // bottom face: the top face of the plane below, as this thread formed
                // it there (same operands in the same order, so the same bits), or
                // formed here on the segment's first plane and on the boundary
                if (k > kb && k > 1) {
                    ab = ab_bottom;
                } else {
                    R fb = rhc * w_c * aij;
                    if constexpr (FAST) {
                        const bool bnd = k == 1;
                        const R num = bnd ? dcc * aij * dzp_b : d_m * dcc * aij * dzp_k;
                        const R den = bnd ? R(1) : (R(1) - fz_m) * dcc + fz_m * d_m;
                        face_fast<R>(sch, num, den, fb, tmp, ab);
                    } else {
                        R db;
                        if (k == 1) {
                            db = dcc * aij * dzp_b;
                        } else {
                            R difb = bdiv(d_m * dcc, (R(1) - fz_m) * dcc + fz_m * d_m);
                            db = difb * aij * dzp_k;
                        }
                        face_coef<R>(sch, db, fb, tmp, ab);
                    }
                }
                ab_bottom = ab_up;
                const R densbydt = FAST ? rhc * inv_delt : bdiv(rhc, (R)delt);
                const R apnot = densbydt * vol;
                R sp = R(0);
                R su = apnot * Bc[FB_HN * FE];
                // ---- calculateSource(5) ----
                if (volsrc) {
                    R srcin = R(0);
                    if (g.z[nkm1] - g.z[k] <= st->heatthick) {
                        double hr2 = st->heatrb * st->heatrb;
                        double bx = st->beamposx - g.x[i], by = st->beamposy - g.y[j];
                        srcin = (R)(st->avolpow * st->avolfact / M_PI / hr2 / st->heatthick *
                                    st->apowseta * exp(-st->avolfact / hr2 * ((bx * bx) + (by * by))) *
                                    (double)st->powerindicator);
                        su += vol * srcin;
                    }
                    g.sourceinput[c] = srcin;
                }
                const R hlatnt = (R)p.hlatnt;
                const R variable1 = FAST ? hlatnt * rhc * inv_delt : bdiv(hlatnt * rhc, (R)delt);
                const R volht = vol * variable1;
                const R flc = f_c;
                su -= volht * (flc - Bc[FB_FN * FE]);
                {
                    const R fl_w = Ac[FA_F * FE - 1], fl_e = Ac[FA_F * FE + 1],
                            fl_s = Ac[FA_F * FE - BX], fl_n = Ac[FA_F * FE + BX];
                    const R f_m = Am[FA_F * FE], f_p = Ap[FA_F * FE];
                    R flew = ajk * (maxd(u_c, R(0)) * fl_w - maxd(-u_c, R(0)) * flc +
                                    maxd(-u_e, R(0)) * fl_e - maxd(u_e, R(0)) * flc);
                    R flns = aik * (maxd(v_c, R(0)) * fl_s - maxd(-v_c, R(0)) * flc +
                                    maxd(-v_n, R(0)) * fl_n - maxd(v_n, R(0)) * flc);
                    R fltb = aij * (maxd(w_c, R(0)) * f_m - maxd(-w_c, R(0)) * flc +
                                    maxd(-w_p, R(0)) * f_p - maxd(w_p, R(0)) * flc);
                    su += rhc * hlatnt * (flew + flns + fltb);
                }
                const R hc = Ac[FA_H * FE];
                const R hjp = Ac[FA_H * FE + BX], hjm = Ac[FA_H * FE - BX], hip = Ac[FA_H * FE + 1],
                        him = Ac[FA_H * FE - 1], hkp = Ap[FA_H * FE], hkm = Am[FA_H * FE];
                // boundary folds, in the reference's order: k, j, i
                if (k == 1) { su += ab * hkm; sp -= ab; ab = R(0); }
                if (k == nkm2) { su += at * hkp; sp -= at; at = R(0); }
                if (j == 1) { su += as_ * hjm; sp -= as_; as_ = R(0); }
                if (j == njm2) { su += an * hjp; sp -= an; an = R(0); }
                if (i == 1) { su += aw * him; sp -= aw; aw = R(0); }
                if (i == nim2) { su += ae * hip; sp -= ae; ae = R(0); }
                R ap = an + as_ + ae + aw + at + ab + apnot - sp;
                const R urfh = (R)p.urfh;
                ap = FAST ? ap * inv_urfh : bdiv(ap, urfh);
                su += (R(1) - urfh) * ap * hc;
                if constexpr (DC) {
                    const double dfc = ae * hip + aw * him + an * hjp + as_ * hjm + at * hkp + ab * hkm + su - ap * hc;
                    dco.an[c] = (float)an; dco.as[c] = (float)as_; dco.ae[c] = (float)ae; dco.aw[c] = (float)aw;
                    dco.at[c] = (float)at; dco.ab[c] = (float)ab; dco.ap[c] = (float)ap; dco.su[c] = (float)dfc;
                    blc += dfc;
                } else {
                    g.an[c] = an; g.as[c] = as_; g.ae[c] = ae; g.aw[c] = aw;
                    g.at[c] = at; g.ab[c] = ab; g.ap[c] = ap; g.su[c] = su;
                }
                // neighbour sum of calculateResiduals(5); the FP32 build also takes the
                // block-correction defect from it (one sum instead of two)
                const R nbsum = an * hjp + as_ * hjm + ae * hip + aw * him + at * hkp + ab * hkm + su;
                if constexpr (!DC) {
                    // ---- block-correction sum of the defect (enhanceConvergenceSpeed(5)) ----
                    if constexpr (kF32)
                        blc += (double)(nbsum - ap * hc);
                    else
                        blc += (double)(ae * hip + aw * him + an * hjp + as_ * hjm + at * hkp + ab * hkm + su - ap * hc);
                }
                // ---- residual (calculateResiduals(5)) ----
                R r = bdiv(nbsum, ap) - hc;
                sumd += fabs((double)r);
                sumh += fabs((double)hc);
                // ---- block-correction sums (enhanceConvergenceSpeed(5)) ----
                bl += (double)(ap - an - as_ - at - ab);
                blp += (double)ae;
                blm += (double)aw;
            }
        }
        // this warp is done with planes k-1 (ring A) and k (ring B); the last warp
        // to finish plane k refills both slots (its reads are ordered before the
        // copies by the warp sync, the CTA-scope fences and the proxy fence)
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            const int r = k - kb;
            const uint32_t n = atomicAdd(&done_cnt[r % kAsmCounters], 1u);
            if (n == (uint32_t)(kAsmWarps * (r / kAsmCounters + 1) - 1)) {
                __threadfence_block();
                if (k - 1 + B::SA <= ke) issueA(k - 1 + B::SA);
                if (k + B::SB < ke) issueB(k + B::SB);
            }
        }
    }
    // every warp has left the plane loop: nothing is issued after this point
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            // drain the copies still in flight (bounded), then leave
            for (int s = 0; s < B::SA; ++s)
                if (lastA[s] != kNone) mbar_try(&barA[s], parA(lastA[s]), kSpinLimit);
            for (int s = 0; s < B::SB; ++s)
                if (lastB[s] != kNone) mbar_try(&barB[s], parB(lastB[s]), kSpinLimit);
        }
        return;
    }
    // per-i partial sums over this block's j-rows and planes, staged in ring A
    // (every copy has been consumed)
    double (*sb)[kTY][kTX + 1] = reinterpret_cast<double (*)[kTY][kTX + 1]>(base);
    sb[0][ty][tx] = bl;
    sb[1][ty][tx] = blp;
    sb[2][ty][tx] = blm;
    sb[3][ty][tx] = blc;
    __syncthreads();
    if (ty < 4 && i < nip) {
        double s = 0.0;
        for (int y = 0; y < kTY; ++y) s += sb[ty][y][tx];
        const int part = blockIdx.z * gridDim.y + blockIdx.y;
        g.bc[((size_t)part * 4 + ty) * nip + i] = s;
    }
    __syncthreads();
    double v[2] = {sumd, sumh};
    const int s[2] = {R_SUMD, R_SUMH};
    const bool m[2] = {false, false};
    const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    block_reduce_store<2>(v, s, m, red, blk);
}

// k-segments: long enough to amortise the two-plane prologue, short enough to
// give every SM several CTAs (at least 4 x 148 tiles x segments); kseg > 0 takes
// that segment length instead (4, 8 or 16 planes: the autotuner's candidates).
dim3 energy_assemble_grid(const Params &p, int kseg)
{
    const int tiles = ((p.ni + kTX - 1) / kTX) * ((p.nj + kTY - 1) / kTY);
    int seg = kKSEG;
    if (kseg > 0)
        seg = std::min(kseg, kKSEG);
    else
        while (seg > 4 && tiles * ((p.nk + seg - 1) / seg) < 4 * 148) seg /= 2;
    return dim3((p.ni + kTX - 1) / kTX, (p.nj + kTY - 1) / kTY, (p.nk + seg - 1) / seg);
}

// Tensor maps of the ten staged fields; set [q] reads diff/rho from the
// buffers that are current at property parity q (parity 0: diff_a, rho_a).
template <typename T> int make_assemble_maps(Inst<T> &I, T *diff_a, T *diff_b, T *rho_a, T *rho_b)
{
    using B = AsmBox<T>;
    const Params &p = I.p;
    const int e = (int)sizeof(T);
    auto enc = [&](CUtensorMap *m, const T *base) {
        return encode_field_map(m, base, e, p.nip, p.nj, p.nk, B::BX, B::BY);
    };
    for (int q = 0; q < 2; ++q) {
        AsmMaps &m = I.asm_maps[q];
        int rc = 0;
        if (!rc) rc = enc(&m.diff, q == 0 ? diff_a : diff_b);
        if (!rc) rc = enc(&m.rho, q == 0 ? rho_a : rho_b);
        if (!rc) rc = enc(&m.h, I.g.h);
        if (!rc) rc = enc(&m.fracl, I.g.fracl);
        if (!rc) rc = enc(&m.w, I.g.wvel);
        if (!rc) rc = enc(&m.u, I.g.uvel);
        if (!rc) rc = enc(&m.v, I.g.vvel);
        if (!rc) rc = enc(&m.temp, I.g.temp);
        if (!rc) rc = enc(&m.hnot, I.g.hnot);
        if (!rc) rc = enc(&m.flnot, I.g.fraclnot);
        if (rc) return rc;
    }
    I.asm_diff_a = diff_a;
    const int sm = (int)B::SMEM;
    cudaFuncSetAttribute(energy_assemble_kernel<T, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(energy_assemble_kernel<T, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(energy_assemble_kernel<T, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if constexpr (sizeof(T) == sizeof(double)) {
        cudaFuncSetAttribute(energy_assemble_kernel<T, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(energy_assemble_kernel<T, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(energy_assemble_kernel<T, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    return 0;
}

template <typename T, bool DC> static void assemble_scheme(Inst<T> &I, const AsmMaps &m)
{
    const dim3 blk(kTX, kTY);
    const size_t sm = AsmBox<T>::SMEM;
    switch (I.p.scheme) {
    case AMCFD_SCHEME_UPWIND:
        launch_k(I.pdl, energy_assemble_kernel<T, 0, DC>, I.asm_grid, blk, sm, I.stream, I.p, I.g, I.red_asm, m, I.dc);
        break;
    case AMCFD_SCHEME_POWER_LAW:
        launch_k(I.pdl, energy_assemble_kernel<T, 1, DC>, I.asm_grid, blk, sm, I.stream, I.p, I.g, I.red_asm, m, I.dc);
        break;
    default:
        launch_k(I.pdl, energy_assemble_kernel<T, 2, DC>, I.asm_grid, blk, sm, I.stream, I.p, I.g, I.red_asm, m, I.dc);
        break;
    }
}

template <typename T> void launch_energy_assemble(Inst<T> &I)
{
    const AsmMaps &m = I.g.diff_cur == I.asm_diff_a ? I.asm_maps[0] : I.asm_maps[1];
    if constexpr (sizeof(T) == sizeof(double)) {
        if (I.dc_on) {
            assemble_scheme<T, true>(I, m);
            return;
        }
    }
    assemble_scheme<T, false>(I, m);
}

template void launch_energy_assemble<double>(Inst<double> &);
template void launch_energy_assemble<float>(Inst<float> &);
template int make_assemble_maps<double>(Inst<double> &, double *, double *, double *, double *);
template int make_assemble_maps<float>(Inst<float> &, float *, float *, float *, float *);

}  // namespace amcfd
