// Momentum and pressure-correction chain over the melt-pool box
// (iterativeLoopSolve, CFDSolverManager.cpp:660-675): cleanVelocities, then for
// u, v, w, p': applyBCs, discretizeEquations + calculateSource +
// calculateResiduals (fused per cell), the line solver, and correctPressure.
// The box (istat..iend, jstat..jend, kstat..nkm1) lives in the device status
// block, so every launch has a fixed grid and walks the box with a stride.
#include <algorithm>

#include <cooperative_groups.h>

#include "kernels.cuh"
#include "linesolve.cuh"
#include "amcfd.h"

namespace cg = cooperative_groups;

namespace amcfd {

struct Box {
    int i0, i1, j0, j1, k0, k1, ni_, nj_, n;
};

__device__ __forceinline__ bool get_box(const Status *st, const Params &p, Box &b)
{
    if (!st->momentum_active) return false;
    b.i0 = st->istatp1; b.i1 = st->iendm1; b.j0 = st->jstat; b.j1 = st->jend;
    b.k0 = st->kstat; b.k1 = p.nkm2;
    b.ni_ = b.i1 - b.i0 + 1; b.nj_ = b.j1 - b.j0 + 1;
    b.n = (b.ni_ > 0 && b.nj_ > 0 && b.k1 >= b.k0) ? b.ni_ * b.nj_ * (b.k1 - b.k0 + 1) : 0;
    return b.n > 0;
}

__device__ __forceinline__ void box_cell(const Box &b, int q, int &i, int &j, int &k)
{
    i = b.i0 + q % b.ni_;
    int r = q / b.ni_;
    j = b.j0 + r % b.nj_;
    k = b.k0 + r / b.nj_;
}

// cleanVelocities (CFDSolverManager.cpp:2577-2620), one box cell.
template <typename T>
__device__ __forceinline__ void clean_cell(const Params &p, const Fields<T> &g, int i, int j, int k)
{
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const T ts = (T)p.tsolid;
    size_t c = cidx(i, j, k, nj, nip);
    T tc = g.temp[c];
    if (mind(tc, g.temp[c + 1]) <= ts) g.uvel[c + 1] = T(0);
    if (mind(tc, g.temp[c + sj]) <= ts) g.vvel[c + sj] = T(0);
    if (mind(tc, g.temp[c + sk]) <= ts) g.wvel[c + sk] = T(0);
}
template <typename T>
__global__ void clean_velocities_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    Box b;
    if (!get_box(g.st, p, b)) return;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < b.n; q += gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        clean_cell<T>(p, g, i, j, k);
    }
}

// Surface-tension gradient dsigma/dT (BoundCondManager.cpp:706-741).
__device__ __forceinline__ double surface_tension_gradient(double t, double a0, double dgdtp)
{
    const double A = 4.3e-4, R = 8314, Ts = 2.03e-8, k1 = 1.38e-2, H0 = -1.46e8;
    if (a0 < 0) return dgdtp;
    double K = k1 * exp(-H0 / R / t);
    double g = (-A - R * Ts * log(1 + K * a0) - (K * a0 / (1 + K * a0)) * (Ts * H0 / t)) * 1;
    if (t >= 2500) g = 0;
    return g;
}

// applyBCs(1..4) (BoundCondManager.cpp:472-564): Marangoni shear on the top
// plane for u and v, zero values on the box's east/west faces.  Item q < ntop is
// a top-plane cell, the rest are east/west edge pairs.  For u it returns |u| on
// the top plane (the reference momentum of calculateResiduals(1),
// CFDSolverManager.cpp:1983-1991), else 0.
__device__ __forceinline__ int mom_bc_items(const Params &p, const Status *st, const Box &b, int ivar,
                                            int &ntop)
{
    ntop = (ivar <= 2) ? b.ni_ * b.nj_ : 0;
    return ntop + b.nj_ * (p.nkm1 - b.k0);
}
template <typename T>
__device__ __forceinline__ double mom_bc_item(const Params &p, const Fields<T> &g, const Status *st,
                                              const Box &b, int ivar, int q, int ntop)
{
    const int nj = p.nj, nip = p.nip, nkm1 = p.nkm1, nkm2 = p.nkm2;
    T *phi = ivar == 1 ? g.uvel : ivar == 2 ? g.vvel : ivar == 3 ? g.wvel : g.pp;
    if (q < ntop) {
        int i = b.i0 + q % b.ni_, j = b.j0 + q / b.ni_;
        size_t ct = cidx(i, j, nkm1, nj, nip), cb = cidx(i, j, nkm2, nj, nip);
        double tt = (double)g.temp[ct];
        double grad, fl, vis1;
        if (ivar == 1) {
            double fx = g.fracx[i - 1];
            grad = (tt - (double)g.temp[ct - 1]) * g.dxpwinv[i];
            fl = (double)g.fracl[ct] * (1.0 - fx) + (double)g.fracl[ct - 1] * fx;
            double vc = (double)g.vis_nxt[cb], vw = (double)g.vis_nxt[cb - 1];
            vis1 = vc * vw / (vc * (1.0 - fx) + vw * fx);
        } else {
            double fy = g.fracy[j - 1];
            grad = (tt - (double)g.temp[ct - nip]) * g.dypsinv[j];
            fl = (double)g.fracl[ct] * (1.0 - fy) + (double)g.fracl[ct - nip] * fy;
            double vc = (double)g.vis_nxt[cb], vs = (double)g.vis_nxt[cb - nip];
            vis1 = vc * vs / (vc * (1.0 - fy) + vs * fy);
        }
        double term1 = fl * surface_tension_gradient(tt, p.a_oxygen, p.dgdtp) * grad /
                       (vis1 * g.dzpbinv[nkm1]);
        T val = (T)((double)phi[cb] + term1);
        phi[ct] = val;
        return ivar == 1 ? fabs((double)val) : 0.0;
    }
    int r = q - ntop;
    int j = b.j0 + r % b.nj_, k = b.k0 + r / b.nj_;
    phi[cidx(st->istat, j, k, nj, nip)] = T(0);
    phi[cidx(st->iend, j, k, nj, nip)] = T(0);
    return 0.0;
}
template <typename T>
__global__ void mom_bc_kernel(Params p, Fields<T> g, int ivar, double *red_umax)
{
    pdl_enter();
    Box b;
    const Status *st = g.st;
    double umax = 0.0;
    if (get_box(st, p, b)) {
        int ntop;
        const int n = mom_bc_items(p, st, b, ivar, ntop);
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
            umax = maxd(umax, mom_bc_item<T>(p, g, st, b, ivar, q, ntop));
    }
    if (ivar == 1) {
        double v[1] = {umax};
        const int s[1] = {R_UMAX};
        const bool m[1] = {true};
        block_reduce_store<1>(v, s, m, red_umax, blockIdx.x);
    }
}

// One cell of the u/v/w equation (ivar 1..3) of the momentum box: coefficients,
// source, under-relaxation, the solid freeze and d = A/ap, written to the shared
// coefficient arrays; returns |residual| of the cell (calculateResiduals(1..3)).
template <typename T>
__device__ __forceinline__ double mom_assemble_cell(const Params &p, const Fields<T> &g, const Status *st,
                                                    int ivar, int i, int j, int k)
{
    using R = T;
    const int nj = p.nj, nip = p.nip, nkm2 = p.nkm2, njm2 = p.njm2, nim2 = p.nim2;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const int sch = p.scheme;
    const R delt = (R)st->delt;
    const R *u = g.uvel, *v = g.vvel, *w = g.wvel, *rho = g.rho_nxt, *vis = g.vis_nxt;
    const double *fx = g.fracx, *fy = g.fracy, *fz = g.fracz, *xu = g.xu, *yv = g.yv, *zw = g.zw;
    const size_t c = cidx(i, j, k, nj, nip);
    R an, as_, ae, aw, at, ab, apnot, su, sp, tmp, areaD, vol;
    const R rc = rho[c];
    R *phi;
    const R *phinot;
    size_t cn;  // upstream scalar node of the staggered cell
    R urf, flv;
    if (ivar == 1) {
        const R fxm = (R)fx[i - 1];
        R vn = v[c + sj] * (R(1) - fxm) + v[c + sj - 1] * fxm;
        R vs = v[c] * (R(1) - fxm) + v[c - 1] * fxm;
        R ue = (u[c + 1] + u[c]) * R(0.5);
        R uw = (u[c - 1] + u[c]) * R(0.5);
        R wt = w[c + sk] * (R(1) - fxm) + w[c + sk - 1] * fxm;
        R wb = w[c] * (R(1) - fxm) + w[c - 1] * fxm;
        const R auik = (R)area_uik(g, i, k), ajk = (R)area_jk(p, g, j, k), auij = (R)area_uij(g, i, j);
        R fn = vn * rc * auik, fs = vs * rc * auik, fe = ue * rc * ajk, fw = uw * rc * ajk;
        R ft = wt * rc * auij, fb = wb * rc * auij;
        R visu = vis[c] * vis[c - 1] / (fxm * vis[c - 1] + (R(1) - fxm) * vis[c]);
        R visun = vis[c + sj] * vis[c + sj - 1] / (fxm * vis[c + sj - 1] + (R(1) - fxm) * vis[c + sj]);
        R visus = vis[c - sj] * vis[c - sj - 1] / (fxm * vis[c - sj - 1] + (R(1) - fxm) * vis[c - sj]);
        R visn = (j == njm2) ? visu : visu * visun / ((R(1) - (R)fy[j]) * visun + (R)fy[j] * visu);
        R viss = (j == 1) ? visu : visu * visus / ((R)fy[j - 1] * visus + (R(1) - (R)fy[j - 1]) * visu);
        R vise = vis[c], visw = vis[c - 1];
        R visut = vis[c + sk] * vis[c + sk - 1] / (fxm * vis[c + sk - 1] + (R(1) - fxm) * vis[c + sk]);
        R visub = vis[c - sk] * vis[c - sk - 1] / (fxm * vis[c - sk - 1] + (R(1) - fxm) * vis[c - sk]);
        R vist = (k == nkm2) ? visu : visut * visu / ((R)fz[k] * visu + (R(1) - (R)fz[k]) * visut);
        R visb = (k == 1) ? visu : visub * visu / ((R(1) - (R)fz[k - 1]) * visu + (R)fz[k - 1] * visub);
        R dn = visn * auik * (R)g.dypsinv[j + 1], ds = viss * auik * (R)g.dypsinv[j];
        R de = vise * ajk / (R)(xu[i + 1] - xu[i]), dw = visw * ajk / (R)(xu[i] - xu[i - 1]);
        R dt = vist * auij * (R)g.dzpbinv[k + 1], db = visb * auij * (R)g.dzpbinv[k];
        face_coef<R>(sch, dn, fn, an, tmp);
        face_coef<R>(sch, ds, fs, tmp, as_);
        face_coef<R>(sch, de, fe, ae, tmp);
        face_coef<R>(sch, dw, fw, tmp, aw);
        face_coef<R>(sch, dt, ft, at, tmp);
        face_coef<R>(sch, db, fb, tmp, ab);
        vol = (R)volume_u(g, i, j, k);
        apnot = rc * vol / delt;
        R delf = fn - fs + fe - fw + ft - fb;
        R cp0 = maxd(R(0), delf), cp1 = mind(R(0), delf);
        su = -cp1 * u[c];
        su += ajk * (g.pressure[c - 1] - g.pressure[c]);
        sp = -cp0;
        su += apnot * g.unot[c];
        R dudxp = (u[c + 1] - u[c]) / (R)(xu[i + 1] - xu[i]);
        R dudxm = (u[c] - u[c - 1]) / (R)(xu[i] - xu[i - 1]);
        su += (vise * dudxp - visw * dudxm) * ajk;
        R dvdxp = (v[c + sj] - v[c + sj - 1]) * (R)g.dxpwinv[i];
        R dvdxm = (v[c] - v[c - 1]) * (R)g.dxpwinv[i];
        su += (visn * dvdxp - viss * dvdxm) * auik;
        R dwdxp = (w[c + sk] - w[c + sk - 1]) * (R)g.dxpwinv[i];
        R dwdxm = (w[c] - w[c - 1]) * (R)g.dxpwinv[i];
        su += (vist * dwdxp - visb * dwdxm) * auij;
        phi = g.uvel; phinot = g.unot; cn = c - 1; urf = (R)p.urfu; areaD = ajk;
        flv = g.fracl[c] * (R(1) - fxm) + g.fracl[c - 1] * fxm;
    } else if (ivar == 2) {
        const R fym = (R)fy[j - 1];
        R vn = (v[c] + v[c + sj]) * R(0.5);
        R vs = (v[c] + v[c - sj]) * R(0.5);
        R ue = u[c + 1] * (R(1) - fym) + u[c + 1 - sj] * fym;
        R uw = u[c] * (R(1) - fym) + u[c - sj] * fym;
        R wt = w[c + sk] * (R(1) - fym) + w[c + sk - sj] * fym;
        R wb = w[c] * (R(1) - fym) + w[c - sj] * fym;
        const R aik = (R)area_ik(p, g, i, k), avjk = (R)area_vjk(g, j, k), avij = (R)area_vij(g, i, j);
        R fn = vn * rc * aik, fs = vs * rc * aik, fe = ue * rc * avjk, fw = uw * rc * avjk;
        R ft = wt * rc * avij, fb = wb * rc * avij;
        R visn = vis[c], viss = vis[c - sj];
        R visv = vis[c] * vis[c - sj] / (fym * vis[c - sj] + (R(1) - fym) * vis[c]);
        R visve = vis[c + 1] * vis[c + 1 - sj] / (fym * vis[c + 1 - sj] + (R(1) - fym) * vis[c + 1]);
        R visvw = vis[c - 1] * vis[c - 1 - sj] / (fym * vis[c - 1 - sj] + (R(1) - fym) * vis[c - 1]);
        R vise = (i == nim2) ? visv : visv * visve / ((R(1) - (R)fx[i]) * visve + (R)fx[i] * visv);
        R visw = (i == 1) ? visv : visv * visvw / ((R)fx[i - 1] * visvw + (R(1) - (R)fx[i - 1]) * visv);
        R visvt = vis[c + sk] * vis[c + sk - sj] / (fym * vis[c + sk - sj] + (R(1) - fym) * vis[c + sk]);
        R visvb = vis[c - sk] * vis[c - sk - sj] / (fym * vis[c - sk - sj] + (R(1) - fym) * vis[c - sk]);
        R vist = (k == nkm2) ? visv : visv * visvt / ((R(1) - (R)fz[k]) * visvt + (R)fz[k] * visv);
        R visb = (k == 1) ? visv : visv * visvb / ((R)fz[k - 1] * visvb + (R(1) - (R)fz[k - 1]) * visv);
        R dn = visn * aik / (R)(yv[j + 1] - yv[j]), ds = viss * aik / (R)(yv[j] - yv[j - 1]);
        R de = vise * avjk * (R)g.dxpwinv[i + 1], dw = visw * avjk * (R)g.dxpwinv[i];
        R dt = vist * avij * (R)g.dzpbinv[k + 1], db = visb * avij * (R)g.dzpbinv[k];
        face_coef<R>(sch, dn, fn, an, tmp);
        face_coef<R>(sch, ds, fs, tmp, as_);
        face_coef<R>(sch, de, fe, ae, tmp);
        face_coef<R>(sch, dw, fw, tmp, aw);
        face_coef<R>(sch, dt, ft, at, tmp);
        face_coef<R>(sch, db, fb, tmp, ab);
        vol = (R)volume_v(g, i, j, k);
        apnot = rc * vol / delt;
        R delf = fn - fs + fe - fw + ft - fb;
        R cp0 = maxd(R(0), delf), cp1 = mind(R(0), delf);
        su = -cp1 * v[c];
        su += aik * (g.pressure[c - sj] - g.pressure[c]);
        sp = -cp0;
        su += apnot * g.vnot[c];
        R dudyp = (u[c + 1] - u[c + 1 - sj]) * (R)g.dypsinv[j];
        R dudym = (u[c] - u[c - sj]) * (R)g.dypsinv[j];
        su += (vise * dudyp - visw * dudym) * avjk;
        R dvdyp = (v[c + sj] - v[c]) / (R)(yv[j + 1] - yv[j]);
        R dvdym = (v[c] - v[c - sj]) / (R)(yv[j] - yv[j - 1]);
        su += (visn * dvdyp - viss * dvdym) * aik;
        R dwdyp = (w[c + sk] - w[c + sk - sj]) * (R)g.dypsinv[j];
        R dwdym = (w[c] - w[c - sj]) * (R)g.dypsinv[j];
        su += (vist * dwdyp - visb * dwdym) * avij;
        phi = g.vvel; phinot = g.vnot; cn = c - sj; urf = (R)p.urfv; areaD = aik;
        flv = g.fracl[c] * (R(1) - fym) + g.fracl[c - sj] * fym;
    } else {
        const R fzm = (R)fz[k - 1];
        R vn = v[c + sj] * (R(1) - fzm) + v[c + sj - sk] * fzm;
        R vs = v[c] * (R(1) - fzm) + v[c - sk] * fzm;
        R ue = u[c + 1] * (R(1) - fzm) + u[c + 1 - sk] * fzm;
        R uw = u[c] * (R(1) - fzm) + u[c - sk] * fzm;
        R wt = (w[c] + w[c + sk]) * R(0.5);
        R wb = (w[c] + w[c - sk]) * R(0.5);
        const R awik = (R)area_wik(g, i, k), awjk = (R)area_wjk(g, j, k), aij = (R)area_ij(p, g, i, j);
        R fn = vn * rc * awik, fs = vs * rc * awik, fe = ue * rc * awjk, fw = uw * rc * awjk;
        R ft = wt * rc * aij, fb = wb * rc * aij;
        R vis_w = vis[c] * vis[c - sk] / (fzm * vis[c - sk] + (R(1) - fzm) * vis[c]);
        R viswn = vis[c + sj] * vis[c + sj - sk] / (fzm * vis[c + sj - sk] + (R(1) - fzm) * vis[c + sj]);
        R visws = vis[c - sj] * vis[c - sj - sk] / (fzm * vis[c - sj - sk] + (R(1) - fzm) * vis[c - sj]);
        R visn = (j == njm2) ? vis_w : vis_w * viswn / ((R(1) - (R)fy[j]) * viswn + (R)fy[j] * vis_w);
        R viss = (j == 1) ? vis_w : vis_w * visws / ((R)fy[j - 1] * visws + (R(1) - (R)fy[j - 1]) * vis_w);
        R viswe = vis[c + 1] * vis[c + 1 - sk] / (fzm * vis[c + 1 - sk] + (R(1) - fzm) * vis[c + 1]);
        R visww = vis[c - 1] * vis[c - 1 - sk] / (fzm * vis[c - 1 - sk] + (R(1) - fzm) * vis[c - 1]);
        R vise = (i == nim2) ? vis_w : vis_w * viswe / ((R(1) - (R)fx[i]) * viswe + (R)fx[i] * vis_w);
        R visw = (i == 1) ? vis_w : vis_w * visww / ((R)fx[i - 1] * visww + (R(1) - (R)fx[i - 1]) * vis_w);
        R vist = vis[c], visb = vis[c - sk];
        R dn = visn * awik * (R)g.dypsinv[j + 1], ds = viss * awik * (R)g.dypsinv[j];
        R de = vise * awjk * (R)g.dxpwinv[i + 1], dw = visw * awjk * (R)g.dxpwinv[i];
        R dt = vist * aij / (R)(zw[k + 1] - zw[k]), db = visb * aij / (R)(zw[k] - zw[k - 1]);
        face_coef<R>(sch, dn, fn, an, tmp);
        face_coef<R>(sch, ds, fs, tmp, as_);
        face_coef<R>(sch, de, fe, ae, tmp);
        face_coef<R>(sch, dw, fw, tmp, aw);
        face_coef<R>(sch, dt, ft, at, tmp);
        face_coef<R>(sch, db, fb, tmp, ab);
        vol = (R)volume_w(g, i, j, k);
        apnot = rc * vol / delt;
        R delf = fn - fs + fe - fw + ft - fb;
        R cp0 = maxd(R(0), delf), cp1 = mind(R(0), delf);
        su = -cp1 * w[c];
        su += aij * (g.pressure[c - sk] - g.pressure[c]);
        sp = -cp0;
        su += apnot * g.wnot[c];
        R dudzp = (u[c + 1] - u[c + 1 - sk]) * (R)g.dzpbinv[k];
        R dudzm = (u[c] - u[c - sk]) * (R)g.dzpbinv[k];
        su += (vise * dudzp - visw * dudzm) * awjk;
        R dvdzp = (v[c + sj] - v[c + sj - sk]) * (R)g.dzpbinv[k];
        R dvdzm = (v[c] - v[c - sk]) * (R)g.dzpbinv[k];
        su += (visn * dvdzp - viss * dvdzm) * awik;
        R dwdzp = (w[c + sk] - w[c]) / (R)(zw[k + 1] - zw[k]);
        R dwdzm = (w[c] - w[c - sk]) / (R)(zw[k] - zw[k - 1]);
        su += (vist * dwdzp - visb * dwdzm) * aij;
        phi = g.wvel; phinot = g.wnot; cn = c - sk; urf = (R)p.urfw; areaD = aij;
        flv = g.fracl[c] * (R(1) - fzm) + g.fracl[c - sk] * fzm;
    }
    (void)phinot;
    // ---- calculateSource ----
    if (flv > R(0)) {
        R term = (R)p.darcyKo * ((R(1) - flv) * (R(1) - flv)) / ((flv * flv * flv) + (R)kSmall);
        sp -= term * vol;
        if (p.steady) {
            R area = ivar == 1 ? (R)area_jk(p, g, j, k) : ivar == 2 ? (R)area_vjk(g, j, k)
                                                                    : (R)area_wjk(g, j, k);
            su += rc * (R)st->scanvel * area * (phi[c - 1] - phi[c]);
        }
        if (ivar == 3) {
            R fzm = (R)fz[k - 1];
            R boufac = rc * (R)p.grav * (R)p.beta;
            R tw = g.temp[c] * (R(1) - fzm) + g.temp[c - sk] * fzm;
            su += boufac * vol * (tw - (R)p.tsolid);
        }
    }
    if (ivar != 3 && k == nkm2) {
        su += at * phi[c + sk];
        sp -= at;
        at = R(0);
    }
    R ap = an + as_ + ae + aw + at + ab + apnot - sp;
    R dcoef = areaD / ap;
    ap /= urf;
    su += (R(1) - urf) * ap * phi[c];
    dcoef *= urf;
    if (mind(g.temp[c], g.temp[cn]) <= (R)p.tsolid) {
        su = R(0);
        an = as_ = ae = aw = at = ab = R(0);
        ap = (R)kLarge;
    }
    g.an[c] = an; g.as[c] = as_; g.ae[c] = ae; g.aw[c] = aw; g.at[c] = at; g.ab[c] = ab;
    g.ap[c] = ap; g.su[c] = su;
    (ivar == 1 ? g.dux : ivar == 2 ? g.dvy : g.dwz)[c] = dcoef;
    R r = an * phi[c + sj] + as_ * phi[c - sj] + ae * phi[c + 1] + aw * phi[c - 1] +
          at * phi[c + sk] + ab * phi[c - sk] + su - ap * phi[c];
    return fabs((double)r);
}

// discretizeEquations(1..3) + calculateSource(1..3) + calculateResiduals(1..3)
// (CFDSolverManager.cpp:771-1111, 1408-1644, 1960-2046), one box cell per thread.
template <typename T>
__global__ void __launch_bounds__(256) mom_assemble_kernel(Params p, Fields<T> g, int ivar, double *red)
{
    pdl_enter();
    Box b;
    double sumd = 0.0;
    if (get_box(g.st, p, b)) {
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < b.n; q += gridDim.x * blockDim.x) {
            int i, j, k;
            box_cell(b, q, i, j, k);
            sumd += mom_assemble_cell<T>(p, g, g.st, ivar, i, j, k);
        }
    }
    double v[1] = {sumd};
    const int s[1] = {R_MSUMD};
    const bool m[1] = {false};
    block_reduce_store<1>(v, s, m, red, blockIdx.x);
}

// discretizeEquations(4) + calculateSource(4) + calculateResiduals(4)
// (CFDSolverManager.cpp:1112-1156, 1645-1676, 2047-2071), one box cell: p'
// coefficients, |mass imbalance| and the mass-flux denominator added to the sums.
template <typename T>
__device__ __forceinline__ void pp_assemble_cell(const Params &p, const Fields<T> &g, int i, int j, int k,
                                                 double &resorm, double &denom)
{
    using R = T;
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const R *u = g.uvel, *v = g.vvel, *w = g.wvel, *rho = g.rho_nxt;
    const size_t c = cidx(i, j, k, nj, nip);
    const R rc = rho[c];
    const R aik = (R)area_ik(p, g, i, k), ajk = (R)area_jk(p, g, j, k), aij = (R)area_ij(p, g, i, j);
    R an = aik * g.dvy[c + sj] * rc;
    R as_ = aik * g.dvy[c] * rc;
    R ae = ajk * g.dux[c + 1] * rc;
    R aw = ajk * g.dux[c] * rc;
    R at = aij * g.dwz[c + sk] * rc;
    R ab = aij * g.dwz[c] * rc;
    R fn = v[c + sj] * aik * rc, fs = v[c] * aik * rc;
    R fe = u[c + 1] * ajk * rc, fw = u[c] * ajk * rc;
    R ft = w[c + sk] * aij * rc, fb = w[c] * aij * rc;
    R delf = fn - fs + fe - fw + ft - fb;
    R sp = R(0), su = -delf;
    resorm += fabs((double)delf);
    R ap = an + as_ + ae + aw + at + ab - sp;
    if (g.temp[c] <= (R)p.tsolid) {
        su = R(0);
        an = as_ = ae = aw = at = ab = R(0);
        ap = (R)kLarge;
    }
    g.an[c] = an; g.as[c] = as_; g.ae[c] = ae; g.aw[c] = aw; g.at[c] = at; g.ab[c] = ab;
    g.ap[c] = ap; g.su[c] = su;
    double dtp = (fabs((double)u[c]) + fabs((double)u[c + 1])) * (double)ajk +
                 (fabs((double)v[c]) + fabs((double)v[c + sj])) * (double)aik +
                 (fabs((double)w[c]) + fabs((double)w[c + sk])) * (double)aij;
    denom += 0.5 * fabs(dtp);
}
template <typename T>
__global__ void __launch_bounds__(256) pp_assemble_kernel(Params p, Fields<T> g, double *red)
{
    pdl_enter();
    Box b;
    double resorm = 0.0, denom = 0.0;
    if (get_box(g.st, p, b)) {
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < b.n; q += gridDim.x * blockDim.x) {
            int i, j, k;
            box_cell(b, q, i, j, k);
            pp_assemble_cell<T>(p, g, i, j, k, resorm, denom);
        }
    }
    double vv[2] = {resorm, denom};
    const int s[2] = {R_MRESORM, R_MDENOM};
    const bool m[2] = {false, false};
    block_reduce_store<2>(vv, s, m, red, blockIdx.x);
}

// correctPressure (CFDSolverManager.cpp:2692-2758): velocity correction, then
// pressure update (two passes: the second zeroes p' that the first reads).
template <typename T>
__device__ __forceinline__ void correct_velocity_cell(const Params &p, const Fields<T> &g, int i, int j, int k)
{
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const T ts = (T)p.tsolid;
    size_t c = cidx(i, j, k, nj, nip);
    T tc = g.temp[c], ppc = g.pp[c];
    if (mind(tc, g.temp[c - 1]) > ts) g.uvel[c] += g.dux[c] * (g.pp[c - 1] - ppc);
    if (mind(tc, g.temp[c - sj]) > ts) g.vvel[c] += g.dvy[c] * (g.pp[c - sj] - ppc);
    if (mind(tc, g.temp[c - sk]) > ts) g.wvel[c] += g.dwz[c] * (g.pp[c - sk] - ppc);
}
template <typename T>
__device__ __forceinline__ void correct_pressure_cell(const Params &p, const Fields<T> &g, int i, int j, int k)
{
    size_t c = cidx(i, j, k, p.nj, p.nip);
    if (g.temp[c] > (T)p.tsolid) {
        g.pressure[c] += (T)p.urfp * g.pp[c];
        g.pp[c] = T(0);
    }
}
template <typename T>
__global__ void correct_velocity_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    Box b;
    if (!get_box(g.st, p, b)) return;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < b.n; q += gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_velocity_cell<T>(p, g, i, j, k);
    }
}
template <typename T>
__global__ void correct_pressure_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    Box b;
    if (!get_box(g.st, p, b)) return;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < b.n; q += gridDim.x * blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_pressure_cell<T>(p, g, i, j, k);
    }
}

// Momentum residual normalisation (CFDSolverManager.cpp:1983-1991, 2018, 2044,
// 2069-2070), one CTA.
__device__ double reduce_region(const double *red, int nb, int slot, bool is_max, double *scratch)
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
    if (warp == 0) {
        double r = (lane < (int)(blockDim.x >> 5)) ? scratch[lane] : (is_max ? -INFINITY : 0.0);
        r = is_max ? warp_max(r) : warp_sum(r);
        if (lane == 0) scratch[32] = r;
    }
    __syncthreads();
    double r = scratch[32];
    __syncthreads();
    return r;
}

// Normalised momentum residuals from the reduced sums (one thread).
__device__ __forceinline__ void mom_finalize_status(const Params &p, Status *st, double s1, double s2,
                                                    double s3, double rm, double dn, double umax)
{
    umax = fmax(umax, 0.0);
    double refmom = 0.25 * M_PI * (st->width * st->width) * p.dens * (umax * umax);
    st->umaxt = umax;
    st->refmom = refmom;
    st->resoru = s1 / refmom;
    st->resorv = s2 / refmom;
    st->resorw = s3 / refmom;
    dn *= p.dens;
    st->mass_denom = dn;
    st->resorm = rm / (dn + kSmall);
}

// Reduces the per-CTA partials of the four equations (regions 0..3, nb CTAs each)
// and max |u| on the top plane (region 4, nb_umax entries).
__device__ void mom_finalize_body(const Params &p, Status *st, const double *red, int nb, int nb_umax,
                                  double *scratch)
{
    const size_t region = (size_t)nb * R_NSLOTS;
    __shared__ double scr5[5 * 33];
    const double *rb[5] = {red, red + region, red + 2 * region, red + 3 * region, red + 3 * region};
    const int rs[5] = {R_MSUMD, R_MSUMD, R_MSUMD, R_MRESORM, R_MDENOM};
    double sv[5];
    reduce_sums<5>(rb, rs, nb, sv, scr5);
    const double s1 = sv[0], s2 = sv[1], s3 = sv[2], rm = sv[3], dn = sv[4];
    double umax = reduce_region(red + 4 * region, nb_umax, R_UMAX, true, scratch);
    if (threadIdx.x == 0) mom_finalize_status(p, st, s1, s2, s3, rm, dn, umax);
}

template <typename T>
__global__ void mom_finalize_kernel(Params p, Fields<T> g, const double *red, int nb)
{
    pdl_enter();
    __shared__ double scratch[40];
    Status *st = g.st;
    if (!st->momentum_active) return;
    mom_finalize_body(p, st, red, nb, nb, scratch);
}

// Pass-completion flags of the box's lines (one int per (j, k) line), for the
// resident passes: a line's flag is base + t + 1 once pass t of it is stored,
// base = 16 x the launch's sequence number, so every value an earlier launch left
// is below every target of this one.
struct LineFlags {
    int *f;
    int nj, j0, j1, k0, k1, base;
};
__device__ __forceinline__ int ld_acquire_gpu_int(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu_int(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Before pass t of line (j, k): lanes 0..3 wait (bounded) until the four
// neighbouring lines in the box, of the other colour, have stored pass t - 1;
// the warp barrier then orders those acquires before every lane's reads.
// False (for the whole warp) when a wait gave up or an error is raised.
__device__ __forceinline__ bool wait_neighbours(const LineFlags &lf, int j, int k, int t, Status *st, long long polls)
{
    const int lane = threadIdx.x & 31;
    int jn = j, kn = k;
    bool need = false;
    if (lane == 0) { jn = j - 1; need = jn >= lf.j0; }
    else if (lane == 1) { jn = j + 1; need = jn <= lf.j1; }
    else if (lane == 2) { kn = k - 1; need = kn >= lf.k0; }
    else if (lane == 3) { kn = k + 1; need = kn <= lf.k1; }
    // the whole warp polls together, so that it leaves the loop converged
    const int *p = lf.f + (size_t)kn * lf.nj + jn;
    const int target = lf.base + t;
    for (long long it = 0;; ++it) {
        const bool ready = !need || ld_acquire_gpu_int(p) - target >= 0;
        if (__all_sync(0xffffffffu, ready)) break;
        if ((it & 63) == 63 && __any_sync(0xffffffffu, *(volatile int *)&st->error != 0)) return false;
        if (it > polls) {
            if (lane == 0 && atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = -4;
            return false;
        }
    }
    __syncwarp();
    return true;
}

// The eight colour passes of a resident warp (one line of each colour, or none)
// from registers.  No grid barrier: each pass of a line waits only for its four
// neighbours' previous pass (the lines it reads), and publishes its own
// completion after its stores (warp barrier, then lane 0's release store), which
// also tells those neighbours that their next pass may overwrite what it read.
// Every line has its warp resident (a cooperative launch), and a pass waits only
// on passes before it, so every wait ends.  False when a wait gave up.
template <typename T, int L>
__device__ __forceinline__ bool box_passes_regs(const Fields<T> &g, T *phi, const size_t (&rows)[2],
                                                const int (&jl)[2], int kl, const bool (&has)[2], int n, int i0,
                                                size_t sj, size_t sk, const LineFlags &lf, Status *st,
                                                long long polls)
{
    const int lane = threadIdx.x & 31;
    bool ok = true;
    LineRegs<T, L> r0, r1;
    LineFetch<T, L> f0, f1;
    if (has[0]) load_line_regs<T, L>(r0, f0, g, rows[0] + i0, n);
    if (has[1]) load_line_regs<T, L>(r1, f1, g, rows[1] + i0, n);
    if (has[0]) factor_line_regs<T, L>(n, f0.w, f0.e, f0.p, r0.pr, r0.cf, r0.id);
    if (has[1]) factor_line_regs<T, L>(n, f1.w, f1.e, f1.p, r1.pr, r1.cf, r1.id);
    for (int sweep = 0; sweep < 4; ++sweep) {
        const int t0 = 2 * sweep, t1 = t0 + 1;
        if (has[0]) {
            if (ok && t0 > 0) ok = wait_neighbours(lf, jl[0], kl, t0, st, polls);
            if (ok) solve_line_regs<T, L>(phi, rows[0], i0, n, sj, sk, r0);
            __syncwarp();
            if (ok && lane == 0) st_release_gpu_int(lf.f + (size_t)kl * lf.nj + jl[0], lf.base + t0 + 1);
        }
        if (has[1]) {
            if (ok) ok = wait_neighbours(lf, jl[1], kl, t1, st, polls);
            if (ok) solve_line_regs<T, L>(phi, rows[1], i0, n, sj, sk, r1);
            __syncwarp();
            if (ok && lane == 0) st_release_gpu_int(lf.f + (size_t)kl * lf.nj + jl[1], lf.base + t1 + 1);
        }
    }
    return ok;
}

// The eight colour passes of a resident FP32 warp from registers, the lines
// exchanging values through the tagged copy `xc` (solve_line_tagged): version
// tb holds the colour-1 lines' values before the first pass, a line's pass t
// reads version tb + t of its neighbours and writes tb + t + 1.  A line's pass
// t + 1 on a neighbour waits for this line's version tb + t + 1, which it
// writes after reading its own inputs, so no value is overwritten before it is
// read.  False when a wait gave up.
template <int L>
__device__ __forceinline__ bool box_passes_tagged(const Fields<float> &g, float *phi, unsigned long long *xc,
                                                  const size_t (&rows)[2], const int (&jl)[2], int kl,
                                                  const bool (&has)[2], int n, int i0, int j0, int j1, int k0,
                                                  int k1, size_t sj, size_t sk, unsigned tb, Status *st,
                                                  long long polls)
{
    const int a = (threadIdx.x & 31) * L;
    LineRegs<float, L> r0, r1;
    LineFetch<float, L> f0, f1;
    if (has[0]) load_line_regs<float, L>(r0, f0, g, rows[0] + i0, n);
    if (has[1]) load_line_regs<float, L>(r1, f1, g, rows[1] + i0, n);
    if (has[0]) factor_line_regs<float, L>(n, f0.w, f0.e, f0.p, r0.pr, r0.cf, r0.id);
    if (has[1]) factor_line_regs<float, L>(n, f1.w, f1.e, f1.p, r1.pr, r1.cf, r1.id);
    if (has[1]) {
#pragma unroll
        for (int v = 0; v < L; ++v)
            if (a + v < n) {
                const size_t c = rows[1] + i0 + a + v;
                xc[c] = xtag(phi[c], tb);
            }
    }
    const bool t0 = kl + 1 <= k1, b0 = kl - 1 >= k0;  // (both lines lie in plane kl)
    bool ok = true;
    for (int sweep = 0; sweep < 4; ++sweep) {
        const unsigned t = tb + 2u * (unsigned)sweep;
        if (ok && has[0])
            ok = solve_line_tagged<L>(phi, xc, rows[0], i0, n, sj, sk, r0, t0, b0, jl[0] + 1 <= j1, jl[0] - 1 >= j0,
                                      t, sweep == 3, st, polls);
        if (ok && has[1])
            ok = solve_line_tagged<L>(phi, xc, rows[1], i0, n, sj, sk, r1, t0, b0, jl[1] + 1 <= j1, jl[1] - 1 >= j0,
                                      t + 1u, sweep == 3, st, polls);
    }
    return ok;
}

// ---------------------------------------------------------------------------
// Momentum-box line solve of equation ivar (1..3: u, v, w; 4: p') in red-black
// order as one cooperative launch (solveLiquidDomain, CFDSolverManager.cpp:
// 2367-2454): the factorisation of every line, then the four sweeps x two
// colours with a grid barrier between colour passes.  Same arithmetic, in the
// same order, as the multi-launch form (factor_kernel<T, true>, then eight
// sweep_rb_kernel<T, true> launches), so the same bits.  The launch also does
// the work that follows the solve in the multi-launch chain: applyBCs(ivar + 1)
// (its items touch only the next equation's unknown), or for p' correctPressure
// (velocity correction, grid barrier, pressure update) and the momentum
// residual normalisation (one CTA, from the partial sums of the assemblies).  Warp w of the W warps that take part solves
// lines w, w + W, ... of each colour.  When no warp has more than one line of a
// colour ("resident"), a warp's two lines stay in its two shared-memory buffers
// (coefficient rows, factorisation, and a scratch row for the recurrences) for
// all eight passes, and a pass reads only the neighbouring lines' phi, from L2:
// other CTAs wrote them.  Otherwise the factorisation goes to pr, cf, iden and
// every visit stages its line again.  CTAs past the W / warps-per-CTA that the
// box needs return at once and take no part in the barriers.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) mom_box_solve_kernel(Params p, Fields<T> g, int ivar, const double *red, int nb,
                                                            int *flags, unsigned long long *xchg)
{
    pdl_enter();
    T *phi = ivar == 1 ? g.uvel : ivar == 2 ? g.vvel : ivar == 3 ? g.wvel : g.pp;
    extern __shared__ unsigned char smraw[];
    Status *st = g.st;
    if (!st->momentum_active || *(volatile int *)&st->error) return;
    int i0, i1, j0, j1, k0, k1;
    box_of<true>(p, st, i0, i1, j0, j1, k0, k1);
    const int J = j1 - j0 + 1, K = k1 - k0 + 1;
    if (J <= 0 || K <= 0 || i1 < i0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const int half = (J + 1) / 2, nl = half * K;  // line slots of a colour
    const int nact = min((int)gridDim.x, (nl + wpb - 1) / wpb);
    if ((int)blockIdx.x >= nact) return;
    const int W = nact * wpb, gw = blockIdx.x * wpb + warp;
    const bool resident = nl <= W;
    // the barrier generation at the start of the launch: no CTA can advance it
    // before every taking part has arrived at the first barrier
    unsigned gen = *(volatile unsigned *)&st->gbar_gen;
    // the launch's sequence number (advanced by the last CTA to finish the passes)
    const unsigned seq = *(volatile unsigned *)&st->gflag_seq;
    const int nmax = p.nip;
    const size_t slot = (size_t)(S_N + 1) * nmax;  // the staged rows and the scratch row
    T *buf = reinterpret_cast<T *>(smraw) + (size_t)warp * 2 * slot;
    uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<T *>(smraw) + (size_t)wpb * 2 * slot) + warp;
    if (lane == 0) mbar_init(bar);
    __syncwarp();
    uint32_t parity = 0;
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    int ib, ie;
    stage_window<T>(i0, i1, ib, ie);
    const int n = i1 - i0 + 1, o = i0 - ib;
    const uint32_t bytes = (uint32_t)((ie - ib) * sizeof(T));
    // node (0, j, k) of slot q of colour c; false past the box's last row
    auto line_jk = [&](int c, int q, size_t &row, int &j, int &k) {
        const int kk = q / half, r = q - kk * half;
        k = k0 + kk;
        j = j0 + ((c - k - j0) % 2 + 2) % 2 + 2 * r;
        row = cidx(0, j, k, nj, nip);
        return j <= j1;
    };
    auto line_row = [&](int c, int q, size_t &row) {
        int j, k;
        return line_jk(c, q, row, j, k);
    };
    bool ok = true;
    // staging of a line's rows for the factorisation: ap, aw, ae go to the
    // iden, cf, pr rows (lane 0; the caller arms the barrier)
    auto stage_factor_rows = [&](T *sl, size_t row) {
        const T *src[S_N] = {g.at, g.ab, g.an, g.as, g.su, g.aw, g.ae, g.ap};
#pragma unroll
        for (int r = 0; r < S_N; ++r) bulk_load(sl + (size_t)r * nmax, src[r] + row + ib, bytes, bar);
    };
    // the warp factorisation (factor_line_mem) of a staged line, in place
    auto factor_staged = [&](T *sl) {
        T *scf = sl + S_CF * nmax + o, *spr = sl + S_PR * nmax + o, *sid = sl + S_ID * nmax + o;
        factor_line_mem<T>(
            n, [&](int i, T &w, T &e, T &pp) { w = scf[i]; e = spr[i]; pp = sid[i]; },
            [&](int i, T pr, T cf, T id) { spr[i] = pr; scf[i] = cf; sid[i] = id; });
        __syncwarp();
    };
    // lines of up to 64 cells of a resident warp live in registers, loaded and
    // factorised there (box_passes_regs); the rest go through shared memory
    const bool regs = resident && n <= 64;
    // resident: the warp's line of each colour (none past the box's rows)
    size_t rows[2] = {0, 0};
    bool has[2] = {false, false};
    int jl[2] = {0, 0}, kl = 0;  // (slot gw of both colours: the same plane)
    if (resident) {
        for (int c = 0; c < 2; ++c) has[c] = gw < nl && line_jk(c, gw, rows[c], jl[c], kl);
        if (!regs && (has[0] || has[1])) {
            // both lines of the warp staged at once
            if (lane == 0) {
                fence_proxy_async();
                mbar_expect_tx(bar, bytes * S_N * ((has[0] ? 1u : 0u) + (has[1] ? 1u : 0u)));
                for (int c = 0; c < 2; ++c)
                    if (has[c]) stage_factor_rows(buf + c * slot, rows[c]);
            }
            ok = mbar_wait(bar, parity, st, -3);
            parity ^= 1u;
            for (int c = 0; c < 2; ++c)
                if (ok && has[c]) factor_staged(buf + c * slot);
        }
    }
    // otherwise one line at a time through buffer 0, the factorisation kept in
    // pr, cf, iden for the passes to stage again
    for (int c = 0; c < 2 && !resident; ++c)
        for (int q = gw; q < nl && ok; q += W) {
            size_t row;
            if (!line_row(c, q, row)) continue;
            T *sl = buf;
            if (lane == 0) {
                fence_proxy_async();
                mbar_expect_tx(bar, bytes * S_N);
                stage_factor_rows(sl, row);
            }
            ok = mbar_wait(bar, parity, st, -3);
            parity ^= 1u;
            if (!ok) break;
            factor_staged(sl);
            const T *scf = sl + S_CF * nmax + o, *spr = sl + S_PR * nmax + o, *sid = sl + S_ID * nmax + o;
            for (int i = lane; i < n; i += 32) {
                g.pr[row + i0 + i] = spr[i];
                g.cf[row + i0 + i] = scf[i];
                g.iden[row + i0 + i] = sid[i];
            }
            fence_proxy_async_global();  // before the copies that stage these rows again
            __syncwarp();
        }
    // the eight colour passes: lines of up to 64 cells from registers when every
    // warp holds its lines, otherwise from the staged buffers
    if (regs) {
        if constexpr (sizeof(T) == 4) {
            // FP32: values and versions exchanged together
            const unsigned tb = (seq + 1u) * 16u;
            ok = n <= 32 ? box_passes_tagged<1>(g, phi, xchg, rows, jl, kl, has, n, i0, j0, j1, k0, k1, sj, sk, tb, st,
                                                p.wait_polls)
                         : box_passes_tagged<2>(g, phi, xchg, rows, jl, kl, has, n, i0, j0, j1, k0, k1, sj, sk, tb, st,
                                                p.wait_polls);
        } else {
            // FP64 (a value and its version do not fit one access): completion flags
            const LineFlags lf{flags, nj, j0, j1, k0, k1, (int)(seq * 16u)};
            ok = n <= 32 ? box_passes_regs<T, 1>(g, phi, rows, jl, kl, has, n, i0, sj, sk, lf, st, p.wait_polls)
                         : box_passes_regs<T, 2>(g, phi, rows, jl, kl, has, n, i0, sj, sk, lf, st, p.wait_polls);
        }
    }
    for (int pass = 0; pass < 8 && !regs; ++pass) {
        const int c = pass & 1;
        if (pass > 0 && !grid_barrier(&st->gbar_count, &st->gbar_gen, ++gen, (unsigned)nact, st, p.wait_polls, -2))
            return;
        for (int q = gw; q < nl && ok; q += W) {
            size_t row;
            if (!line_row(c, q, row)) continue;
            T *sl = buf + (resident ? c : 0) * slot;
            if (!resident) {
                if (lane == 0) stage_line<T>(g, row, ib, ie, sl, nmax, bar);
                ok = mbar_wait(bar, parity, st, -3);
                parity ^= 1u;
                if (!ok) break;
                __syncwarp();
            }
            solve_staged<T, true>(phi, row, i0, i1, ib, sj, sk, sl, nmax, resident ? S_Q : S_SU);
            __syncwarp();
        }
    }
    // the last CTA through advances the sequence number for the next launch
    __syncthreads();
    if (threadIdx.x == 0 && atom_add_acq_rel_gpu(&st->gflag_done, 1u) == (unsigned)nact - 1) {
        st_relaxed_gpu(&st->gflag_done, 0u);
        st_release_gpu(&st->gflag_seq, seq + 1u);
    }
    // ---- what follows the solve ----
    Box b;
    get_box(st, p, b);
    const int t = blockIdx.x * blockDim.x + threadIdx.x, nt = nact * blockDim.x;
    if (ivar <= 3) {
        int ntop;
        const int nbc = mom_bc_items(p, st, b, ivar + 1, ntop);
        for (int q = t; q < nbc; q += nt) mom_bc_item<T>(p, g, st, b, ivar + 1, q, ntop);
        return;
    }
    if (!grid_barrier(&st->gbar_count, &st->gbar_gen, ++gen, (unsigned)nact, st, p.wait_polls, -2)) return;
    for (int q = t; q < b.n; q += nt) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_velocity_cell<T>(p, g, i, j, k);
    }
    if (!grid_barrier(&st->gbar_count, &st->gbar_gen, ++gen, (unsigned)nact, st, p.wait_polls, -2)) return;
    for (int q = t; q < b.n; q += nt) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_pressure_cell<T>(p, g, i, j, k);
    }
    if (blockIdx.x == 0) {
        __shared__ double scratch[40];
        mom_finalize_body(p, st, red, nb, nb, scratch);
    }
}


// ---------------------------------------------------------------------------
// Small melt-pool boxes (red-black line order).  A melt pool spans a few
// hundred to a few thousand cells; as ~50 grid launches the momentum chain is
// bound by launch and drain latency, not by work.  Here the coefficient
// assembly of each equation stays a grid launch (the arithmetic-heavy part),
// and everything between two assemblies -- the line solve, applyBCs of the next
// equation, cleanVelocities, correctPressure and the residual normalisation --
// runs in one CTA: 9 launches instead of ~50.  For the solve the box's
// coefficients and unknown (with its one-cell halo) are held in shared memory
// while one warp per x-line runs the Thomas recurrences of solveLiquidDomain
// (CFDSolverManager.cpp:2367-2454) for the four sweeps x two colours, as warp
// scans of affine maps over per-lane chunks (the factorisation is one thread
// per line, once per equation).  A box
// larger than the shared memory is solved in place in global memory by the
// same code (views carry the strides).
// ---------------------------------------------------------------------------
constexpr int kMomThreads = 512;

template <typename T> struct V3 {
    T *b;
    int sj;
    long long sk;
    __device__ __forceinline__ T &operator()(int i, int j, int k) const { return b[i + (long long)j * sj + k * sk]; }
};

// Deterministic CTA reductions; the result is valid in thread 0.
__device__ __forceinline__ double cta_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    return r;
}
__device__ __forceinline__ double cta_max(double v, double *sh)
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = -INFINITY;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    return r;
}

constexpr int kShortG = 8, kShortL = 3;

// One line of a box held in shared memory, solved by a group of G = 8 lanes: each
// lane runs its chunk a..e-1, and segmented shuffle scans of the affine maps
// chain the chunks (x -> cf x + e forward, x -> pr x + qr backward).  Every lane
// of the warp calls it (shuffles take all 32 lanes); a group without a line
// (act false) carries identity maps.
struct BoxLine {
    int NI, sub, a, e;
};
template <typename T>
__device__ __forceinline__ void group_line_shared(const V3<T> &at, const V3<T> &ab, const V3<T> &an,
                                                  const V3<T> &as, const V3<T> &su, const V3<T> &pr,
                                                  const V3<T> &cf, const V3<T> &id, const V3<T> &qr,
                                                  const V3<T> &ph, const BoxLine &bl, int jj, int kk, bool act)
{
    constexpr int G = kShortG;
    const int NI = bl.NI, sub = bl.sub, a = bl.a, e = bl.e;
        T A = T(1), B = T(0);
        if (act)
            for (int ii = a; ii < e; ++ii) {
                const T d = at(ii, jj, kk) * ph(ii, jj, kk + 1) + ab(ii, jj, kk) * ph(ii, jj, kk - 1) +
                            an(ii, jj, kk) * ph(ii, jj + 1, kk) + as(ii, jj, kk) * ph(ii, jj - 1, kk) +
                            su(ii, jj, kk);
                const T ev = d * id(ii, jj, kk), c = cf(ii, jj, kk);
                qr(ii, jj, kk) = ev;
                B = c * B + ev;
                A = c * A;
            }
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const T A2 = __shfl_up_sync(0xffffffffu, A, o, G), B2 = __shfl_up_sync(0xffffffffu, B, o, G);
            if (sub >= o) { B = A * B2 + B; A = A * A2; }
        }
        T Ae = __shfl_up_sync(0xffffffffu, A, 1, G), Be = __shfl_up_sync(0xffffffffu, B, 1, G);
        if (sub == 0) { Ae = T(1); Be = T(0); }
        A = T(1);
        B = T(0);
        if (act) {
            T q = Ae * ph(-1, jj, kk) + Be;
            for (int ii = a; ii < e; ++ii) {
                q = cf(ii, jj, kk) * q + qr(ii, jj, kk);
                qr(ii, jj, kk) = q;
            }
            for (int ii = e - 1; ii >= a; --ii) {
                const T pv = pr(ii, jj, kk);
                B = pv * B + qr(ii, jj, kk);
                A = pv * A;
            }
        }
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const T A2 = __shfl_down_sync(0xffffffffu, A, o, G), B2 = __shfl_down_sync(0xffffffffu, B, o, G);
            if (sub + o < G) { B = A * B2 + B; A = A * A2; }
        }
        Ae = __shfl_down_sync(0xffffffffu, A, 1, G);
        Be = __shfl_down_sync(0xffffffffu, B, 1, G);
        if (sub == G - 1) { Ae = T(1); Be = T(0); }
        if (act) {
            T x = Ae * ph(NI, jj, kk) + Be;
            for (int ii = e - 1; ii >= a; --ii) {
                x = pr(ii, jj, kk) * x + qr(ii, jj, kk);
                ph(ii, jj, kk) = x;
            }
        }
}

// The four sweeps of an FP32 box held in shared memory whose lines are short (at
// most 3 cells a lane in groups of 8 lanes): each lane keeps its cells'
// coefficients (at ab an as su) and factorisation (cf id pr) of its group's first
// line of each colour in registers across the sweeps, so a pass reads only the
// neighbour values of phi; a group's second line of a colour, where the box has
// more lines than groups, is solved from shared memory (group_line_shared).  The
// recurrences and their order of operations are those of the shared-memory path.
template <typename T, bool TWO, class Between>  // TWO: some groups have a second line of a colour
__device__ __forceinline__ void sweep_short_regs(const Box &b, int NI, int NJ, int NK, const T *sm, int ncell,
                                                 T *ph0, int HI, int HJ, const V3<T> &at, const V3<T> &ab,
                                                 const V3<T> &an, const V3<T> &as, const V3<T> &su,
                                                 const V3<T> &pr, const V3<T> &cf, const V3<T> &id,
                                                 const V3<T> &qr, const V3<T> &ph, Between &between)
{
    constexpr int G = kShortG, LM = kShortL;
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = lane & (G - 1), gid = warp * (32 / G) + lane / G;
    const int L = (NI + G - 1) / G;
    const int a = min(sub * L, NI), n = min(a + L, NI) - a;  // this lane's cells a .. a+n-1
    const int half = (NJ + 1) / 2, nline = half * NK, HIJ = HI * HJ;
    const int ngroups = (int)(blockDim.x >> 5) * (32 / G);
    T rat[2][LM], rab[2][LM], ran[2][LM], ras[2][LM], rsu[2][LM], rpr[2][LM], rcf[2][LM], rid[2][LM];
    int oh[2];
    bool act[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        int kk = 0, jj = 0;
        bool ac = gid < nline;
        if (ac) {
            kk = gid / half;
            const int r = gid - kk * half, k = b.k0 + kk;
            jj = ((c - k - b.j0) % 2 + 2) % 2 + 2 * r;
            ac = jj < NJ;
        }
        act[c] = ac;
        oh[c] = jj * HI + kk * HIJ;
        const int o = a + jj * NI + kk * NI * NJ;
#pragma unroll
        for (int v = 0; v < LM; ++v) {
            const bool in = ac && v < n;
            rat[c][v] = in ? sm[o + v] : T(0);
            rab[c][v] = in ? sm[ncell + o + v] : T(0);
            ran[c][v] = in ? sm[2 * ncell + o + v] : T(0);
            ras[c][v] = in ? sm[3 * ncell + o + v] : T(0);
            rsu[c][v] = in ? sm[4 * ncell + o + v] : T(0);
            rpr[c][v] = in ? sm[5 * ncell + o + v] : T(0);
            rcf[c][v] = in ? sm[6 * ncell + o + v] : T(0);
            rid[c][v] = in ? sm[7 * ncell + o + v] : T(0);
        }
    }
    for (int sweep = 0; sweep < 4; ++sweep) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int h = oh[c] + a;
            T qv[LM];
            T A = T(1), B = T(0);
#pragma unroll
            for (int v = 0; v < LM; ++v) {
                qv[v] = T(0);
                if (act[c] && v < n) {
                    const T d = rat[c][v] * ph0[h + v + HIJ] + rab[c][v] * ph0[h + v - HIJ] +
                                ran[c][v] * ph0[h + v + HI] + ras[c][v] * ph0[h + v - HI] + rsu[c][v];
                    const T ev = d * rid[c][v], cc = rcf[c][v];
                    qv[v] = ev;
                    B = cc * B + ev;
                    A = cc * A;
                }
            }
#pragma unroll
            for (int o = 1; o < G; o <<= 1) {
                const T A2 = __shfl_up_sync(full, A, o, G), B2 = __shfl_up_sync(full, B, o, G);
                if (sub >= o) { B = A * B2 + B; A = A * A2; }
            }
            T Ae = __shfl_up_sync(full, A, 1, G), Be = __shfl_up_sync(full, B, 1, G);
            if (sub == 0) { Ae = T(1); Be = T(0); }
            A = T(1);
            B = T(0);
            if (act[c]) {
                T q = Ae * ph0[oh[c] - 1] + Be;
#pragma unroll
                for (int v = 0; v < LM; ++v)
                    if (v < n) {
                        q = rcf[c][v] * q + qv[v];
                        qv[v] = q;
                    }
#pragma unroll
                for (int v = LM - 1; v >= 0; --v)
                    if (v < n) {
                        const T pv = rpr[c][v];
                        B = pv * B + qv[v];
                        A = pv * A;
                    }
            }
#pragma unroll
            for (int o = 1; o < G; o <<= 1) {
                const T A2 = __shfl_down_sync(full, A, o, G), B2 = __shfl_down_sync(full, B, o, G);
                if (sub + o < G) { B = A * B2 + B; A = A * A2; }
            }
            Ae = __shfl_down_sync(full, A, 1, G);
            Be = __shfl_down_sync(full, B, 1, G);
            if (sub == G - 1) { Ae = T(1); Be = T(0); }
            if (act[c]) {
                T x = Ae * ph0[oh[c] + NI] + Be;
#pragma unroll
                for (int v = LM - 1; v >= 0; --v)
                    if (v < n) {
                        x = rpr[c][v] * x + qv[v];
                        ph0[h + v] = x;
                    }
            }
            if (TWO) {  // the CTA's groups all take part
                const int l = gid + ngroups;
                int kk = 0, jj = 0;
                bool ac = l < nline;
                if (ac) {
                    kk = l / half;
                    const int r = l - kk * half, k = b.k0 + kk;
                    jj = ((c - k - b.j0) % 2 + 2) % 2 + 2 * r;
                    ac = jj < NJ;
                }
                __syncwarp();
                group_line_shared<T>(at, ab, an, as, su, pr, cf, id, qr, ph, BoxLine{NI, sub, a, a + n}, jj, kk, ac);
            }
            between(sweep, c);
        }
    }
}

// Shared-memory elements a slab of nj rows of a box needs: nine arrays of its
// cells and phi with a one-cell halo.
__host__ __device__ __forceinline__ long long slab_elems(int ni, int nj, int nk)
{
    return 9ll * ni * nj * nk + (long long)(ni + 2) * (nj + 2) * (nk + 2);
}

// Rows [jl0, jl0 + njl) of a box: what one CTA of a cluster holds (the whole box
// on the one-CTA path).
struct Slab {
    int jl0, njl;
};
// Rows of the slab of CTA `rank` of `nc` over a box of nj rows.
__host__ __device__ __forceinline__ Slab slab_of(int nj, int rank, int nc)
{
    const int a = (int)((long long)nj * rank / nc), e = (int)((long long)nj * (rank + 1) / nc);
    return Slab{a, e - a};
}

// solveLiquidDomain over the lines of one slab of the box: load (fits: into
// shared memory, else views of the global arrays), factorise, and the four
// red-black sweeps; `between(sweep, colour)` runs after every colour pass (a CTA
// barrier on the one-CTA path; on a cluster the cluster barrier and the exchange
// of the rows next to the slab).  Every thread of the CTA calls it, also for an
// empty slab.
// REGS: the FP32 register-resident sweep may be used (the one-CTA path; a cluster's
// slabs take the shared-memory sweep, which keeps the kernel within its registers).
template <typename T, bool REGS, class Between>
__device__ void solve_box_slab(const Params &p, const Fields<T> &g, const Box &bx, const Slab &sl, T *phi,
                               T *sm, bool fits, T *scratch, Between &between)
{
    // the slab as a box of its own: its first row fixes the colour parity
    Box b = bx;
    b.j0 = bx.j0 + sl.jl0;
    b.nj_ = sl.njl;
    b.j1 = b.j0 + sl.njl - 1;
    const int NI = b.ni_, NJ = b.nj_, NK = b.k1 - b.k0 + 1;
    const int ncell = NI * NJ * NK;
    const int HI = NI + 2, HJ = NJ + 2;
    const int nhalo = HI * HJ * (NK + 2);
    const int gsj = p.nip;
    const long long gsk = (long long)p.nj * p.nip;
    const size_t g0 = cidx(b.i0, b.j0, b.k0, p.nj, p.nip);
    const int tid = threadIdx.x, nth = blockDim.x;
    V3<T> at, ab, an, as, su, pr, cf, id, qr, ph;
    const T *ae_src, *aw_src, *ap_src;
    if (fits) {
        // array f of the box: cell (ii, jj, kk) at f * ncell + ii + NI (jj + NJ kk)
        auto box_array = [&](long long f) { return V3<T>{sm + f * ncell, NI, (long long)NI * NJ}; };
        at = box_array(0); ab = box_array(1); an = box_array(2); as = box_array(3);
        su = box_array(4); pr = box_array(5); cf = box_array(6); id = box_array(7);
        qr = box_array(8);
        ph = {sm + 9ll * ncell + 1 + HI + (long long)HI * HJ, HI, (long long)HI * HJ};
        // every load of a batch is issued before its shared-memory stores; the
        // arrays at ab an as su pr(=ae) cf(=aw) id(=ap) follow one another, cell
        // (ii, jj, kk) at q = ii + NI (jj + NJ kk), and the halo of phi after them
        constexpr int kBc = 2, kBh = 4;
        for (int q0 = tid; q0 < ncell; q0 += kBc * nth) {
            T v[kBc][8];
#pragma unroll
            for (int u = 0; u < kBc; ++u) {
                const int q = q0 + u * nth;
                if (q < ncell) {
                    const int ii = q % NI, r = q / NI, jj = r % NJ, kk = r / NJ;
                    const size_t c = g0 + ii + (size_t)jj * gsj + (size_t)kk * gsk;
                    v[u][0] = g.at[c]; v[u][1] = g.ab[c]; v[u][2] = g.an[c]; v[u][3] = g.as[c];
                    v[u][4] = g.su[c]; v[u][5] = g.ae[c]; v[u][6] = g.aw[c]; v[u][7] = g.ap[c];
                }
            }
#pragma unroll
            for (int u = 0; u < kBc; ++u) {
                const int q = q0 + u * nth;
                if (q < ncell) {
#pragma unroll
                    for (int f = 0; f < 8; ++f) sm[(size_t)f * ncell + q] = v[u][f];
                }
            }
        }
        for (int q0 = tid; NJ > 0 && q0 < nhalo; q0 += kBh * nth) {  // (an empty slab loads nothing)
            T v[kBh];
#pragma unroll
            for (int u = 0; u < kBh; ++u) {
                const int q = q0 + u * nth;
                if (q < nhalo) {
                    const int ii = q % HI, r = q / HI, jj = r % HJ, kk = r / HJ;
                    v[u] = phi[(long long)g0 + (ii - 1) + (long long)(jj - 1) * gsj + (kk - 1) * gsk];
                }
            }
#pragma unroll
            for (int u = 0; u < kBh; ++u) {
                const int q = q0 + u * nth;
                if (q < nhalo) sm[9ll * ncell + q] = v[u];
            }
        }
        ae_src = nullptr; aw_src = nullptr; ap_src = nullptr;
        __syncthreads();
    } else {
        at = {g.at + g0, gsj, gsk}; ab = {g.ab + g0, gsj, gsk};
        an = {g.an + g0, gsj, gsk}; as = {g.as + g0, gsj, gsk};
        su = {g.su + g0, gsj, gsk}; pr = {g.pr + g0, gsj, gsk};
        cf = {g.cf + g0, gsj, gsk}; id = {g.iden + g0, gsj, gsk};
        qr = {scratch + g0, gsj, gsk};
        ph = {phi + g0, gsj, gsk};
        ae_src = g.ae + g0; aw_src = g.aw + g0; ap_src = g.ap + g0;
    }
    // factorisation, one thread per line (pr = ae/den, cf = aw/den, id = 1/den),
    // with solveLiquidDomain's guard on |den| (:2438-2439)
    for (int l = tid; l < NJ * NK; l += nth) {
        const int jj = l % NJ, kk = l / NJ;
        T prv = T(0);
        for (int ii = 0; ii < NI; ++ii) {
            const long long o = ii + (long long)jj * gsj + kk * gsk;
            const T apv = fits ? id(ii, jj, kk) : ap_src[o];
            const T aev = fits ? pr(ii, jj, kk) : ae_src[o];
            const T awv = fits ? cf(ii, jj, kk) : aw_src[o];
            T den = apv - awv * prv;
            if (fabs(den) <= T(1e-12)) den += T(kSmall);
            const T iv = T(1) / den;
            const T pv = aev * iv;
            pr(ii, jj, kk) = pv;
            cf(ii, jj, kk) = awv * iv;
            id(ii, jj, kk) = iv;
            prv = pv;
        }
    }
    __syncthreads();
    // 4 sweeps x 2 colours; a line of one colour reads only rows of the other.
    // Short lines (the usual melt-pool box): one thread per line, sequential
    // recurrences over per-line base pointers.  Long lines: one warp per line,
    // warp scans of affine maps over per-lane chunks.
    const int half = (NJ + 1) / 2;
    // (FP64 registers for both colours would spill: FP64 keeps the shared-memory path)
    bool regs = false;
    if constexpr (REGS && sizeof(T) == 4)
        regs = fits && NI <= kShortG * kShortL && half * NK <= 2 * (nth >> 5) * (32 / kShortG);
    if (regs) {
        if constexpr (REGS && sizeof(T) == 4) {
            if (half * NK <= (nth >> 5) * (32 / kShortG))
                sweep_short_regs<T, false>(b, NI, NJ, NK, sm, ncell, &ph(0, 0, 0), HI, HJ, at, ab, an, as, su, pr,
                                           cf, id, qr, ph, between);
            else
                sweep_short_regs<T, true>(b, NI, NJ, NK, sm, ncell, &ph(0, 0, 0), HI, HJ, at, ab, an, as, su, pr,
                                          cf, id, qr, ph, between);
        }
    } else if (NI <= 48) {
        // Short lines (the usual melt-pool box): a group of G lanes per line, each
        // lane a chunk of at most 6 cells, chained by segmented shuffle scans of
        // the affine maps (x -> cf x + e forward, x -> pr x + qr backward).  The
        // loop over lines advances a warp's four groups together, so that every
        // shuffle has all 32 lanes; a group without a line carries identity maps.
        constexpr int G = 8;
        const int lane = tid & 31, warp = tid >> 5, nwarp = nth >> 5;
        const int sub = lane & (G - 1), gw = lane / G;  // lane in its group, group in its warp
        const int L = (NI + G - 1) / G;
        const int a = min(sub * L, NI), e = min(a + L, NI);
        const int nline = half * NK;
        for (int sweep = 0; sweep < 4; ++sweep)
            for (int color = 0; color < 2; ++color) {
                for (int l0 = warp * (32 / G); l0 < nline; l0 += nwarp * (32 / G)) {
                    const int l = l0 + gw;
                    int kk = 0, jj = 0;
                    bool act = l < nline;
                    if (act) {
                        kk = l / half;
                        const int r = l - kk * half;
                        const int k = b.k0 + kk;
                        const int jpar = ((color - k - b.j0) % 2 + 2) % 2;
                        jj = jpar + 2 * r;
                        act = jj < NJ;
                    }
                    group_line_shared<T>(at, ab, an, as, su, pr, cf, id, qr, ph, BoxLine{NI, sub, a, e}, jj, kk, act);
                    __syncwarp();
                }
                between(sweep, color);
            }
    } else {
        const int lane = tid & 31, warp = tid >> 5, nwarp = nth >> 5;
        const int L = (NI + 31) >> 5;
        const int a = min(lane * L, NI), e = min(a + L, NI);
        for (int sweep = 0; sweep < 4; ++sweep)
            for (int color = 0; color < 2; ++color) {
                for (int l = warp; l < half * NK; l += nwarp) {
                    const int kk = l / half, r = l - kk * half;
                    const int k = b.k0 + kk;
                    const int jpar = ((color - k - b.j0) % 2 + 2) % 2;
                    const int jj = jpar + 2 * r;
                    if (jj >= NJ) continue;  // warp-uniform
                    // right-hand side over this lane's chunk, and its forward map
                    T A = T(1), B = T(0);
                    for (int ii = a; ii < e; ++ii) {
                        const T d = at(ii, jj, kk) * ph(ii, jj, kk + 1) + ab(ii, jj, kk) * ph(ii, jj, kk - 1) +
                                    an(ii, jj, kk) * ph(ii, jj + 1, kk) + as(ii, jj, kk) * ph(ii, jj - 1, kk) +
                                    su(ii, jj, kk);
                        const T ev = d * id(ii, jj, kk), c = cf(ii, jj, kk);
                        qr(ii, jj, kk) = ev;
                        B = c * B + ev;
                        A = c * A;
                    }
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const T A2 = __shfl_up_sync(0xffffffffu, A, o), B2 = __shfl_up_sync(0xffffffffu, B, o);
                        if (lane >= o) { B = A * B2 + B; A = A * A2; }
                    }
                    T Ae = __shfl_up_sync(0xffffffffu, A, 1), Be = __shfl_up_sync(0xffffffffu, B, 1);
                    if (lane == 0) { Ae = T(1); Be = T(0); }
                    T q = Ae * ph(-1, jj, kk) + Be;
                    for (int ii = a; ii < e; ++ii) {
                        q = cf(ii, jj, kk) * q + qr(ii, jj, kk);
                        qr(ii, jj, kk) = q;
                    }
                    A = T(1);
                    B = T(0);
                    for (int ii = e - 1; ii >= a; --ii) {
                        const T pv = pr(ii, jj, kk);
                        B = pv * B + qr(ii, jj, kk);
                        A = pv * A;
                    }
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const T A2 = __shfl_down_sync(0xffffffffu, A, o), B2 = __shfl_down_sync(0xffffffffu, B, o);
                        if (lane + o < 32) { B = A * B2 + B; A = A * A2; }
                    }
                    Ae = __shfl_down_sync(0xffffffffu, A, 1);
                    Be = __shfl_down_sync(0xffffffffu, B, 1);
                    if (lane == 31) { Ae = T(1); Be = T(0); }
                    T x = Ae * ph(NI, jj, kk) + Be;
                    for (int ii = e - 1; ii >= a; --ii) {
                        x = pr(ii, jj, kk) * x + qr(ii, jj, kk);
                        ph(ii, jj, kk) = x;
                    }
                    __syncwarp();
                }
                between(sweep, color);
            }
    }
    if (fits) {
        for (int q = tid; q < ncell; q += nth) {
            const int ii = q % NI, r = q / NI, jj = r % NJ, kk = r / NJ;
            phi[g0 + ii + (size_t)jj * gsj + (size_t)kk * gsk] = ph(ii, jj, kk);
        }
        __syncthreads();
    }
}

// The whole box in one CTA (shared memory when it fits, else in place in global
// memory), a CTA barrier after every colour pass.
template <typename T>
__device__ void solve_box_small(const Params &p, const Fields<T> &g, const Box &b, T *phi, T *sm,
                                int smem_elems, T *scratch)
{
    const int NK = b.k1 - b.k0 + 1;
    const bool fits = slab_elems(b.ni_, b.nj_, NK) <= (long long)smem_elems;
    auto bar = [](int, int) { __syncthreads(); };
    solve_box_slab<T, true>(p, g, b, Slab{0, b.nj_}, phi, sm, fits, scratch, bar);
}

// The box over the CTAs of a cluster, one slab of rows each.  With the slabs in
// shared memory, after a colour pass each CTA copies the lines of that colour in
// the rows either side of its slab from the CTAs that own them (distributed
// shared memory): the next pass, of the other colour, reads exactly those.
// Without, every CTA works in place in global memory and the cluster barrier
// orders the passes.  Every pass ends at a cluster barrier, the last one too, so
// that no CTA leaves while another may still read its shared memory.
// After each colour pass of a cluster's slabs: the cluster barrier and, with the
// slabs in shared memory, the copy of the lines of that colour in the rows either
// side of this CTA's slab from the CTAs that own them (values, not references, so
// that the line loops keep their registers).
template <typename T>
struct ClusterBetween {
    T *sm, *my_ph;
    int NI, NJ, NK, HI, nc, j0, k0;
    Slab sl;
    bool fits;
    __device__ int owner(int jg) const
    {
        int o = 0;
        for (int r = 1; r < nc; ++r)
            if (slab_of(NJ, r, nc).jl0 <= jg) o = r;
        return o;
    }
    __device__ void operator()(int sweep, int color) const
    {
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        if (!fits || sl.njl == 0 || (sweep == 3 && color == 1)) return;
        for (int side = 0; side < 2; ++side) {
            const int jg = side == 0 ? sl.jl0 - 1 : sl.jl0 + sl.njl;  // box row next to the slab
            if (jg < 0 || jg >= NJ) continue;
            const int o = owner(jg);
            const Slab os = slab_of(NJ, o, nc);
            // phi of o's slab, with its halo, after its nine cell arrays
            const T *rph = cl.map_shared_rank(sm, (unsigned)o) + 9ll * NI * os.njl * NK;
            const int rj = jg - os.jl0 + 1, lj = side == 0 ? 0 : sl.njl + 1;  // halo row indices
            const long long rsk = (long long)HI * (os.njl + 2), lsk = (long long)HI * (sl.njl + 2);
            const int j = j0 + jg;
            for (int q = threadIdx.x; q < NI * NK; q += blockDim.x) {
                const int ii = q % NI, kk = q / NI;
                if (((j + k0 + kk) & 1) != color) continue;  // a line of the colour just solved
                my_ph[(ii + 1) + lj * HI + (kk + 1) * lsk] = rph[(ii + 1) + rj * HI + (kk + 1) * rsk];
            }
        }
        __syncthreads();
    }
};

// The box over the CTAs of a cluster, one slab of rows each.  With the slabs in
// shared memory, after a colour pass each CTA copies the lines of that colour in
// the rows either side of its slab from the CTAs that own them (distributed
// shared memory): the next pass, of the other colour, reads exactly those.
// Without, every CTA works in place in global memory and the cluster barrier
// orders the passes.  Every pass ends at a cluster barrier, the last one too, so
// that no CTA leaves while another may still read its shared memory.
template <typename T>
__device__ void solve_box_cluster(const Params &p, const Fields<T> &g, const Box &b, T *phi, T *sm,
                                  int smem_elems, T *scratch, int nc, int rank)
{
    const int NI = b.ni_, NJ = b.nj_, NK = b.k1 - b.k0 + 1;
    ClusterBetween<T> bw;
    bw.sl = slab_of(NJ, rank, nc);
    // the same decision in every CTA: the largest slab has ceil(NJ / nc) rows
    bw.fits = slab_elems(NI, (NJ + nc - 1) / nc, NK) <= (long long)smem_elems;
    bw.sm = sm;
    bw.my_ph = sm + 9ll * NI * bw.sl.njl * NK;
    bw.NI = NI; bw.NJ = NJ; bw.NK = NK; bw.HI = NI + 2; bw.nc = nc; bw.j0 = b.j0; bw.k0 = b.k0;
    solve_box_slab<T, false>(p, g, b, bw.sl, phi, sm, bw.fits, scratch, bw);
}

// Phase helpers of the one-CTA and cluster kernels.  `t`/`nt`: this thread's
// index and the thread count over which box items are spread.
template <typename T>
__device__ __forceinline__ double box_bc(const Params &p, const Fields<T> &g, Status *st, const Box &b, int ivar,
                                         int t, int nt)
{
    int ntop;
    const int nbc = mom_bc_items(p, st, b, ivar, ntop);
    double um = 0.0;
    for (int q = t; q < nbc; q += nt) um = maxd(um, mom_bc_item<T>(p, g, st, b, ivar, q, ntop));
    return um;
}
template <typename T>
__device__ __forceinline__ void small_bc(const Params &p, const Fields<T> &g, Status *st, const Box &b,
                                         int ivar, double *red_umax, double *sh)
{
    double um = box_bc<T>(p, g, st, b, ivar, threadIdx.x, blockDim.x);
    if (ivar == 1) {
        um = cta_max(um, sh);
        if (threadIdx.x == 0) red_umax[R_UMAX] = um;  // entry 0 of the umax region
    }
}

// Whether a box is spread over the cluster: it does not fit one CTA's shared
// memory.  Read from the status block, so the same in every CTA.
__device__ __forceinline__ bool spread(const Box &b, int smem_elems)
{
    return slab_elems(b.ni_, b.nj_, b.k1 - b.k0 + 1) > (long long)smem_elems;
}

// ---- one CTA (boxes that fit its shared memory, and with `wide` 0 every box; a
// no-op for the boxes a cluster takes) ---------------------------------------------------
// cleanVelocities + applyBCs(1).
template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_small_pre_kernel(Params p, Fields<T> g, double *red_umax, int smem_elems, int wide)
{
    pdl_enter();
    __shared__ double sh[32];
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || (wide && spread(b, smem_elems))) return;
    for (int q = threadIdx.x; q < b.n; q += blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        clean_cell<T>(p, g, i, j, k);
    }
    __syncthreads();
    small_bc<T>(p, g, st, b, 1, red_umax, sh);
}

// Line solve of equation ivar (1..3) on the box, then applyBCs(ivar + 1).
template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_small_mid_kernel(Params p, Fields<T> g, int ivar, T *scratch, int smem_elems, double *red_umax, int wide)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double sh[32];
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || (wide && spread(b, smem_elems))) return;
    T *phi = ivar == 1 ? g.uvel : ivar == 2 ? g.vvel : g.wvel;
    solve_box_small<T>(p, g, b, phi, reinterpret_cast<T *>(smraw), smem_elems, scratch);
    small_bc<T>(p, g, st, b, ivar + 1, red_umax, sh);
}

// Line solve of p', correctPressure and the residual normalisation.
template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_small_post_kernel(Params p, Fields<T> g, T *scratch, int smem_elems, const double *red, int nb, int wide)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double scratch_r[40];
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || (wide && spread(b, smem_elems))) return;
    solve_box_small<T>(p, g, b, g.pp, reinterpret_cast<T *>(smraw), smem_elems, scratch);
    for (int q = threadIdx.x; q < b.n; q += blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_velocity_cell<T>(p, g, i, j, k);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < b.n; q += blockDim.x) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_pressure_cell<T>(p, g, i, j, k);
    }
    __syncthreads();
    mom_finalize_body(p, st, red, nb, 1, scratch_r);
}

// ---- one cluster of CTAs (boxes past one CTA's shared memory; a no-op otherwise) ------
// The same three steps with the box items spread over all threads of the cluster
// and the cluster barrier where one step reads what another CTA wrote.
template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_cluster_pre_kernel(Params p, Fields<T> g, double *red_umax, int smem_elems)
{
    pdl_enter();
    __shared__ double sh[32];
    __shared__ double cmax;
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || !spread(b, smem_elems)) return;
    cg::cluster_group cl = cg::this_cluster();
    const int nc = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    const int t = rank * blockDim.x + threadIdx.x, nt = nc * blockDim.x;
    for (int q = t; q < b.n; q += nt) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        clean_cell<T>(p, g, i, j, k);
    }
    cl.sync();
    double um = cta_max(box_bc<T>(p, g, st, b, 1, t, nt), sh);
    if (threadIdx.x == 0) cmax = um;
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) {
        double m = cmax;
        for (int r = 1; r < nc; ++r) m = maxd(m, *cl.map_shared_rank(&cmax, (unsigned)r));
        red_umax[R_UMAX] = m;
    }
    cl.sync();  // every CTA's maximum is read before any CTA leaves
}

template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_cluster_mid_kernel(Params p, Fields<T> g, int ivar, T *scratch, int smem_elems)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || !spread(b, smem_elems)) return;
    cg::cluster_group cl = cg::this_cluster();
    const int nc = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    T *phi = ivar == 1 ? g.uvel : ivar == 2 ? g.vvel : g.wvel;
    solve_box_cluster<T>(p, g, b, phi, reinterpret_cast<T *>(smraw), smem_elems, scratch, nc, rank);
    box_bc<T>(p, g, st, b, ivar + 1, rank * blockDim.x + threadIdx.x, nc * blockDim.x);
}

template <typename T>
__global__ void __launch_bounds__(kMomThreads, 1)
mom_cluster_post_kernel(Params p, Fields<T> g, T *scratch, int smem_elems, const double *red, int nb)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double scratch_r[40];
    Status *st = g.st;
    Box b;
    if (!get_box(st, p, b) || !spread(b, smem_elems)) return;
    cg::cluster_group cl = cg::this_cluster();
    const int nc = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    solve_box_cluster<T>(p, g, b, g.pp, reinterpret_cast<T *>(smraw), smem_elems, scratch, nc, rank);
    const int t = rank * blockDim.x + threadIdx.x, nt = nc * blockDim.x;
    cl.sync();  // p' of the whole box is in global memory
    for (int q = t; q < b.n; q += nt) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_velocity_cell<T>(p, g, i, j, k);
    }
    cl.sync();
    for (int q = t; q < b.n; q += nt) {
        int i, j, k;
        box_cell(b, q, i, j, k);
        correct_pressure_cell<T>(p, g, i, j, k);
    }
    if (rank == 0) {
        __syncthreads();
        mom_finalize_body(p, st, red, nb, 1, scratch_r);
    }
}

// Largest box (cells) the one-CTA / cluster path takes: one CTA's shared memory
// holds about smem/12 cells of a thin box; a cluster of nc CTAs about nc/2 times
// as many (slabs of whole rows, uneven by up to one row, each with two halo rows).
template <typename T> int mom_small_capacity(const Inst<T> &I)
{
    const int one = (int)(I.mom_small_smem / sizeof(T) / 12);
    return I.mom_cluster > 1 ? one * I.mom_cluster / 2 : one;
}

// Default cluster size of the box solve (the options may pin another): none.  On
// the 400 x 200 x 100 deck's steady box (about 5800 cells) the cluster path took
// 0.246 / 0.256 / 0.299 ms per outer iteration with 4 / 8 / 16 CTAs against 0.211
// for the multi-kernel path: a cluster launch of the line solve spends its time at
// the barriers between colour passes (27 % issue active, 51 us a launch).
constexpr int kDefaultCluster = 1;

// Cluster size of the small-box kernels: the largest the device schedules with
// this shared memory, at most 16.
template <typename T> static int max_cluster(size_t smem)
{
    cudaFuncSetAttribute(mom_cluster_mid_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(mom_cluster_post_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(mom_cluster_pre_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int best = 1;
    for (int nc : {16, 8, 4, 2}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = nc;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(nc);
        cfg.blockDim = dim3(kMomThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (void *)mom_cluster_mid_kernel<T>, &cfg) == cudaSuccess && n > 0) {
            best = nc;
            break;
        }
        cudaGetLastError();
    }
    return best;
}

template <typename T> void setup_mom_small(Inst<T> &I)
{
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t bytes = std::min<size_t>((size_t)std::max(optin, 48 * 1024) - 1024, 200 * 1024);
    bytes = bytes / 16 * 16;
    cudaFuncSetAttribute(mom_small_mid_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(mom_small_post_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(mom_cluster_mid_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(mom_cluster_post_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    I.mom_small_smem = bytes;
    const int most = max_cluster<T>(bytes);
    I.mom_cluster = I.mom_cluster > 0 ? std::min(I.mom_cluster, most) : std::min(kDefaultCluster, most);
}

// A launch of nc CTAs forming one cluster (with `pdl`, also programmatic stream
// serialisation, as launch_k).
template <typename... K, typename... A>
static void launch_cluster(bool pdl, void (*kern)(K...), int nc, size_t smem, cudaStream_t s, A... args)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = nc;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3(nc);
    cfg.blockDim = dim3(kMomThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 2 : 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<K>(args)...);
}

// The momentum box's red-black line solve of equation ivar as one cooperative
// launch (mom_box_solve_kernel).
template <typename T> static void launch_box_solve(Inst<T> &I, int ivar)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.gridDim = dim3(I.box_grid);
    cfg.blockDim = dim3(32 * I.box_warps);
    cfg.dynamicSmemBytes = I.box_smem;
    cfg.stream = I.stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, mom_box_solve_kernel<T>, I.p, I.g, ivar, (const double *)I.red_mom, I.nb_mom,
                       I.flags_mom, I.xchg);
}
// Launch shape of mom_box_solve_kernel: the most warps per CTA (4, 2 or 1) whose
// buffers (two lines of 8 staged rows and a scratch row each, one mbarrier) fit
// 200 KiB, and as many CTAs as the box's largest colour needs, at most as many as
// are resident at once (a cooperative launch).  box_grid 0: none fits, or not
// enabled (exact order; the serial launch form), and the chain keeps the
// multi-launch line solve.
template <typename T> void setup_box_solve(Inst<T> &I, bool enable)
{
    I.box_grid = 0;
    if (!enable || I.order != AMCFD_ORDER_REDBLACK) return;
    for (int w = 4; w >= 1; w /= 2) {
        const size_t need = (size_t)w * (2 * (S_N + 1) * (size_t)I.p.nip * sizeof(T) + 8);
        if (need > 200 * 1024) continue;
        if (raise_smem_limit((const void *)mom_box_solve_kernel<T>, need) != cudaSuccess) return;
        int bps = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, mom_box_solve_kernel<T>, 32 * w, need);
        if (bps < 1) return;
        const int lines = ((I.p.nj - 2 + 1) / 2) * (I.p.nk - 2);  // most lines of a colour
        I.box_warps = w;
        I.box_smem = need;
        I.box_grid = std::max(1, std::min((lines + w - 1) / w, bps * I.sm_count));
        return;
    }
}

// ---------------------------------------------------------------------------
// launcher: the whole momentum chain of one outer iteration
// ---------------------------------------------------------------------------
template <typename T> void launch_momentum(Inst<T> &I, bool small)
{
    const int nb = I.nb_mom;
    const size_t region = (size_t)nb * R_NSLOTS;
    if (small) {
        // assemblies over a grid sized for the box capacity (one cell a thread),
        // everything latency-bound in one CTA between them, or in one cluster of
        // CTAs when the box is larger than one CTA's shared memory
        const int se = (int)(I.mom_small_smem / sizeof(T));
        const int nbs = std::max(1, std::min(nb, (mom_small_capacity<T>(I) + 255) / 256));
        const size_t rs = (size_t)nbs * R_NSLOTS;
        double *red_umax = I.red_mom + 4 * rs;
        // (each step is one launch on one CTA and one on the cluster; the one whose
        // case it is not returns at once)
        const int nc = I.mom_cluster;
        const size_t sm = I.mom_small_smem;
        const int wide = nc > 1;
        launch_k(I.pdl, mom_small_pre_kernel<T>, 1, kMomThreads, 0, I.stream, I.p, I.g, red_umax, se, wide);
        if (nc > 1) launch_cluster(I.pdl, mom_cluster_pre_kernel<T>, nc, 0, I.stream, I.p, I.g, red_umax, se);
        for (int ivar = 1; ivar <= 3; ++ivar) {
            launch_k(I.pdl, mom_assemble_kernel<T>, nbs, 256, 0, I.stream, I.p, I.g, ivar,
                     I.red_mom + (ivar - 1) * rs);
            launch_k(I.pdl, mom_small_mid_kernel<T>, 1, kMomThreads, sm, I.stream, I.p, I.g, ivar, I.mom_scratch,
                     se, red_umax, wide);
            if (nc > 1)
                launch_cluster(I.pdl, mom_cluster_mid_kernel<T>, nc, sm, I.stream, I.p, I.g, ivar, I.mom_scratch,
                               se);
        }
        launch_k(I.pdl, pp_assemble_kernel<T>, nbs, 256, 0, I.stream, I.p, I.g, I.red_mom + 3 * rs);
        launch_k(I.pdl, mom_small_post_kernel<T>, 1, kMomThreads, sm, I.stream, I.p, I.g, I.mom_scratch, se,
                 I.red_mom, nbs, wide);
        if (nc > 1)
            launch_cluster(I.pdl, mom_cluster_post_kernel<T>, nc, sm, I.stream, I.p, I.g, I.mom_scratch, se,
                           (const double *)I.red_mom, nbs);
        return;
    }
    if (I.box_grid > 0) {
        // red-black: per equation its assembly and one cooperative launch that
        // solves it and applies the next equation's boundary conditions (for p',
        // corrects velocity and pressure and normalises the residuals)
        launch_k(I.pdl, clean_velocities_kernel<T>, nb, 256, 0, I.stream, I.p, I.g);
        launch_k(I.pdl, mom_bc_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, 1, I.red_mom + 4 * region);
        for (int ivar = 1; ivar <= 4; ++ivar) {
            if (ivar <= 3)
                launch_k(I.pdl, mom_assemble_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, ivar,
                         I.red_mom + (ivar - 1) * region);
            else
                launch_k(I.pdl, pp_assemble_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, I.red_mom + 3 * region);
            launch_box_solve<T>(I, ivar);
        }
        return;
    }
    if (I.order == AMCFD_ORDER_EXACT) launch_box_tickets<T>(I);  // the exact-order sweep's visit order
    launch_k(I.pdl, clean_velocities_kernel<T>, nb, 256, 0, I.stream, I.p, I.g);
    for (int ivar = 1; ivar <= 4; ++ivar) {
        launch_k(I.pdl, mom_bc_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, ivar, I.red_mom + 4 * region);
        if (ivar <= 3)
            launch_k(I.pdl, mom_assemble_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, ivar,
                     I.red_mom + (ivar - 1) * region);
        else
            launch_k(I.pdl, pp_assemble_kernel<T>, nb, 256, 0, I.stream, I.p, I.g, I.red_mom + 3 * region);
        launch_box_factor<T>(I);
        launch_box_sweeps<T>(I, ivar);
        if (ivar == 4) {
            launch_k(I.pdl, correct_velocity_kernel<T>, nb, 256, 0, I.stream, I.p, I.g);
            launch_k(I.pdl, correct_pressure_kernel<T>, nb, 256, 0, I.stream, I.p, I.g);
        }
    }
    launch_k(I.pdl, mom_finalize_kernel<T>, 1, 1024, 0, I.stream, I.p, I.g, I.red_mom, nb);
}

template void launch_momentum<double>(Inst<double> &, bool);
template void launch_momentum<float>(Inst<float> &, bool);
template int mom_small_capacity<double>(const Inst<double> &);
template int mom_small_capacity<float>(const Inst<float> &);
template void setup_mom_small<double>(Inst<double> &);
template void setup_mom_small<float>(Inst<float> &);
template void setup_box_solve<double>(Inst<double> &, bool);
template void setup_box_solve<float>(Inst<float> &, bool);

}  // namespace amcfd
