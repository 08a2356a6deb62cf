// Fused energy assembly: discretizeEquations(5) (CFDSolverManager.cpp:1157-1264),
// calculateSource(5) (:1677-1843), calculateResiduals(5) (:2073-2101), the
// coefficient/residual sums of enhanceConvergenceSpeed(5) (:2310-2332) and
// bareplateMaterialProps (:2137-2189, written to the *_nxt buffers so that the
// old properties stay readable by neighbouring cells).
//
// 2.5-D stencil: a CTA owns a 32 (i) x 8 (j) tile and walks a segment of k
// planes.  Each thread keeps its column's k-1 / k / k+1 values in registers and
// loads plane k+2 one plane ahead; i+-1 and j+-1 neighbours come from a
// shared-memory copy of the current plane with a one-cell halo.  Face areas and
// volumes are products of per-column (x, y) and per-plane (z) widths, formed in
// FP64 in the reference's order.  The arithmetic is the reference's expression
// by expression; the FP32 build evaluates properties and divisions in FP32.
#include "kernels.cuh"

namespace amcfd {

constexpr int kTX = 32, kTY = 8, kKSEG = 16;
// resident CTAs per SM the register budget is sized for (three FP32 CTAs spill and
// measured slower than two)
template <typename T> constexpr int asm_min_blocks() { return 2; }

template <typename T>
__global__ void __launch_bounds__(256, asm_min_blocks<T>()) energy_assemble_kernel(Params p, Fields<T> g, double *red)
{
    using R = T;
    __shared__ R s_d[kTY + 2][kTX + 2], s_h[kTY + 2][kTX + 2], s_f[kTY + 2][kTX + 2],
        s_r[kTY + 2][kTX + 2];
    __shared__ R s_u[kTY][kTX + 1], s_v[kTY + 1][kTX];
    __shared__ double sb[4][kTY][kTX + 1];
    const Status *st = g.st;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * kTX + tx, j = blockIdx.y * kTY + ty;
    const int ni = p.ni, nj = p.nj, nk = p.nk, nip = p.nip;
    const int nim1 = p.nim1, njm1 = p.njm1, nkm1 = p.nkm1, nim2 = p.nim2, njm2 = p.njm2,
              nkm2 = p.nkm2;
    const int kseg = (nk + gridDim.z - 1) / gridDim.z;
    const int kb = blockIdx.z * kseg, ke = min(kb + kseg, nk);
    const bool in = (i < ni && j < nj);
    const bool colint = in && i >= 1 && i <= nim2 && j >= 1 && j <= njm2;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const size_t col = in ? cidx(i, j, 0, nj, nip) : 0;
    const int sch = p.scheme;
    const double delt = st->delt;
    const bool volsrc = p.volsrc != 0;
    auto ld = [&](const R *a, int k) -> R { return (in && k >= 0 && k < nk) ? a[col + (size_t)k * sk] : R(0); };

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
    const R dxp_e = (R)g.dxpwinv[nim1], dxp_w = (R)g.dxpwinv[1];
    const R dyp_n = (R)g.dypsinv[njm1], dyp_s = (R)g.dypsinv[1];
    const R dzp_t = (R)g.dzpbinv[nkm1], dzp_b = (R)g.dzpbinv[1];
    const R thla = (R)p.thconla, thlb = (R)p.thconlb, acpl = (R)p.acpl, thsa = (R)p.thconsa,
            thsb = (R)p.thconsb, thsc = (R)p.thconsc, acpa = (R)p.acpa, acpb = (R)p.acpb,
            tliq = (R)p.tliquid, tsol = (R)p.tsolid, denl = (R)p.denl, dens = (R)p.dens,
            visc = (R)p.viscos;

    R d_m = ld(g.diff_cur, kb - 1), d_c = ld(g.diff_cur, kb), d_p = ld(g.diff_cur, kb + 1);
    R h_m = ld(g.h, kb - 1), h_c = ld(g.h, kb), h_p = ld(g.h, kb + 1);
    R f_m = ld(g.fracl, kb - 1), f_c = ld(g.fracl, kb), f_p = ld(g.fracl, kb + 1);
    R r_c = ld(g.rho_cur, kb), r_p = ld(g.rho_cur, kb + 1);
    R w_c = ld(g.wvel, kb), w_p = ld(g.wvel, kb + 1);
    double sumd = 0.0, sumh = 0.0;
    double bl = 0.0, blp = 0.0, blm = 0.0, blc = 0.0;

    for (int k = kb; k < ke; ++k) {
        // one plane ahead for the rolling registers
        const R d_n = ld(g.diff_cur, k + 2), h_n = ld(g.h, k + 2), f_n = ld(g.fracl, k + 2),
                r_n = ld(g.rho_cur, k + 2), w_n = ld(g.wvel, k + 2);
        const size_t c = col + (size_t)k * sk;
        const R t_c = in ? g.temp[c] : R(0);
        const R hnot_c = in ? g.hnot[c] : R(0);
        const R flnot_c = in ? g.fraclnot[c] : R(0);
        // ---- stage plane k with a one-cell halo ----
        s_d[ty + 1][tx + 1] = d_c;
        s_h[ty + 1][tx + 1] = h_c;
        s_f[ty + 1][tx + 1] = f_c;
        s_r[ty + 1][tx + 1] = r_c;
        s_u[ty][tx] = in ? g.uvel[c] : R(0);
        s_v[ty][tx] = in ? g.vvel[c] : R(0);
        if (in) {
            if (tx == 0 && i >= 1) {
                s_d[ty + 1][0] = g.diff_cur[c - 1];
                s_h[ty + 1][0] = g.h[c - 1];
                s_f[ty + 1][0] = g.fracl[c - 1];
            }
            if (tx == kTX - 1 && i + 1 < ni) {
                s_d[ty + 1][kTX + 1] = g.diff_cur[c + 1];
                s_h[ty + 1][kTX + 1] = g.h[c + 1];
                s_f[ty + 1][kTX + 1] = g.fracl[c + 1];
                s_r[ty + 1][kTX + 1] = g.rho_cur[c + 1];
                s_u[ty][kTX] = g.uvel[c + 1];
            }
            if (ty == 0 && j >= 1) {
                s_d[0][tx + 1] = g.diff_cur[c - sj];
                s_h[0][tx + 1] = g.h[c - sj];
                s_f[0][tx + 1] = g.fracl[c - sj];
            }
            if (ty == kTY - 1 && j + 1 < nj) {
                s_d[kTY + 1][tx + 1] = g.diff_cur[c + sj];
                s_h[kTY + 1][tx + 1] = g.h[c + sj];
                s_f[kTY + 1][tx + 1] = g.fracl[c + sj];
                s_r[kTY + 1][tx + 1] = g.rho_cur[c + sj];
                s_v[kTY][tx] = g.vvel[c + sj];
            }
        }
        __syncthreads();
        if (in) {
            // ---- material properties (every node) ----
            {
                const R t = t_c, fl = f_c;
                const R diffl = bdiv(thla * t + thlb, acpl);
                R dn = diffl, rn = denl, vn = visc;
                if (!(t >= tliq)) {
                    const R diffs = bdiv(thsa * (t * t) + thsb * t + thsc, acpa * t + acpb);
                    dn = diffs; rn = dens; vn = R(1e10);
                    if (!(t <= tsol)) {
                        dn = fl * diffl + (R(1) - fl) * diffs;
                        rn = fl * denl + (R(1) - fl) * dens;
                        vn = visc;
                    }
                }
                g.diff_nxt[c] = dn;
                g.rho_nxt[c] = rn;
                g.vis_nxt[c] = vn;
            }
            if (colint && k >= 1 && k <= nkm2) {
                const double dz = g.zw[k + 1] - g.zw[k];
                const R aik = (R)(dx * dz), ajk = (R)(dy * dz);
                const R vol = (R)(dx * dy * dz);
                const R fz_k = (R)g.fracz[k], fz_m = (R)g.fracz[k - 1];
                const R dzp_k = (R)g.dzpbinv[k], dzp_p = (R)g.dzpbinv[k + 1];
                const R dcc = d_c, rhc = r_c;
                const R d_e = s_d[ty + 1][tx + 2], d_w = s_d[ty + 1][tx], d_nn = s_d[ty + 2][tx + 1],
                        d_s = s_d[ty][tx + 1];
                R an, as_, ae, aw, at, ab, tmp;
                const R u_c = s_u[ty][tx], u_e = s_u[ty][tx + 1];
                const R v_c = s_v[ty][tx], v_n = s_v[ty + 1][tx];
                // north face
                {
                    R fn = s_r[ty + 2][tx + 1] * v_n * aik;
                    R dn;
                    if (j == njm2) {
                        dn = dcc * aik * dyp_n;
                    } else {
                        R difn = bdiv(dcc * d_nn, (R(1) - fy_j) * d_nn + fy_j * dcc);
                        dn = difn * aik * dyp_p;
                    }
                    face_coef<R>(sch, dn, fn, an, tmp);
                }
                // south face
                {
                    R fs = rhc * v_c * aik;
                    R ds;
                    if (j == 1) {
                        ds = dcc * aik * dyp_s;
                    } else {
                        R difs = bdiv(d_s * dcc, (R(1) - fy_m) * dcc + fy_m * d_s);
                        ds = difs * aik * dyp_j;
                    }
                    face_coef<R>(sch, ds, fs, tmp, as_);
                }
                // east face
                {
                    R fe = s_r[ty + 1][tx + 2] * u_e * ajk;
                    R de;
                    if (i == nim2) {
                        de = dcc * ajk * dxp_e;
                    } else {
                        R dife = bdiv(dcc * d_e, (R(1) - fx_i) * d_e + fx_i * dcc);
                        de = dife * ajk * dxp_p;
                    }
                    face_coef<R>(sch, de, fe, ae, tmp);
                }
                // west face
                {
                    R fw = rhc * u_c * ajk;
                    R dw;
                    if (i == 1) {
                        dw = dcc * ajk * dxp_w;
                    } else {
                        R difw = bdiv(d_w * dcc, (R(1) - fx_m) * dcc + fx_m * d_w);
                        dw = difw * ajk * dxp_i;
                    }
                    face_coef<R>(sch, dw, fw, tmp, aw);
                }
                // top face
                {
                    R ft = r_p * w_p * aij;
                    R dt;
                    if (k == nkm2) {
                        dt = dcc * aij * dzp_t;
                    } else {
                        R dift = bdiv(dcc * d_p, (R(1) - fz_k) * d_p + fz_k * dcc);
                        dt = dift * aij * dzp_p;
                    }
                    face_coef<R>(sch, dt, ft, at, tmp);
                }
                // bottom face
                {
                    R fb = rhc * w_c * aij;
                    R db;
                    if (k == 1) {
                        db = dcc * aij * dzp_b;
                    } else {
                        R difb = bdiv(d_m * dcc, (R(1) - fz_m) * dcc + fz_m * d_m);
                        db = difb * aij * dzp_k;
                    }
                    face_coef<R>(sch, db, fb, tmp, ab);
                }
                const R densbydt = bdiv(rhc, (R)delt);
                const R apnot = densbydt * vol;
                R sp = R(0);
                R su = apnot * hnot_c;
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
                const R variable1 = bdiv(hlatnt * rhc, (R)delt);
                const R volht = vol * variable1;
                const R flc = f_c;
                su -= volht * (flc - flnot_c);
                {
                    const R fl_w = s_f[ty + 1][tx], fl_e = s_f[ty + 1][tx + 2], fl_s = s_f[ty][tx + 1],
                            fl_n = s_f[ty + 2][tx + 1];
                    R flew = ajk * (maxd(u_c, R(0)) * fl_w - maxd(-u_c, R(0)) * flc +
                                    maxd(-u_e, R(0)) * fl_e - maxd(u_e, R(0)) * flc);
                    R flns = aik * (maxd(v_c, R(0)) * fl_s - maxd(-v_c, R(0)) * flc +
                                    maxd(-v_n, R(0)) * fl_n - maxd(v_n, R(0)) * flc);
                    R fltb = aij * (maxd(w_c, R(0)) * f_m - maxd(-w_c, R(0)) * flc +
                                    maxd(-w_p, R(0)) * f_p - maxd(w_p, R(0)) * flc);
                    su += rhc * hlatnt * (flew + flns + fltb);
                }
                const R hc = h_c;
                const R hjp = s_h[ty + 2][tx + 1], hjm = s_h[ty][tx + 1], hip = s_h[ty + 1][tx + 2],
                        him = s_h[ty + 1][tx], hkp = h_p, hkm = h_m;
                // boundary folds, in the reference's order: k, j, i
                if (k == 1) { su += ab * hkm; sp -= ab; ab = R(0); }
                if (k == nkm2) { su += at * hkp; sp -= at; at = R(0); }
                if (j == 1) { su += as_ * hjm; sp -= as_; as_ = R(0); }
                if (j == njm2) { su += an * hjp; sp -= an; an = R(0); }
                if (i == 1) { su += aw * him; sp -= aw; aw = R(0); }
                if (i == nim2) { su += ae * hip; sp -= ae; ae = R(0); }
                R ap = an + as_ + ae + aw + at + ab + apnot - sp;
                const R urfh = (R)p.urfh;
                ap = bdiv(ap, urfh);
                su += (R(1) - urfh) * ap * hc;
                g.an[c] = an; g.as[c] = as_; g.ae[c] = ae; g.aw[c] = aw;
                g.at[c] = at; g.ab[c] = ab; g.ap[c] = ap; g.su[c] = su;
                // ---- residual (calculateResiduals(5)) ----
                R r = bdiv(an * hjp + as_ * hjm + ae * hip + aw * him + at * hkp + ab * hkm + su, ap) - hc;
                sumd += fabs((double)r);
                sumh += fabs((double)hc);
                // ---- block-correction sums (enhanceConvergenceSpeed(5)) ----
                bl += (double)(ap - an - as_ - at - ab);
                blp += (double)ae;
                blm += (double)aw;
                blc += (double)(ae * hip + aw * him + an * hjp + as_ * hjm + at * hkp + ab * hkm + su - ap * hc);
            }
        }
        __syncthreads();
        d_m = d_c; d_c = d_p; d_p = d_n;
        h_m = h_c; h_c = h_p; h_p = h_n;
        f_m = f_c; f_c = f_p; f_p = f_n;
        r_c = r_p; r_p = r_n;
        w_c = w_p; w_p = w_n;
    }
    // per-i partial sums over this block's j-rows and planes
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
// give every SM several CTAs (at least 4 x 148 tiles x segments).
dim3 energy_assemble_grid(const Params &p)
{
    const int tiles = ((p.ni + kTX - 1) / kTX) * ((p.nj + kTY - 1) / kTY);
    int seg = kKSEG;
    while (seg > 4 && tiles * ((p.nk + seg - 1) / seg) < 4 * 148) seg /= 2;
    return dim3((p.ni + kTX - 1) / kTX, (p.nj + kTY - 1) / kTY, (p.nk + seg - 1) / seg);
}

template <typename T> void launch_energy_assemble(Inst<T> &I)
{
    energy_assemble_kernel<T><<<I.asm_grid, dim3(kTX, kTY), 0, I.stream>>>(I.p, I.g, I.red_asm);
}

template void launch_energy_assemble<double>(Inst<double> &);
template void launch_energy_assemble<float>(Inst<float> &);

}  // namespace amcfd
