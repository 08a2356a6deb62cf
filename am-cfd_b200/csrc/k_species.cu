// Species conservation: the ivar = 6 branch of iterativeLoopSolve
// (CFDSolverManager.cpp:677-687), solved on avgconcentration after momentum:
//   applyBCs(6)                 BoundCondManager.cpp:655-699   species_bc_kernel
//   discretizeEquations(6)      CFDSolverManager.cpp:1265-1362 species_assemble_kernel
//   calculateSource(6)          CFDSolverManager.cpp:1844-1920   (same kernel)
//   calculateResiduals(6)       CFDSolverManager.cpp:2102-2128   (same kernel)
//   enhanceConvergenceSpeed(6)  CFDSolverManager.cpp:2271-2361 block_correct_kernel + factor_kernel
//   solveEntireDomain(6)        CFDSolverManager.cpp:2459-2526 the energy line sweeps
// The block-correction solve, the line factorisation and the sweeps are the
// energy equation's kernels applied to a different phi.
//
// Traits of the reference's species discretisation that this reproduces:
//  * the face velocities enter the mass fluxes doubled (vvel*2.0 etc.);
//  * the diffusion conductance of a face uses the diffusivity of the cell on
//    its low side only (no harmonic mean): a_n, a_e, a_t of cell P use P's,
//    a_s, a_w, a_b of P use the south/west/bottom neighbour's, except on the
//    first interior row, plane and column (j, i, k = 1), where they use P's;
//  * the diffusivity is 1e-11 in cells at or below the solidus and
//    massdiff * rho (rho after this iteration's property update) elsewhere;
//  * the top boundary value is a flux condition towards the fixed surface
//    concentration 13 where the top node is above the liquidus.
#include <algorithm>

#include "kernels.cuh"

namespace amcfd {

constexpr int kSX = 32, kSY = 8;
constexpr double kSurfaceConc = 13.0;   // BoundCondManager.cpp:666
constexpr double kSolidDiff = 1e-11;    // CFDSolverManager.cpp:1277

// ---------------------------------------------------------------------------
// applyBCs(6).  The reference runs three loops in order: the top and bottom
// planes over interior (j, i); the south and north rows over every (k, i);
// the west and east columns over every (k, j).  Each copies an inner node
// outwards, so the final value of every boundary node is a function of
// interior nodes only:
//   A1(k,j,i), 1<=j<=njm2, 1<=i<=nim2:  k = nkm1 -> top(j,i); k = 0 -> initconc;
//                                       else the node itself (interior);
//   A2(k,j,i), 1<=i<=nim2:              A1(k, clamp(j, 1, njm2), i);
//   boundary node (k,j,i):              A2(k, j, clamp(i, 1, nim2)).
// One pass writes every boundary node from that formula and reads no
// boundary node, so the pass has no ordering hazards.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T species_a1(const Params &p, const Fields<T> &g, int k, int j, int i)
{
    const int nj = p.nj, nip = p.nip;
    if (k == 0) return (T)p.initconc;
    if (k == p.nkm1) {
        const double c2 = (double)g.conc[cidx(i, j, p.nkm2, nj, nip)];
        if ((double)g.temp[cidx(i, j, p.nkm1, nj, nip)] > p.tliquid) {
            const double dsl = p.dens * p.massdiff;
            return (T)(2.0 * (kSurfaceConc - c2) / g.dzpbinv[p.nkm1] / dsl + c2);
        }
        return (T)c2;
    }
    return g.conc[cidx(i, j, k, nj, nip)];
}

template <typename T>
__global__ void __launch_bounds__(256) species_bc_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    const int ni = p.ni, nj = p.nj, nk = p.nk, nip = p.nip;
    const long long fij = (long long)ni * nj, fik = (long long)ni * nk, fjk = (long long)nj * nk;
    const long long total = 2 * (fij + fik + fjk);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        long long r = q;
        if (r < 2 * fij) {            // k = 0 and k = nkm1
            k = r < fij ? 0 : p.nkm1;
            r = r < fij ? r : r - fij;
            j = (int)(r / ni); i = (int)(r - (long long)j * ni);
        } else if ((r -= 2 * fij) < 2 * fik) {  // j = 0 and j = njm1
            j = r < fik ? 0 : p.njm1;
            r = r < fik ? r : r - fik;
            k = (int)(r / ni); i = (int)(r - (long long)k * ni);
        } else {                      // i = 0 and i = nim1
            r -= 2 * fik;
            i = r < fjk ? 0 : p.nim1;
            r = r < fjk ? r : r - fjk;
            k = (int)(r / nj); j = (int)(r - (long long)k * nj);
        }
        const int ic = min(max(i, 1), p.nim2), jc = min(max(j, 1), p.njm2);
        g.conc[cidx(i, j, k, nj, nip)] = species_a1<T>(p, g, k, jc, ic);
    }
}

// ---------------------------------------------------------------------------
// discretizeEquations(6) + calculateSource(6) + calculateResiduals(6) and the
// block-correction sums of enhanceConvergenceSpeed(6), one interior cell per
// thread.  Grid and per-CTA partial layout are those of the energy assembly
// (32 x 8 columns per CTA, a k-segment per blockIdx.z), so block_correct_kernel
// reduces them unchanged.  Along k each thread carries conc and the cell
// diffusivity of the plane below in registers.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T species_diff(const Params &p, const Fields<T> &g, size_t c)
{
    return g.temp[c] <= (T)p.tsolid ? (T)kSolidDiff : (T)p.massdiff * g.rho_nxt[c];
}

template <typename T>
__global__ void __launch_bounds__(kSX * kSY)
species_assemble_kernel(Params p, Fields<T> g, double *red)
{
    pdl_enter();
    using R = T;
    __shared__ double sb[4][kSY][kSX + 1];
    const Status *st = g.st;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * kSX + tx, j = blockIdx.y * kSY + ty;
    const int nj = p.nj, nk = p.nk, nip = p.nip;
    const int nkm2 = p.nkm2, nim2 = p.nim2, njm2 = p.njm2;
    const int kseg = (nk + gridDim.z - 1) / gridDim.z;
    const int kb = max(blockIdx.z * kseg, 1), ke = min(blockIdx.z * kseg + kseg, nk - 1);
    const bool colint = i >= 1 && i <= nim2 && j >= 1 && j <= njm2;
    const size_t sj = nip, sk = (size_t)nj * nip;
    const int sch = p.scheme;
    const double delt = st->delt;
    const R urfc = (R)p.urfc;
    double sumd = 0.0, sumc = 0.0;
    double bl = 0.0, blp = 0.0, blm = 0.0, blc = 0.0;
    if (colint && kb < ke) {
        const double dx = g.xu[i + 1] - g.xu[i], dy = g.yv[j + 1] - g.yv[j];
        const R dxp_i = (R)g.dxpwinv[i], dxp_p = (R)g.dxpwinv[i + 1];
        const R dyp_j = (R)g.dypsinv[j], dyp_p = (R)g.dypsinv[j + 1];
        const R aij = (R)(dx * dy);
        const R *u = g.uvel, *v = g.vvel, *w = g.wvel, *rho = g.rho_nxt, *cn = g.conc;
        size_t c = cidx(i, j, kb, nj, nip);
        R c_m = cn[c - sk], c_c = cn[c];
        R ds_m = kb > 1 ? species_diff<T>(p, g, c - sk) : R(0);  // diffusivity of the plane below
        for (int k = kb; k < ke; ++k, c += sk) {
            const double dz = g.zw[k + 1] - g.zw[k];
            const R aik = (R)(dx * dz), ajk = (R)(dy * dz);
            const R vol = (R)(dx * dy * dz);
            const R c_p = cn[c + sk];
            const R ds_c = species_diff<T>(p, g, c);
            const R ds_s = j > 1 ? species_diff<T>(p, g, c - sj) : ds_c;
            const R ds_w = i > 1 ? species_diff<T>(p, g, c - 1) : ds_c;
            const R ds_b = k > 1 ? ds_m : ds_c;
            const R rho_c = rho[c];
            R an, as_, ae, aw, at, ab, tmp;
            {   // faces on the high side of the cell
                const R fn = rho[c + sj] * (v[c + sj] * R(2)) * aik;
                const R fe = rho[c + 1] * (u[c + 1] * R(2)) * ajk;
                const R ft = rho[c + sk] * (w[c + sk] * R(2)) * aij;
                face_coef<R>(sch, ds_c * aik * dyp_p, fn, an, tmp);
                face_coef<R>(sch, ds_c * ajk * dxp_p, fe, ae, tmp);
                face_coef<R>(sch, ds_c * aij * (R)g.dzpbinv[k + 1], ft, at, tmp);
            }
            {   // faces on the low side: the mass flux through the face itself
                const R fs = rho_c * (v[c] * R(2)) * aik;
                const R fw = rho_c * (u[c] * R(2)) * ajk;
                const R fb = rho_c * (w[c] * R(2)) * aij;
                face_coef<R>(sch, ds_s * aik * dyp_j, fs, tmp, as_);
                face_coef<R>(sch, ds_w * ajk * dxp_i, fw, tmp, aw);
                face_coef<R>(sch, ds_b * aij * (R)g.dzpbinv[k], fb, tmp, ab);
            }
            const R apnot = bdiv(rho_c, (R)delt) * vol;
            R sp = R(0);
            R su = apnot * g.concnot[c];
            const R c_n = cn[c + sj], c_s = cn[c - sj], c_e = cn[c + 1], c_w = cn[c - 1];
            // boundary folds, in the reference's order: k, j, i
            if (k == 1) { su += ab * c_m; sp -= ab; ab = R(0); }
            if (k == nkm2) { su += at * c_p; sp -= at; at = R(0); }
            if (j == 1) { su += as_ * c_s; sp -= as_; as_ = R(0); }
            if (j == njm2) { su += an * c_n; sp -= an; an = R(0); }
            if (i == 1) { su += aw * c_w; sp -= aw; aw = R(0); }
            if (i == nim2) { su += ae * c_e; sp -= ae; ae = R(0); }
            R ap = an + as_ + ae + aw + at + ab + apnot - sp;
            ap = bdiv(ap, urfc);
            su += (R(1) - urfc) * ap * c_c;
            g.an[c] = an; g.as[c] = as_; g.ae[c] = ae; g.aw[c] = aw;
            g.at[c] = at; g.ab[c] = ab; g.ap[c] = ap; g.su[c] = su;
            const R r = bdiv(an * c_n + as_ * c_s + ae * c_e + aw * c_w + at * c_p + ab * c_m + su, ap) - c_c;
            sumd += fabs((double)r);
            sumc += fabs((double)c_c);
            bl += (double)(ap - an - as_ - at - ab);
            blp += (double)ae;
            blm += (double)aw;
            blc += (double)(ae * c_e + aw * c_w + an * c_n + as_ * c_s + at * c_p + ab * c_m + su - ap * c_c);
            c_m = c_c;
            c_c = c_p;
            ds_m = ds_c;
        }
    }
    sb[0][ty][tx] = bl;
    sb[1][ty][tx] = blp;
    sb[2][ty][tx] = blm;
    sb[3][ty][tx] = blc;
    __syncthreads();
    if (ty < 4 && i < nip) {
        double s = 0.0;
        for (int y = 0; y < kSY; ++y) s += sb[ty][y][tx];
        const int part = blockIdx.z * gridDim.y + blockIdx.y;
        g.bc[((size_t)part * 4 + ty) * nip + i] = s;
    }
    __syncthreads();
    double vv[2] = {sumd, sumc};
    const int s[2] = {R_SUMD, R_SUMH};
    const bool m[2] = {false, false};
    const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    block_reduce_store<2>(vv, s, m, red, blk);
}

// updateSolutions, species part (CFDSolverManager.cpp:2680-2685).
template <typename T>
__global__ void species_update_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    const size_t total = (size_t)p.nk * p.nj * p.nip;
    const T kp = (T)p.kp;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (size_t)gridDim.x * blockDim.x) {
        if ((int)(c % p.nip) >= p.ni) continue;
        const T a = g.conc[c], fl = g.fracl[c];
        g.concnot[c] = a;
        g.concn[c] = a / (fl + kp * (T(1) - fl));
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T> void launch_species(Inst<T> &I)
{
    if (!I.p.species) return;
    const Params &p = I.p;
    const long long nb = 2ll * ((long long)p.ni * p.nj + (long long)p.ni * p.nk + (long long)p.nj * p.nk);
    const int grid = (int)std::max(1ll, std::min((long long)I.sm_count * 4, (nb + 255) / 256));
    launch_k(I.pdl, species_bc_kernel<T>, grid, 256, 0, I.stream, I.p, I.g);
    // the energy assembly's grid: its per-CTA partial buffers are reused
    launch_k(I.pdl, species_assemble_kernel<T>, I.asm_grid, dim3(kSX, kSY), 0, I.stream, I.p, I.g, I.red_asm);
    launch_block_correct<T>(I, 6);
    launch_phi_factor<T>(I, I.g.conc);
    launch_phi_sweeps<T>(I, I.g.conc);
}
template <typename T> void launch_species_update(Inst<T> &I)
{
    if (!I.p.species) return;
    launch_k(I.pdl, species_update_kernel<T>, I.grid_1d, 256, 0, I.stream, I.p, I.g);
}

template void launch_species<double>(Inst<double> &);
template void launch_species<float>(Inst<float> &);
template void launch_species_update<double>(Inst<double> &);
template void launch_species_update<float>(Inst<float> &);

}  // namespace amcfd
