// Energy-balance free surface (FreeSurfaceManager.cpp): post-processing of the
// top surface run before each output, with no effect on the solution.
//
// execute (:74-209): a bisection on the pressure multiplier lambda drives the
// volume under the surface deflection fi (getDeltaVol, :214-237) to -vd.  For
// each lambda, ebal (:242-341) relaxes fi on the molten top nodes with Jacobi
// sweeps of the balance between gravity (dens*g), surface tension (the
// curvature of fi) and lambda.  Then every node is lifted to
// zr = z (1 - fi/z_top), and the temperature there is interpolated along the
// column (tempr).
//
// Kernel layout.  The bisection is sequential and every sweep depends on the
// previous one, so one CTA of 1024 threads runs the whole bisection.  The
// sweeps touch only the bounding box of molten top nodes plus a one-node halo;
// fi and its iterate live in global memory (a plane, L2 resident).  fi
// persists between calls, as the reference's member array does: nodes that
// are not molten keep the deflection of earlier calls, and both the sweeps
// (through the halo) and the volume sum see those values.
//
// The sweep loop stops when the largest relative change is below the
// tolerance.  In the reference that maximum is never reset, and the first
// sweep divides by the zero iterate (:262-263, 298-300), so it becomes
// infinite as soon as one node is molten.  The loop therefore runs every
// sweep when a top node is molten, and stops after the first otherwise; here
// the maximum is kept the same way, as a running fmax over sweeps.
#include "kernels.cuh"

namespace amcfd {

constexpr int kFsThreads = 1024;

__device__ __forceinline__ double block_sum_fs(double v, double *sh)
{
    // fixed-order tree: per-warp shuffle sums, then warp 0 sums the 32 partials
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = threadIdx.x < 32 ? sh[threadIdx.x] : 0.0;
    if (warp == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[32] = t;
    __syncthreads();
    return sh[32];
}
__device__ __forceinline__ double block_fmax_fs(double v, double *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = threadIdx.x < 32 ? sh[threadIdx.x] : -INFINITY;
    if (warp == 0) t = warp_max(t);
    if (threadIdx.x == 0) sh[32] = t;
    __syncthreads();
    return sh[32];
}

template <typename T>
__global__ void __launch_bounds__(kFsThreads) free_surface_kernel(Params p, Fields<T> g, FsIn a, FsOut *out)
{
    __shared__ double sh[33];
    __shared__ int box[4];
    __shared__ int stop_s;
    const int ni = p.ni, nj = p.nj, nip = p.nip, nkm1 = p.nkm1;
    const int tid = threadIdx.x;
    const T *ttop = g.temp + cidx(0, 0, nkm1, nj, nip);
    const T ts = (T)p.tsolid;
    double *FI = g.fs_fi, *ZZ = g.fs_zz;
    const double *x = g.x, *y = g.y, *xu = g.xu, *yv = g.yv;

    // molten top nodes (the reference skips a node when T < T_solidus)
    if (tid == 0) { box[0] = INT_MAX; box[1] = INT_MIN; box[2] = INT_MAX; box[3] = INT_MIN; }
    __syncthreads();
    {
        int ilo = INT_MAX, ihi = INT_MIN, jlo = INT_MAX, jhi = INT_MIN;
        const int I = ni - 2;
        for (int q = tid; q < I * (nj - 2); q += kFsThreads) {
            const int j = 1 + q / I, i = 1 + q % I;
            if (!(ttop[(size_t)j * nip + i] < ts)) {
                ilo = min(ilo, i); ihi = max(ihi, i); jlo = min(jlo, j); jhi = max(jhi, j);
            }
        }
        if (ilo != INT_MAX) {
            atomicMin(&box[0], ilo); atomicMax(&box[1], ihi);
            atomicMin(&box[2], jlo); atomicMax(&box[3], jhi);
        }
    }
    __syncthreads();
    const bool any = box[0] != INT_MAX;
    // box + halo (the iterate is read one node out)
    const int hi0 = any ? box[0] - 1 : 0, hi1 = any ? box[1] + 1 : -1;
    const int hj0 = any ? box[2] - 1 : 0, hj1 = any ? box[3] + 1 : -1;
    const int HW = hi1 - hi0 + 1, HN = HW * (hj1 - hj0 + 1);
    // volume of the interior nodes outside the box: constant during this call
    double s_out;
    {
        double s = 0.0;
        const int I = ni - 2;
        for (int q = tid; q < I * (nj - 2); q += kFsThreads) {
            const int j = 1 + q / I, i = 1 + q % I;
            const bool inbox = any && i >= box[0] && i <= box[1] && j >= box[2] && j <= box[3];
            if (!inbox) s += ((xu[i + 1] - xu[i]) * (yv[j + 1] - yv[j])) * FI[(size_t)j * nip + i];
        }
        s_out = block_sum_fs(s, sh);
    }

    // getDeltaVol(lambda) = ebal(lambda), then the volume sum
    auto delta_vol = [&](double lam) -> double {
        for (int q = tid; q < HN; q += kFsThreads) ZZ[(size_t)(hj0 + q / HW) * nip + hi0 + q % HW] = 0.0;
        __syncthreads();
        double difmax = 0.0;
        for (int it = 0; it < a.maxit_e; ++it) {
            double dloc = -INFINITY;
            if (any) {
                const int BW = box[1] - box[0] + 1, BN = BW * (box[3] - box[2] + 1);
                for (int q = tid; q < BN; q += kFsThreads) {
                    const int j = box[2] + q / BW, i = box[0] + q % BW;
                    if (ttop[(size_t)j * nip + i] < ts) continue;
                    const size_t c = (size_t)j * nip + i;
                    const double dely = yv[j + 1] - yv[j - 1], dely1 = y[j + 1] - y[j - 1];
                    const double delyp = y[j + 1] - y[j], delym = y[j] - y[j - 1];
                    const double delx = xu[i + 1] - xu[i - 1], delx1 = x[i + 1] - x[i - 1];
                    const double delxp = x[i + 1] - x[i], delxm = x[i] - x[i - 1];
                    const double c2 = 0.0 + lam;  // apdis = 0 (:97-103)
                    const double dzdx = (ZZ[c + 1] - ZZ[c - 1]) / delx1;
                    const double dzdy = (ZZ[c + nip] - ZZ[c - nip]) / dely1;
                    const double dzdyp1 = (ZZ[c + nip + 1] - ZZ[c - nip + 1]) / dely1;
                    const double dzdym1 = (ZZ[c + nip - 1] - ZZ[c - nip - 1]) / dely1;
                    const double d2zdxdy = (dzdyp1 - dzdym1) / delx1;
                    const double c3 = pow(1.0 + dzdx * dzdx + dzdy * dzdy, 1.5);
                    const double c4 = 1.0 + dzdy * dzdy, c5 = 1.0 + dzdx * dzdx;
                    const double c6 = 2.0 * dzdx * dzdy * d2zdxdy;
                    const double c7 = ZZ[c + 1] / (delxp * delx) + ZZ[c - 1] / (delxm * delx);
                    const double c8 = ZZ[c + nip] / (delyp * dely) + ZZ[c - nip] / (delym * dely);
                    const double c9 = 1.0 / (delxp * delx) + 1.0 / (delxm * delx);
                    const double c10 = 1.0 / (delyp * dely) + 1.0 / (delym * dely);
                    const double c11 = a.gamma / c3;
                    const double term1 = c2 + c11 * (c4 * c7 + c5 * c8 - c6);
                    const double term2 = a.c1 + c11 * (c4 * c9 + c5 * c10);
                    const double fi = a.urf * term1 / term2 + (1.0 - a.urf) * ZZ[c];
                    FI[c] = fi;
                    dloc = fmax(dloc, fabs((fi - ZZ[c]) / ZZ[c]));
                }
            }
            difmax = fmax(difmax, block_fmax_fs(dloc, sh));  // never reset, as in the reference
            if (difmax < a.tol_e) break;
            for (int q = tid; q < HN; q += kFsThreads) {
                const size_t c = (size_t)(hj0 + q / HW) * nip + hi0 + q % HW;
                ZZ[c] = FI[c];
            }
            __syncthreads();
        }
        double s = 0.0;
        if (any) {
            const int BW = box[1] - box[0] + 1, BN = BW * (box[3] - box[2] + 1);
            for (int q = tid; q < BN; q += kFsThreads) {
                const int j = box[2] + q / BW, i = box[0] + q % BW;
                s += ((xu[i + 1] - xu[i]) * (yv[j + 1] - yv[j])) * FI[(size_t)j * nip + i];
            }
        }
        return s_out + block_sum_fs(s, sh);
    };

    // execute: bisection (:126-165), decided by thread 0 and broadcast
    double alamopt = 0.0, dx = 0.0, xmid = 0.0, fmid;
    const double f = delta_vol(a.lam1) + a.vd;
    fmid = delta_vol(a.lam2) + a.vd;
    int bracketed = !(f * fmid >= 0.0 && f != a.vd);
    if (f < 0.0) { alamopt = a.lam1; dx = a.lam2 - a.lam1; }
    else { alamopt = a.lam2; dx = a.lam1 - a.lam2; }
    int niter = 0;
    for (niter = 0; niter < a.maxit_b; niter++) {
        dx *= 0.5;
        xmid = alamopt + dx;
        fmid = delta_vol(xmid) + a.vd;
        if (fmid < 0.0) alamopt = xmid;
        if (tid == 0) stop_s = (fabs(dx) < 1.0e-5 || (fabs(fmid) < a.tol_b && niter != 0));
        __syncthreads();
        const int stop = stop_s;
        __syncthreads();
        if (stop) break;
    }
    // extremes of fi over the whole plane (:199-201)
    double mn = INFINITY, mx = -INFINITY;
    for (int q = tid; q < ni * nj; q += kFsThreads) {
        const double v = FI[(size_t)(q / ni) * nip + q % ni];
        mn = fmin(mn, v);
        mx = fmax(mx, v);
    }
    const double fimax = block_fmax_fs(mx, sh);
    const double fimin = -block_fmax_fs(-mn, sh);
    if (tid == 0) {
        out->xmid = xmid; out->fmid = fmid; out->fimin = fimin; out->fimax = fimax;
        out->niter = niter; out->bracketed = bracketed;
    }
}

// Deformed heights and the temperatures interpolated onto them (:171-193), every
// node of the active domain.
template <typename T>
__global__ void free_surface_project_kernel(Params p, Fields<T> g)
{
    const int ni = p.ni, nj = p.nj, nip = p.nip, nkm1 = p.nkm1;
    const long long n = (long long)ni * nj * p.nk;
    const size_t sk = (size_t)nj * nip;
    const double ztop = g.z[nkm1];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % ni);
        const long long r = q / ni;
        const int j = (int)(r % nj), k = (int)(r / nj);
        const size_t col = (size_t)j * nip + i, c = col + (size_t)k * sk;
        const double factor = g.fs_fi[col] / ztop;
        const double zr = g.z[k] * (1.0 - factor);
        g.fs_zr[c] = (T)zr;
        if (zr > ztop) continue;
        if (zr == ztop) g.fs_tempr[c] = g.temp[col + (size_t)nkm1 * sk];
        for (int l = nkm1 - 1; l >= 0; l--) {
            if (g.z[l] <= zr) {
                const double tl = (double)g.temp[col + (size_t)l * sk], tu = (double)g.temp[col + (size_t)(l + 1) * sk];
                g.fs_tempr[c] = (T)((zr - g.z[l]) / (g.z[l + 1] - g.z[l]) * (tu - tl) + tl);
                break;
            }
        }
    }
}

template <typename T> void launch_free_surface(Inst<T> &I, const FsIn &a, FsOut *out_dev)
{
    free_surface_kernel<T><<<1, kFsThreads, 0, I.stream>>>(I.p, I.g, a, out_dev);
    free_surface_project_kernel<T><<<I.grid_1d, 256, 0, I.stream>>>(I.p, I.g);
}
template void launch_free_surface<double>(Inst<double> &, const FsIn &, FsOut *);
template void launch_free_surface<float>(Inst<float> &, const FsIn &, FsOut *);

}  // namespace amcfd
