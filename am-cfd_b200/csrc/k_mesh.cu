// Moving mesh and solidification parameters.
//
// remapSolutions (CFDSolverManager.cpp:2810-3051): after the grid has moved
// with the beam, every field of the remapped set (enthalpy, its previous-step
// value, T, f_l, u, v, w and their previous-step values, p, p', and with the
// species equation avgconcentration and its previous-step value) is moved to
// the new node positions by linear interpolation, first along x over every
// (k, j) row, then along y over every (k, i) column.  A node is moved where its
// centre coordinate changed by more than 1e-6; the partner node is the one in
// the direction the mesh moved.  The reference updates in place in ascending
// index order, so when the mesh moved towards lower coordinates the partner
// is the already-remapped neighbour: each row (column) is one sequential
// recurrence, and each is run by one thread in that order here.  Rows are
// j = 0..nj-2 and i = 1..ni-2 as in the reference loops.
//
// getSolidificationParameters (:2764-2804): per (k, j) row below the top
// plane, the first node i with T >= T_solidus defines the solidification
// front; at node i-1 the gradient G = |grad T| (one-sided in x from T(i) and
// T(i-2), central in y and z) and the growth rate R = scanvel * dT/dx / G are
// stored.  Other nodes keep their previous values.  The reference reads
// outside its arrays for rows with the front at i < 2, on the j = 0 or
// j = nj-1 row or on the k = 0 plane; those rows are skipped here.
#include "kernels.cuh"

namespace amcfd {

template <typename T> struct RemapSet {
    T *f[14];
    int n;
};

__device__ __forceinline__ double lerp_ref(double x0, double x1, double y0, double y1, double x)
{
    // CFDSolverManager::interpolate, :3056-3063
    return y0 + (x - x0) * ((y1 - y0) / (x1 - x0));
}

// x pass: 32 rows per CTA; rows are staged through shared memory in 32-node
// chunks (coalesced loads and stores) and warp 0 runs each row's recurrence.
template <typename T>
__global__ void __launch_bounds__(256) remap_x_kernel(Params p, RemapSet<T> set, const double *oldx,
                                                      const double *newx, int dir)
{
    __shared__ T tile[32][34];
    const int nj = p.nj, nip = p.nip, ni = p.ni;
    const int J = nj - 1, nrows = J * p.nk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int l0 = blockIdx.x * 32; l0 < nrows; l0 += gridDim.x * 32) {
        for (int q = 0; q < set.n; ++q) {
            T *f = set.f[q];
            T prev = T(0);  // remapped value of node i-1 (warp 0, one row per lane)
            if (warp == 0 && l0 + lane < nrows) {
                const int l = l0 + lane, k = l / J, j = l - k * J;
                prev = f[cidx(0, j, k, nj, nip)];
            }
            for (int ib = 1; ib <= ni - 2; ib += 32) {
                for (int r = warp; r < 32; r += 8) {
                    const int l = l0 + r;
                    if (l < nrows) {
                        const int k = l / J, j = l - k * J;
                        const size_t row = cidx(0, j, k, nj, nip);
                        const int i = ib + lane;
                        if (i <= ni - 1) tile[r][lane] = f[row + i];
                        if (lane == 0 && ib + 32 <= ni - 1) tile[r][32] = f[row + ib + 32];
                    }
                }
                __syncthreads();
                if (warp == 0 && l0 + lane < nrows) {
                    const int r = lane, n = min(32, ni - 1 - ib);
                    for (int qq = 0; qq < n; ++qq) {
                        const int i = ib + qq;
                        const double xo = oldx[i], xn = newx[i];
                        if (fabs(xo - xn) > 1e-6) {
                            const double y1 = dir > 0 ? (double)tile[r][qq + 1] : (double)prev;
                            tile[r][qq] = (T)lerp_ref(xo, oldx[i + dir], (double)tile[r][qq], y1, xn);
                        }
                        prev = tile[r][qq];
                    }
                }
                __syncthreads();
                for (int r = warp; r < 32; r += 8) {
                    const int l = l0 + r;
                    const int i = ib + lane;
                    if (l < nrows && i <= ni - 2) {
                        const int k = l / J, j = l - k * J;
                        f[cidx(i, j, k, nj, nip)] = tile[r][lane];
                    }
                }
                __syncthreads();
            }
        }
    }
}

// y pass: one thread per (k, i) column, j ascending (consecutive threads take
// consecutive i, so every step of the recurrence is a coalesced access).
template <typename T>
__global__ void __launch_bounds__(256) remap_y_kernel(Params p, RemapSet<T> set, const double *oldy,
                                                      const double *newy, int dir)
{
    const int nj = p.nj, nip = p.nip, ni = p.ni, nk = p.nk;
    const int I = ni - 2;
    const size_t sj = nip;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)I * nk;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / I), i = 1 + (int)(t - (long long)k * I);
        for (int q = 0; q < set.n; ++q) {
            T *f = set.f[q];
            T *col = f + cidx(i, 0, k, nj, nip);
            for (int j = 0; j <= nj - 2; ++j) {
                const double yo = oldy[j], yn = newy[j];
                // y(0) = 0 never moves; the guard keeps row j-1 inside the array regardless
                if (fabs(yo - yn) > 1e-6 && j + dir >= 0)
                    col[j * sj] = (T)lerp_ref(yo, oldy[j + dir], (double)col[j * sj],
                                              (double)col[(j + dir) * (long long)sj], yn);
            }
        }
    }
}

// one warp per (k, j) row, k < nkm1
template <typename T>
__global__ void __launch_bounds__(256) solidification_kernel(Params p, Fields<T> g, double scanvel)
{
    const int ni = p.ni, nj = p.nj, nip = p.nip;
    const int lane = threadIdx.x & 31;
    const long long nrows = (long long)p.nkm1 * nj;
    const long long W = (long long)gridDim.x * (blockDim.x >> 5);
    const T ts = (T)p.tsolid;
    for (long long w = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); w < nrows; w += W) {
        const int k = (int)(w / nj), j = (int)(w - (long long)k * nj);
        const T *row = g.temp + cidx(0, j, k, nj, nip);
        int front = -1;
        for (int ib = 0; ib < ni && front < 0; ib += 32) {
            const int i = ib + lane;
            const unsigned hot = __ballot_sync(0xffffffffu, i < ni && row[i] >= ts);
            if (hot) front = ib + __ffs(hot) - 1;
        }
        if (lane == 0 && front >= 2 && j >= 1 && j <= nj - 2 && k >= 1) {
            const int i = front;
            const size_t sj = nip, sk = (size_t)nj * nip;
            const size_t c = cidx(i - 1, j, k, nj, nip);
            const double gx = ((double)row[i] - (double)row[i - 2]) / (g.x[i] - g.x[i - 1]) / 2;
            const double gy = ((double)g.temp[c + sj] - (double)g.temp[c - sj]) / (g.y[j] - g.y[j - 1]) / 2;
            const double gz = ((double)g.temp[c + sk] - (double)g.temp[c - sk]) / (g.z[k] - g.z[k - 1]) / 2;
            const double gr = sqrt(gx * gx + gy * gy + gz * gz);
            g.grad[c] = (T)gr;
            g.rate[c] = (T)(scanvel * gx / gr);
        }
    }
}

template <typename T>
void launch_remap(Inst<T> &I, const double *oldx, const double *oldy, int dirx, int diry)
{
    RemapSet<T> s{};
    const Fields<T> &g = I.g;
    T *list[] = {g.h, g.hnot, g.temp, g.fracl, g.uvel, g.vvel, g.wvel, g.unot, g.vnot, g.wnot,
                 g.pressure, g.pp, g.conc, g.concnot};
    for (T *f : list)
        if (f) s.f[s.n++] = f;
    const int rows = (I.p.nj - 1) * I.p.nk;
    remap_x_kernel<T><<<(rows + 31) / 32, 256, 0, I.stream>>>(I.p, s, oldx, g.x, dirx);
    const long long cols = (long long)(I.p.ni - 2) * I.p.nk;
    const int grid = (int)std::min<long long>((cols + 255) / 256, (long long)I.sm_count * 8);
    remap_y_kernel<T><<<std::max(grid, 1), 256, 0, I.stream>>>(I.p, s, oldy, g.y, diry);
}

template <typename T> void launch_solidification(Inst<T> &I, double scanvel)
{
    const long long rows = (long long)I.p.nkm1 * I.p.nj;
    const int grid = (int)std::min<long long>((rows + 7) / 8, (long long)I.sm_count * 16);
    solidification_kernel<T><<<std::max(grid, 1), 256, 0, I.stream>>>(I.p, I.g, scanvel);
}

template void launch_remap<double>(Inst<double> &, const double *, const double *, int, int);
template void launch_remap<float>(Inst<float> &, const double *, const double *, int, int);
template void launch_solidification<double>(Inst<double> &, double);
template void launch_solidification<float>(Inst<float> &, double);

}  // namespace amcfd
