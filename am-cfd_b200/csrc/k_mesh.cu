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
// recurrence, and each is run by one thread in that order here (one thread
// per line and field; the fields are independent).  Rows are j = 0..nj-2 and
// i = 1..ni-2 as in the reference loops.
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

// One thread per (line, field): a row of nodes along x (stride 1) or a column
// along y (stride nip), walked in ascending order in chunks of kChunk nodes.
// A chunk's kChunk + 1 values are loaded together (the loads overlap), updated
// in registers in the reference's order, and stored: towards higher
// coordinates the partner is the next node's old value (the extra load), towards
// lower ones the previous node's remapped value (carried across chunks).
constexpr int kChunk = 8;

template <typename T>
__device__ __forceinline__ void remap_line(T *f, long long stride, int n0, int n1, const double *oldc,
                                           const double *newc, int dir)
{
    // nodes n0..n1 of the line f[m * stride]
    T prev = f[(long long)(n0 - 1) * stride];  // the node before n0 (never remapped in this pass)
    for (int mb = n0; mb <= n1; mb += kChunk) {
        T v[kChunk + 1];
#pragma unroll
        for (int q = 0; q <= kChunk; ++q)
            if (mb + q <= n1 + 1) v[q] = f[(long long)(mb + q) * stride];
#pragma unroll
        for (int q = 0; q < kChunk; ++q) {
            const int m = mb + q;
            if (m > n1) break;
            const double co = oldc[m], cn = newc[m];
            if (fabs(co - cn) > 1e-6 && m + dir >= 0) {
                const double y1 = dir > 0 ? (double)v[q + 1] : (double)(q == 0 ? prev : v[q - 1]);
                v[q] = (T)lerp_ref(co, oldc[m + dir], (double)v[q], y1, cn);
            }
        }
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            if (mb + q <= n1) f[(long long)(mb + q) * stride] = v[q];
        prev = v[kChunk - 1];
    }
}

// x pass: rows (k, j), j = 0..nj-2, nodes i = 1..ni-2
template <typename T>
__global__ void __launch_bounds__(256) remap_x_kernel(Params p, RemapSet<T> set, const double *oldx,
                                                      const double *newx, int dir)
{
    const int nj = p.nj, nip = p.nip, J = nj - 1;
    const long long nrows = (long long)J * p.nk, total = nrows * set.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / nrows);
        const long long l = t - (long long)q * nrows;
        const int k = (int)(l / J), j = (int)(l - (long long)k * J);
        remap_line<T>(set.f[q] + cidx(0, j, k, nj, nip), 1, 1, p.ni - 2, oldx, newx, dir);
    }
}

// y pass: columns (k, i), i = 1..ni-2, nodes j = 0..nj-2; consecutive threads take
// consecutive i, so every load and store of a chunk is coalesced
template <typename T>
__global__ void __launch_bounds__(256) remap_y_kernel(Params p, RemapSet<T> set, const double *oldy,
                                                      const double *newy, int dir)
{
    const int nj = p.nj, nip = p.nip, I = p.ni - 2;
    const long long ncols = (long long)I * p.nk, total = ncols * set.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / ncols);
        const long long l = t - (long long)q * ncols;
        const int k = (int)(l / I), i = 1 + (int)(l - (long long)k * I);
        // node 0 never moves (y(0) = 0); the walk starts at node 1 with node 0 as its
        // predecessor, which is what the reference's in-place loop sees
        remap_line<T>(set.f[q] + cidx(i, 0, k, nj, nip), nip, 1, nj - 2, oldy, newy, dir);
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
    const long long rows = (long long)(I.p.nj - 1) * I.p.nk * s.n;
    const long long cols = (long long)(I.p.ni - 2) * I.p.nk * s.n;
    auto grid = [&](long long n) { return (int)std::max(1ll, std::min((n + 255) / 256, (long long)I.sm_count * 16)); };
    remap_x_kernel<T><<<grid(rows), 256, 0, I.stream>>>(I.p, s, oldx, g.x, dirx);
    remap_y_kernel<T><<<grid(cols), 256, 0, I.stream>>>(I.p, s, oldy, g.y, diry);
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
