// Line-by-line TDMA on x-lines (solveEntireDomain, CFDSolverManager.cpp:2459-2526;
// solveLiquidDomain, :2367-2454).
//
// Each x-line system  ap_i phi_i = aw_i phi_{i-1} + ae_i phi_{i+1} + d_i  with
// d_i = at phi(k+1) + ab phi(k-1) + an phi(j+1) + as phi(j-1) + su  is solved
// by the Thomas recurrences
//     den_i = ap_i - aw_i pr_{i-1},  pr_i = ae_i/den_i,
//     qr_i  = (d_i + aw_i qr_{i-1})/den_i,   phi_i = pr_i phi_{i+1} + qr_i.
// den/pr do not depend on phi, so they are factored once per call
// (factor kernels below).  The two remaining recurrences are affine maps and
// are evaluated by one warp per line: each lane composes the maps of a
// contiguous chunk of cells, a 5-step shuffle scan combines the chunks, and
// each lane then applies the combined map to its own chunk.
//
// Sweep order.  The reference visits lines in the order
//   ksweep(2) x k = nkm2..1 x jsweep(2) x j = 1..njm2
// (Gauss-Seidel in j and k).  Visit (ks,k,s,j) only depends on visits at
// wave t' < t, where t = 3m + (j-j0) + 2s and m = ks*M + (k1-k): writes of
// one wave never touch a row another visit of the same wave reads.  The exact
// mode runs visits in (t, m, s) order with per-line counters, reproducing the
// reference iterates; the red-black mode updates all lines of one (j+k)
// colour at once.
#include "kernels.cuh"
#include "amcfd.h"
#include "async.cuh"
#include "linesolve.cuh"

namespace amcfd {

// ---------------------------------------------------------------------------
// Factorisation: pr, cf = aw/den, iden = 1/den for every line of a box.
// 32 lines per CTA, 32-cell chunks staged through shared memory so global
// accesses stay coalesced; one thread per line walks its chunk sequentially.
// The whole-domain form (enthalpy or avgconcentration as phi) also applies the block
// correction phi += delphi[i] (enhanceConvergenceSpeed, CFDSolverManager.cpp:2351-2361);
// BOX applies the |den| <= 1e-12 guard of
// solveLiquidDomain (:2438-2439) and reads the box from the status block.
// ---------------------------------------------------------------------------
template <typename T, bool BOX>
__global__ void __launch_bounds__(256) factor_kernel(Params p, Fields<T> g, T *phi)
{
    pdl_enter();
    __shared__ T tap[32][33], taw[32][33], tae[32][33], tph[32][33];
    const Status *st = g.st;
    int i0, i1, j0, j1, k0, k1;
    if (BOX) {
        if (!st->momentum_active) return;
        i0 = st->istatp1; i1 = st->iendm1; j0 = st->jstat; j1 = st->jend; k0 = st->kstat; k1 = p.nkm2;
    } else {
        i0 = 1; i1 = p.nim2; j0 = 1; j1 = p.njm2; k0 = 1; k1 = p.nkm2;
    }
    const int J = j1 - j0 + 1, nlines = J * (k1 - k0 + 1);
    if (J <= 0 || k1 < k0 || i1 < i0) return;
    const int nj = p.nj, nip = p.nip;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int l0 = blockIdx.x * 32; l0 < nlines; l0 += gridDim.x * 32) {
        T prv = T(0);  // pr of the previous cell (pr[istat] = 0)
        for (int ib = i0; ib <= i1; ib += 32) {
            for (int r = warp; r < 32; r += 8) {
                int l = l0 + r, i = ib + lane;
                if (l < nlines && i <= i1) {
                    int k = k0 + l / J, j = j0 + l % J;
                    size_t c = cidx(i, j, k, nj, nip);
                    tap[r][lane] = g.ap[c];
                    taw[r][lane] = g.aw[c];
                    tae[r][lane] = g.ae[c];
                    if (!BOX) tph[r][lane] = phi[c] + (T)g.delphi[i];
                }
            }
            __syncthreads();
            if (warp == 0 && l0 + lane < nlines) {
                const int r = lane;
                const int n = min(32, i1 - ib + 1);
                for (int q = 0; q < n; ++q) {
                    T den = tap[r][q] - taw[r][q] * prv;
                    if (BOX && fabs(den) <= T(1e-12)) den += T(kSmall);
                    T id = T(1) / den;
                    T pr = tae[r][q] * id;
                    tap[r][q] = pr;
                    taw[r][q] = taw[r][q] * id;
                    tae[r][q] = id;
                    prv = pr;
                }
            }
            __syncthreads();
            for (int r = warp; r < 32; r += 8) {
                int l = l0 + r, i = ib + lane;
                if (l < nlines && i <= i1) {
                    int k = k0 + l / J, j = j0 + l % J;
                    size_t c = cidx(i, j, k, nj, nip);
                    g.pr[c] = tap[r][lane];
                    g.cf[c] = taw[r][lane];
                    g.iden[c] = tae[r][lane];
                    if (!BOX) phi[c] = tph[r][lane];
                }
            }
            __syncthreads();
        }
    }
}

// Bounded wait until *f >= target (wrap-safe); false after `limit` polls or once
// another warp has raised an error.
__device__ bool wait_ge(const int *f, int target, Status *st, int where, long long limit)
{
    long long it = 0;
    while (true) {
        int v = *(volatile const int *)f;
        if (v - target >= 0) return true;
        if ((it & 63) == 63 && *(volatile int *)&st->error) return false;
        if (++it > limit) {
            if (atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = where;
            return false;
        }
        __nanosleep(64);
    }
}

// ---------------------------------------------------------------------------
// Exact-order sweep: persistent warps take visits in topological order.
// Per-line counters hold seq*4 + (visits done in the current call).
// ---------------------------------------------------------------------------
template <typename T, bool BOX>
__global__ void sweep_exact_kernel(Params p, Fields<T> g, T *phi, int *flags, const int2 *tickets,
                                   int nt_static, unsigned long long *seqp,
                                   unsigned long long *donep, unsigned long long *ticketp)
{
    extern __shared__ unsigned char smraw[];
    Status *st = g.st;
    __shared__ unsigned long long seq_s;
    __shared__ int active_s, nt_s;
    if (threadIdx.x == 0) {
        seq_s = *(volatile unsigned long long *)seqp;
        active_s = BOX ? st->momentum_active : 1;
        nt_s = BOX ? *g.ntickets_mom : nt_static;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const int nmax = p.nip;
    T *sl = reinterpret_cast<T *>(smraw) + (size_t)warp * S_N * nmax;
    uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<T *>(smraw) +
                                                 (size_t)nwarps * S_N * nmax) + warp;
    if (lane == 0) mbar_init(bar);
    __syncwarp();
    uint32_t parity = 0;
    const int base = (int)(seq_s * 4ull);
    int i0, i1, j0, j1, k0, k1;
    box_of<BOX>(p, st, i0, i1, j0, j1, k0, k1);
    if (active_s && i1 >= i0) {
        const int M = k1 - k0 + 1;
        const int nj = p.nj, nip = p.nip;
        const size_t sj = nip, sk = (size_t)nj * nip;
        const int nt = nt_s;
        int ib, ie;
        stage_window<T>(i0, i1, ib, ie);
        while (true) {
            unsigned long long tk = 0;
            if (lane == 0) tk = atomicAdd(ticketp, 1ull);
            tk = __shfl_sync(0xffffffffu, tk, 0);
            if (tk >= (unsigned long long)nt) break;
            int2 e = tickets[tk];
            const int m = e.x, s = e.y >> 16, jj = e.y & 0xffff;
            const int ks = m / M, k = k1 - (m - ks * M), j = j0 + jj, v = 2 * ks + s;
            const size_t row = cidx(0, j, k, nj, nip);
            int ok = 1;
            if (lane == 0) {
                stage_line<T>(g, row, ib, ie, sl, nmax, bar);  // overlaps the waits below
                const int where = k * nj + j;
                const long long lim = p.wait_polls;
                if (ok && j > j0) ok = wait_ge(&flags[k * nj + j - 1], base + v + 1, st, where, lim);
                if (ok && j < j1 && v > 0) ok = wait_ge(&flags[k * nj + j + 1], base + v, st, where, lim);
                if (ok && k < k1) ok = wait_ge(&flags[(k + 1) * nj + j], base + 2 * ks + 2, st, where, lim);
                if (ok && k > k0 && ks > 0) ok = wait_ge(&flags[(k - 1) * nj + j], base + 2 * ks, st, where, lim);
                __threadfence();
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            // the staged copies complete whatever the waits decided
            const bool staged = mbar_wait(bar, parity, st);
            parity ^= 1u;
            if (!ok || !staged) break;
            __syncwarp();
            solve_staged<T, true>(phi, row, i0, i1, ib, sj, sk, sl, nmax);
            __threadfence();
            __syncwarp();
            if (lane == 0) atomicExch(&flags[k * nj + j], base + v + 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long prev = atomicAdd(donep, 1ull);
        if (prev == (unsigned long long)gridDim.x - 1) {
            // last CTA of this call: reset the counters for the next call
            atomicExch(donep, 0ull);
            atomicExch(ticketp, 0ull);
            __threadfence();
            atomicAdd(seqp, 1ull);
        }
    }
}

// ---------------------------------------------------------------------------
// Red-black sweep: every line of one (j+k) colour, one warp per line.
// ---------------------------------------------------------------------------
// Red-black order, momentum box: the factorisation of every line of the box, one
// warp per line (factor_line_mem), the same operations as the cooperative box
// solve forms them with.  The exact order keeps factor_kernel<T, true>, the
// reference's serial recurrence.
template <typename T>
__global__ void __launch_bounds__(256) factor_box_warp_kernel(Params p, Fields<T> g)
{
    pdl_enter();
    const Status *st = g.st;
    if (!st->momentum_active) return;
    int i0, i1, j0, j1, k0, k1;
    box_of<true>(p, st, i0, i1, j0, j1, k0, k1);
    const int J = j1 - j0 + 1, K = k1 - k0 + 1, n = i1 - i0 + 1;
    if (J <= 0 || K <= 0 || n <= 0) return;
    const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5;
    for (int l = blockIdx.x * wpb + warp; l < J * K; l += gridDim.x * wpb) {
        const size_t row = cidx(i0, j0 + l % J, k0 + l / J, p.nj, p.nip);
        factor_line_mem<T>(
            n, [&](int i, T &w, T &e, T &pp) { w = g.aw[row + i]; e = g.ae[row + i]; pp = g.ap[row + i]; },
            [&](int i, T pr, T cf, T id) { g.pr[row + i] = pr; g.cf[row + i] = cf; g.iden[row + i] = id; });
    }
}

template <typename T, bool BOX>
__global__ void sweep_rb_kernel(Params p, Fields<T> g, T *phi, int color)
{
    pdl_enter();
    extern __shared__ unsigned char smraw[];
    const Status *st = g.st;
    if (BOX && !st->momentum_active) return;
    int i0, i1, j0, j1, k0, k1;
    box_of<BOX>(p, st, i0, i1, j0, j1, k0, k1);
    const int J = j1 - j0 + 1, K = k1 - k0 + 1;
    if (J <= 0 || K <= 0 || i1 < i0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int nmax = p.nip;
    T *sl = reinterpret_cast<T *>(smraw) + (size_t)warp * S_N * nmax;
    uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<T *>(smraw) +
                                                 (size_t)wpb * S_N * nmax) + warp;
    if (lane == 0) mbar_init(bar);
    __syncwarp();
    uint32_t parity = 0;
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    int ib, ie;
    stage_window<T>(i0, i1, ib, ie);
    // lines of this colour: for each k, j runs over one parity
    const int half = (J + 1) / 2;
    const int nl = half * K;
    for (int q = blockIdx.x * wpb + warp; q < nl; q += gridDim.x * wpb) {
        int kk = q / half, r = q - kk * half;
        int k = k0 + kk;
        int jpar = ((color - k - j0) % 2 + 2) % 2;  // offset of the first j of this colour
        int j = j0 + jpar + 2 * r;
        if (j > j1) continue;
        const size_t row = cidx(0, j, k, nj, nip);
        if (lane == 0) stage_line<T>(g, row, ib, ie, sl, nmax, bar);
        const bool staged = mbar_wait(bar, parity, g.st);
        parity ^= 1u;
        if (!staged) return;
        __syncwarp();
        solve_staged<T, false>(phi, row, i0, i1, ib, sj, sk, sl, nmax);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Red-black sweep of the whole domain (enthalpy, avgconcentration) in rounds,
// one warp per line.  In round m lane l holds the 16-byte vector of V cells
// starting at i = ib + 32 V m + V l (V = 4 in FP32, 2 in FP64; ib = i0 rounded
// down to 32, so every row access is an aligned 16-byte vector and a round is
// 12 coalesced row segments of 32 V cells in flight per warp).
//   forward:  e_i = (at phi_t + ab phi_b + an phi_n + as phi_s + su) * iden_i;
//             each lane composes the maps x -> cf_i x + e_i of its V cells, an
//             inclusive warp scan chains the lanes, the chain is applied to qr
//             carried from the round before (qr_{i0-1} = phi_{i0-1}), and the
//             lane then runs its cells to get qr; qr and pr go to a per-warp
//             buffer;
//   backward: rounds in reverse, the maps x -> pr_i x + qr_i likewise with a
//             suffix scan, applied to phi carried from the round after
//             (phi_{i1+1} fixed); phi is stored.
// Cells outside i0..i1 carry the identity map.  The neighbours phi_t, phi_b,
// phi_n, phi_s lie on lines of the other colour, which this launch does not
// write; vectors past the end of the padded row read its first vector and are
// masked.
// FACTOR (the first pass of each colour): the line's factorisation is formed in
// the same rounds from ap, aw, ae, exactly as factor_rounds_kernel forms it, and
// stored for the later passes.  With `correct` (the first colour's first pass)
// the block correction phi += delphi, which the factorisation kernel would have
// stored into every interior line, is added to the neighbour values read from
// interior lines instead: each line's own values are overwritten by its pass,
// and the second colour reads the first colour's lines only after that.
// correct = 2 (defect correction, phi = the correction of the current iterate):
// every interior line's correction starts at delphi, so the first colour's
// neighbour values are delphi on interior lines and zero on boundary lines,
// and nothing is read from phi for them.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mat_rescale(T &a, T &b, T &c, T &d);

// 16-byte vector load; CG: through L2 only (rows that other SMs write while the
// kernel runs: the pipelined sweep's neighbour values and factorisation rows).
template <bool CG, typename T>
__device__ __forceinline__ void ld16x(const T *ptr, T (&o)[16 / sizeof(T)])
{
    if constexpr (CG) {
        const typename Vec16<T>::type v = __ldcg(reinterpret_cast<const typename Vec16<T>::type *>(ptr));
        memcpy(o, &v, 16);
    } else {
        ld16(ptr, o);
    }
}

// One pass over the interior x-line (j, k) by the calling warp; sq/spr are the
// warp's qr/pr buffers (2 R RC elements).  The same operations whichever kernel
// calls it, so the per-pass launches and the pipelined launch give the same bits.
template <typename T>
__device__ __forceinline__ void pf_l1(const T *ptr)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(ptr));
}
template <typename T>
__device__ __forceinline__ void pf_l2(const T *ptr)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// PF: each round starts the next round's vectors towards the SM (rows that
// nothing writes during the launch into L1, the factorisation and phi rows into
// L2); measured on the 400x200x100 deck: 0.314 -> 0.299 ms a pipelined solve
// (a second round ahead into L2 as well: 0.309; a bulk prefetch of the whole
// line's twelve rows into L2 before the waits: 0.322).  The per-pass launches,
// with more warps per SM, measured slower with it (0.344 -> 0.377) and run
// without.
template <typename T, bool FACTOR, bool CG, bool PF>
__device__ __forceinline__ void rb_line_rounds(const Params &p, const Fields<T> &g, T *phi, int j, int k,
                                               int correct, T *sq, T *spr)
{
    constexpr int V = 16 / (int)sizeof(T);
    constexpr int RC = 32 * V;
    const int i0 = 1, i1 = p.nim2, j0 = 1, j1 = p.njm2, k0 = 1, k1 = p.nkm2;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int ib = i0 & ~31;
    const int R = (i1 - ib) / RC + 1;
    const int nj = p.nj, nip = p.nip;
    const size_t sj = nip, sk = (size_t)nj * nip;
    {
        const size_t row = cidx(0, j, k, nj, nip);
        T carry = phi[row + i0 - 1];
        T carry_pr = T(0);  // FACTOR: pr at cell i0 - 1
        // FACTOR: which neighbour lines are interior (block-corrected)
        const bool ct = correct && k + 1 <= k1, cb = correct && k - 1 >= k0, cn = correct && j + 1 <= j1,
                   cs = correct && j - 1 >= j0;
        for (int m = 0; m < R; ++m) {
            const int base = ib + RC * m + V * lane;
            const bool inrow = base + V <= nip;
            const size_t c = row + (inrow ? base : 0);
            if (PF && m + 1 < R && base + RC + V <= nip) {
                // the next round's vectors start towards this SM while this round runs:
                // rows nothing writes during the launch into L1, the others into L2
                const size_t cn = c + RC;
                pf_l1(g.at + cn); pf_l1(g.ab + cn); pf_l1(g.an + cn); pf_l1(g.as + cn); pf_l1(g.su + cn);
                if constexpr (FACTOR) {
                    pf_l1(g.aw + cn); pf_l1(g.ap + cn); pf_l1(g.ae + cn);
                } else {
                    pf_l2(g.cf + cn); pf_l2(g.iden + cn); pf_l2(g.pr + cn);
                }
                pf_l2(phi + cn + sk); pf_l2(phi + cn - sk); pf_l2(phi + cn + sj); pf_l2(phi + cn - sj);
            }
            T vt[V], vb[V], vn[V], vs[V], wt[V], wb[V], wn[V], ws[V], wu[V], wc[V], wi[V], wp[V];
            if (FACTOR && correct == 2) {
#pragma unroll
                for (int v = 0; v < V; ++v) vt[v] = vb[v] = vn[v] = vs[v] = T(0);
            } else {
                ld16x<CG>(phi + c + sk, vt); ld16x<CG>(phi + c - sk, vb);
                ld16x<CG>(phi + c + sj, vn); ld16x<CG>(phi + c - sj, vs);
            }
            ld16(g.at + c, wt); ld16(g.ab + c, wb); ld16(g.an + c, wn); ld16(g.as + c, ws);
            ld16(g.su + c, wu);
            if constexpr (FACTOR) {
                // wc, wi, wp receive aw, ap, ae, then cf, iden, pr
                ld16(g.aw + c, wc); ld16(g.ap + c, wi); ld16(g.ae + c, wp);
                T m00 = T(1), m01 = T(0), m10 = T(0), m11 = T(1);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    if (base + v >= i0 && base + v <= i1) {  // [[0, ae], [-aw, ap]] * M
                        const T n00 = wp[v] * m10, n01 = wp[v] * m11;
                        const T n10 = -wc[v] * m00 + wi[v] * m10, n11 = -wc[v] * m01 + wi[v] * m11;
                        m00 = n00; m01 = n01; m10 = n10; m11 = n11;
                    }
                }
                mat_rescale(m00, m01, m10, m11);
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const T b00 = __shfl_up_sync(full, m00, o), b01 = __shfl_up_sync(full, m01, o);
                    const T b10 = __shfl_up_sync(full, m10, o), b11 = __shfl_up_sync(full, m11, o);
                    if (lane >= o) {  // own * lower
                        const T n00 = m00 * b00 + m01 * b10, n01 = m00 * b01 + m01 * b11;
                        const T n10 = m10 * b00 + m11 * b10, n11 = m10 * b01 + m11 * b11;
                        m00 = n00; m01 = n01; m10 = n10; m11 = n11;
                        mat_rescale(m00, m01, m10, m11);
                    }
                }
                const T e00 = __shfl_up_sync(full, m00, 1), e01 = __shfl_up_sync(full, m01, 1);
                const T e10 = __shfl_up_sync(full, m10, 1), e11 = __shfl_up_sync(full, m11, 1);
                T x = carry_pr;
                if (lane > 0) x = (e00 * carry_pr + e01) / (e10 * carry_pr + e11);
                T fpr[V], fcf[V], fid[V];
                bool all = true;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const bool ok = base + v >= i0 && base + v <= i1;
                    all = all && ok;
                    if (ok) {
                        const T den = wi[v] - wc[v] * x;
                        const T idv = T(1) / den;
                        fpr[v] = wp[v] * idv;
                        fcf[v] = wc[v] * idv;
                        fid[v] = idv;
                        x = fpr[v];
                        const T dl = (T)g.delphi[base + v];
                        if (ct) vt[v] = vt[v] + dl;
                        if (cb) vb[v] = vb[v] + dl;
                        if (cn) vn[v] = vn[v] + dl;
                        if (cs) vs[v] = vs[v] + dl;
                    } else {
                        fpr[v] = fcf[v] = fid[v] = T(0);
                    }
                    wp[v] = fpr[v]; wc[v] = fcf[v]; wi[v] = fid[v];
                }
                carry_pr = __shfl_sync(full, x, 31);
                if (all) {
                    typename Vec16<T>::type w;
                    memcpy(&w, fpr, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.pr + c) = w;
                    memcpy(&w, fcf, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.cf + c) = w;
                    memcpy(&w, fid, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.iden + c) = w;
                } else if (inrow) {
#pragma unroll
                    for (int v = 0; v < V; ++v)
                        if (base + v >= i0 && base + v <= i1) {
                            g.pr[c + v] = fpr[v]; g.cf[c + v] = fcf[v]; g.iden[c + v] = fid[v];
                        }
                }
            } else {
                ld16x<CG>(g.cf + c, wc); ld16x<CG>(g.iden + c, wi); ld16x<CG>(g.pr + c, wp);
            }
            T a[V], e[V];
            T Al = T(1), Bl = T(0);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const bool ok = base + v >= i0 && base + v <= i1;
                const T d = wt[v] * vt[v] + wb[v] * vb[v] + wn[v] * vn[v] + ws[v] * vs[v] + wu[v];
                a[v] = ok ? wc[v] : T(1);
                e[v] = ok ? d * wi[v] : T(0);
                Bl = a[v] * Bl + e[v];
                Al = a[v] * Al;
            }
            T A = Al, B = Bl;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T A2 = __shfl_up_sync(full, A, o), B2 = __shfl_up_sync(full, B, o);
                if (lane >= o) {
                    B = A * B2 + B;
                    A = A * A2;
                }
            }
            T Ae = __shfl_up_sync(full, A, 1), Be = __shfl_up_sync(full, B, 1);
            if (lane == 0) { Ae = T(1); Be = T(0); }
            T x = Ae * carry + Be;
            T qv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                x = a[v] * x + e[v];
                qv[v] = x;
            }
            T *dq = sq + (size_t)m * RC + V * lane, *dp = spr + (size_t)m * RC + V * lane;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                dq[v] = qv[v];
                dp[v] = wp[v];
            }
            carry = __shfl_sync(full, A * carry + B, 31);
        }
        __syncwarp();
        T next = phi[row + i1 + 1];
        for (int m = R - 1; m >= 0; --m) {
            const int base = ib + RC * m + V * lane;
            const T *dq = sq + (size_t)m * RC + V * lane, *dp = spr + (size_t)m * RC + V * lane;
            T qv[V], pv[V];
            bool okv[V];
            T Al = T(1), Bl = T(0);
#pragma unroll
            for (int v = V - 1; v >= 0; --v) {
                okv[v] = base + v >= i0 && base + v <= i1;
                qv[v] = okv[v] ? dq[v] : T(0);
                pv[v] = okv[v] ? dp[v] : T(1);
                Bl = pv[v] * Bl + qv[v];
                Al = pv[v] * Al;
            }
            T A = Al, B = Bl;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T A2 = __shfl_down_sync(full, A, o), B2 = __shfl_down_sync(full, B, o);
                if (lane + o < 32) {
                    B = A * B2 + B;
                    A = A * A2;
                }
            }
            T Ae = __shfl_down_sync(full, A, 1), Be = __shfl_down_sync(full, B, 1);
            if (lane == 31) { Ae = T(1); Be = T(0); }
            T x = Ae * next + Be;
            T out[V];
#pragma unroll
            for (int v = V - 1; v >= 0; --v) {
                x = pv[v] * x + qv[v];
                out[v] = x;
            }
            bool all = true;
#pragma unroll
            for (int v = 0; v < V; ++v) all = all && okv[v];
            if (all) {
                typename Vec16<T>::type w;
                memcpy(&w, out, 16);
                *reinterpret_cast<typename Vec16<T>::type *>(phi + row + base) = w;
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (okv[v]) phi[row + base + v] = out[v];
            }
            next = __shfl_sync(full, A * next + B, 0);
        }
        __syncwarp();
    }
}

// One red-black pass: every line of colour `color`, one warp per line.
template <typename T, bool FACTOR>
__global__ void __launch_bounds__(256) sweep_rb_rounds_kernel(Params p, Fields<T> g, T *phi, int color,
                                                              int correct)
{
    pdl_enter();
    constexpr int RC = 32 * (16 / (int)sizeof(T));
    extern __shared__ unsigned char smraw[];
    const int i0 = 1, i1 = p.nim2, j0 = 1, j1 = p.njm2, k0 = 1, k1 = p.nkm2;
    const int J = j1 - j0 + 1, K = k1 - k0 + 1;
    if (J <= 0 || K <= 0 || i1 < i0) return;
    const int warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int R = (i1 - (i0 & ~31)) / RC + 1;
    T *sq = reinterpret_cast<T *>(smraw) + (size_t)warp * 2 * R * RC;
    T *spr = sq + (size_t)R * RC;
    const int half = (J + 1) / 2;
    const int nl = half * K;
    for (int q = blockIdx.x * wpb + warp; q < nl; q += gridDim.x * wpb) {
        const int kk = q / half, r = q - kk * half;
        const int k = k0 + kk;
        const int jpar = ((color - k - j0) % 2 + 2) % 2;  // offset of the first j of this colour
        const int j = j0 + jpar + 2 * r;
        if (j > j1) continue;  // warp-uniform
        rb_line_rounds<T, FACTOR, false, false>(p, g, phi, j, k, correct, sq, spr);
    }
}

// ---------------------------------------------------------------------------
// The eight red-black passes of one solve (2 colours x 4 sweeps) in a single
// launch: a pass starts on a plane as soon as the planes it reads have been
// through the pass before, instead of after the whole previous launch has
// drained.
//
// Work item (pass q, plane k, line j of colour q&1).  Its inputs are the
// values of the four neighbouring lines after pass q-1 (and the line's own
// factorisation, formed in pass q&1); the neighbours' pass q-1 in turn read
// the values that pass q overwrites.  So an item may run once the four
// neighbours have finished pass q-1 and the line itself pass q-2 -- exactly
// the values the per-pass launches give it, hence the same bits.
//
// Items are handed out by an atomic ticket in the order of the key
// s = (k - k0) + D q (D = `stride` planes), then q, then j: every item an
// item waits for has a smaller key, so the smallest outstanding ticket is
// always runnable (no co-residency assumption).  An item waits for items
// D - 1 keys back, so D must exceed the keys in flight (about 3500 warps over
// 800 items a key on the 400x200x100 deck) for the waits to be short; a
// window small enough for the later passes to find a plane's rows in L2 (D of
// 2-4) makes every item wait on the one before it instead, and was measured
// slower than a launch per pass.
// Per-line flags hold 16 seq + (last pass finished + 1), seq counting launches;
// every wait is bounded (wait_polls) and records AMCFD_E_TIMEOUT.
// ---------------------------------------------------------------------------
// (pass, plane) pairs with key below s, for K planes: sum over q of clamp(s - 2q, 0, K).
__device__ __forceinline__ int pipe_pairs_before(int s, int K, int D)
{
    int n = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) n += min(max(s - D * q, 0), K);
    return n;
}

// A warp waits until, in every lane with a flag, *f >= target (wrap-safe): one
// vote per poll, so the warp leaves converged; false after `limit` polls (the
// error is recorded) or once another warp has raised an error.
__device__ bool warp_wait_ge(const int *f, int target, Status *st, int where, long long limit)
{
    const unsigned full = 0xffffffffu;
    for (long long it = 0;; ++it) {
        const bool ok = f == nullptr || *(volatile const int *)f - target >= 0;
        if (__all_sync(full, ok)) return true;
        if ((it & 63) == 63) {
            int e = 0;
            if ((threadIdx.x & 31) == 0) e = *(volatile int *)&st->error;
            if (__shfl_sync(full, e, 0)) return false;
        }
        if (it >= limit) {
            if ((threadIdx.x & 31) == 0 && atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = where;
            return false;
        }
        __nanosleep(64);
    }
}

template <typename T>
__global__ void __launch_bounds__(256, 3) sweep_rb_pipe_kernel(Params p, Fields<T> g, T *phi, int correct, int stride,
                                                               int *flags, unsigned long long *seqp,
                                                               unsigned long long *donep, unsigned long long *ticketp)
{
    pdl_enter();
    constexpr int RC = 32 * (16 / (int)sizeof(T));
    extern __shared__ unsigned char smraw[];
    __shared__ unsigned long long seq_s;
    Status *st = g.st;
    if (threadIdx.x == 0) seq_s = *(volatile unsigned long long *)seqp;
    __syncthreads();
    const int i0 = 1, i1 = p.nim2, j0 = 1, j1 = p.njm2, k0 = 1, k1 = p.nkm2;
    const int J = j1 - j0 + 1, K = k1 - k0 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (J > 0 && K > 0 && i1 >= i0) {
        const int R = (i1 - (i0 & ~31)) / RC + 1;
        T *sq = reinterpret_cast<T *>(smraw) + (size_t)warp * 2 * R * RC;
        T *spr = sq + (size_t)R * RC;
        const int nj = p.nj;
        const int half = (J + 1) / 2;
        const unsigned long long nt = (unsigned long long)half * 8ull * (unsigned long long)K;
        const int base = (int)(seq_s * 16ull);
        const long long lim = p.wait_polls;
        while (true) {
            unsigned long long tk = 0;
            if (lane == 0) tk = atomicAdd(ticketp, 1ull);
            tk = __shfl_sync(0xffffffffu, tk, 0);
            if (tk >= nt) break;
            const int idx = (int)(tk / (unsigned)half), r = (int)(tk - (unsigned long long)idx * half);
            int lo = 0, hi = K - 1 + 7 * stride;  // the key: the largest s with pipe_pairs_before(s) <= idx
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (pipe_pairs_before(mid, K, stride) <= idx) lo = mid;
                else hi = mid - 1;
            }
            const int pass = (lo >= K ? (lo - K + stride) / stride : 0) + (idx - pipe_pairs_before(lo, K, stride));
            const int k = k0 + lo - stride * pass;
            const int jpar = (((pass & 1) - k - j0) % 2 + 2) % 2;
            const int j = j0 + jpar + 2 * r;
            if (j > j1) continue;  // warp-uniform: this colour has one line fewer in the plane
            // lane 0: the line itself after pass - 2; lanes 1-4: its neighbours after pass - 1
            const int *f = nullptr;
            int target = 0;
            if (lane == 0 && pass >= 2) f = &flags[k * nj + j], target = base + pass - 1;
            if (pass >= 1) {
                if (lane == 1 && j > j0) f = &flags[k * nj + j - 1];
                if (lane == 2 && j < j1) f = &flags[k * nj + j + 1];
                if (lane == 3 && k > k0) f = &flags[(k - 1) * nj + j];
                if (lane == 4 && k < k1) f = &flags[(k + 1) * nj + j];
                if (lane >= 1 && lane <= 4) target = base + pass;
            }
            if (!warp_wait_ge(f, target, st, k * nj + j, lim)) break;
            __threadfence();
            if (pass < 2)
                rb_line_rounds<T, true, true, true>(p, g, phi, j, k, pass == 0 ? correct : 0, sq, spr);
            else
                rb_line_rounds<T, false, true, true>(p, g, phi, j, k, 0, sq, spr);
            __threadfence();
            __syncwarp();
            if (lane == 0) atomicExch(&flags[k * nj + j], base + pass + 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long prev = atomicAdd(donep, 1ull);
        if (prev == (unsigned long long)gridDim.x - 1) {
            // last CTA of this launch: reset the counters for the next one
            atomicExch(donep, 0ull);
            atomicExch(ticketp, 0ull);
            __threadfence();
            atomicAdd(seqp, 1ull);
        }
    }
}

// ---------------------------------------------------------------------------
// Whole-domain factorisation in the same 16-byte-vector rounds (one warp per
// line): den_i = ap_i - aw_i pr_{i-1}, pr_i = ae_i/den_i, cf_i = aw_i/den_i,
// iden_i = 1/den_i from pr_{i0-1} = 0, and phi += delphi (the block correction).
// pr follows the projective map x -> ae/(ap - aw x), i.e. the 2x2 matrix
// [[0, ae], [-aw, ap]]: each lane multiplies the matrices of its cells, a warp
// scan (rescaled as it goes; the map ignores scale) gives each lane the product
// of the lanes below, applied to the carried pr of the previous round it is
// the lane's entry value, and the lane then runs the recurrence itself.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mat_rescale(T &a, T &b, T &c, T &d)
{
    const T mx = fmax(fmax(fabs(a), fabs(b)), fmax(fabs(c), fabs(d)));
    if (mx > T(0)) {
        const T s = T(1) / mx;
        a *= s; b *= s; c *= s; d *= s;
    }
}

template <typename T>
__global__ void __launch_bounds__(128) factor_rounds_kernel(Params p, Fields<T> g, T *phi)
{
    pdl_enter();
    constexpr int V = 16 / (int)sizeof(T);
    constexpr int RC = 32 * V;
    const int i0 = 1, i1 = p.nim2;
    const int J = p.njm2, K = p.nkm2;
    if (J <= 0 || K <= 0 || i1 < i0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const unsigned full = 0xffffffffu;
    const int ib = i0 & ~31;
    const int R = (i1 - ib) / RC + 1;
    const int nj = p.nj, nip = p.nip, nl = J * K;
    for (int q = blockIdx.x * wpb + warp; q < nl; q += gridDim.x * wpb) {
        const int k = 1 + q / J, j = 1 + q % J;
        const size_t row = cidx(0, j, k, nj, nip);
        T carry = T(0);  // pr at cell i0 - 1
        for (int m = 0; m < R; ++m) {
            const int base = ib + RC * m + V * lane;
            const bool inrow = base + V <= nip;
            const size_t c = row + (inrow ? base : 0);
            T ap[V], aw[V], ae[V], ph[V];
            ld16(g.ap + c, ap); ld16(g.aw + c, aw); ld16(g.ae + c, ae); ld16(phi + c, ph);
            bool ok[V];
            // product of this lane's matrices, last cell leftmost
            T m00 = T(1), m01 = T(0), m10 = T(0), m11 = T(1);
#pragma unroll
            for (int v = 0; v < V; ++v) {
                ok[v] = base + v >= i0 && base + v <= i1;
                if (ok[v]) {  // [[0, ae], [-aw, ap]] * M
                    const T n00 = ae[v] * m10, n01 = ae[v] * m11;
                    const T n10 = -aw[v] * m00 + ap[v] * m10, n11 = -aw[v] * m01 + ap[v] * m11;
                    m00 = n00; m01 = n01; m10 = n10; m11 = n11;
                }
            }
            mat_rescale(m00, m01, m10, m11);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T b00 = __shfl_up_sync(full, m00, o), b01 = __shfl_up_sync(full, m01, o);
                const T b10 = __shfl_up_sync(full, m10, o), b11 = __shfl_up_sync(full, m11, o);
                if (lane >= o) {  // own * lower
                    const T n00 = m00 * b00 + m01 * b10, n01 = m00 * b01 + m01 * b11;
                    const T n10 = m10 * b00 + m11 * b10, n11 = m10 * b01 + m11 * b11;
                    m00 = n00; m01 = n01; m10 = n10; m11 = n11;
                    mat_rescale(m00, m01, m10, m11);
                }
            }
            // exclusive product applied to the carried pr
            T e00 = __shfl_up_sync(full, m00, 1), e01 = __shfl_up_sync(full, m01, 1);
            T e10 = __shfl_up_sync(full, m10, 1), e11 = __shfl_up_sync(full, m11, 1);
            T x = carry;
            if (lane > 0) x = (e00 * carry + e01) / (e10 * carry + e11);
            T pr[V], cf[V], id[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (ok[v]) {
                    const T den = ap[v] - aw[v] * x;
                    const T idv = T(1) / den;
                    pr[v] = ae[v] * idv;
                    cf[v] = aw[v] * idv;
                    id[v] = idv;
                    x = pr[v];
                    ph[v] = ph[v] + (T)g.delphi[base + v];
                } else {
                    pr[v] = cf[v] = id[v] = T(0);
                }
            }
            carry = __shfl_sync(full, x, 31);
            bool all = true;
#pragma unroll
            for (int v = 0; v < V; ++v) all = all && ok[v];
            if (all) {
                typename Vec16<T>::type w;
                memcpy(&w, pr, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.pr + c) = w;
                memcpy(&w, cf, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.cf + c) = w;
                memcpy(&w, id, 16); *reinterpret_cast<typename Vec16<T>::type *>(g.iden + c) = w;
                memcpy(&w, ph, 16); *reinterpret_cast<typename Vec16<T>::type *>(phi + c) = w;
            } else {
#pragma unroll
                for (int v = 0; v < V; ++v)
                    if (ok[v]) {
                        g.pr[c + v] = pr[v]; g.cf[c + v] = cf[v]; g.iden[c + v] = id[v]; phi[c + v] = ph[v];
                    }
            }
        }
    }
}

// Dynamic shared memory of sweep_rb_rounds_kernel: qr and pr of every round.
template <typename T> size_t rounds_smem(const Params &p, int warps)
{
    const int RC = 32 * (16 / (int)sizeof(T));
    const int R = (p.nim2 - 0) / RC + 1;
    return (size_t)warps * 2 * R * RC * sizeof(T);
}

// ---------------------------------------------------------------------------
// Ticket list of the momentum box, in (t, m, s) order (one CTA).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) box_tickets_kernel(Params p, int2 *tickets, int *ntickets,
                                                           Status *st)
{
    pdl_enter();
    __shared__ int cnt[1024];
    if (!st->momentum_active) return;
    const int J = st->jend - st->jstat + 1, M = p.nkm2 - st->kstat + 1;
    if (J <= 0 || M <= 0) {
        if (threadIdx.x == 0) *ntickets = 0;
        return;
    }
    const int T = 3 * (2 * M - 1) + (J - 1) + 2 + 1;
    auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };  // floor
    auto count_t = [&](int t) {
        int c = 0;
        for (int s = 0; s < 2; ++s) {
            int lo = max(0, -fdiv(-(t - 2 * s - (J - 1)), 3));  // ceil((t-2s-(J-1))/3)
            int hi = min(2 * M - 1, fdiv(t - 2 * s, 3));
            if (hi >= lo) c += hi - lo + 1;
        }
        return c;
    };
    int running = 0;  // tickets written by earlier rounds of 1024 waves
    for (int t0 = 0; t0 < T; t0 += 1024) {
        const int t = t0 + threadIdx.x;
        const int c = t < T ? count_t(t) : 0;
        cnt[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan
            int v = threadIdx.x >= o ? cnt[threadIdx.x - o] : 0;
            __syncthreads();
            cnt[threadIdx.x] += v;
            __syncthreads();
        }
        int off = running + cnt[threadIdx.x] - c;
        if (t < T) {
            int mlo = max(0, -fdiv(-(t - 2 - (J - 1)), 3));
            int mhi = min(2 * M - 1, fdiv(t, 3));
            for (int m = mlo; m <= mhi; ++m) {
                for (int s = 0; s < 2; ++s) {
                    int jj = t - 3 * m - 2 * s;
                    if (jj >= 0 && jj < J) tickets[off++] = make_int2(m, (s << 16) | jj);
                }
            }
        }
        int total = cnt[1023];
        __syncthreads();
        running += total;
    }
    if (threadIdx.x == 0) *ntickets = running;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Red-black order forms the factorisation inside the first sweep of each colour
// (sweep_rb_rounds_kernel<T, true>), so this launch is the exact order's only.
template <typename T> void launch_phi_factor(Inst<T> &I, T *phi)
{
    if (I.order != AMCFD_ORDER_EXACT) return;
    const int lines = (I.p.nj - 2) * (I.p.nk - 2);
    launch_k(I.pdl, factor_rounds_kernel<T>, std::max(1, (lines + 3) / 4), 128, 0, I.stream, I.p, I.g, phi);
}
template <typename T> void launch_energy_factor(Inst<T> &I) { launch_phi_factor<T>(I, I.g.h); }
template <typename T> void launch_box_factor(Inst<T> &I)
{
    // the box is small (a melt pool); one CTA per SM covers up to 4736 lines per pass
    if (I.order == AMCFD_ORDER_REDBLACK) {
        const int grid = std::min((I.max_lines + 7) / 8, 2 * I.sm_count);
        launch_k(I.pdl, factor_box_warp_kernel<T>, grid, 256, 0, I.stream, I.p, I.g);
        return;
    }
    int grid = std::min((I.max_lines + 31) / 32, I.sm_count);
    launch_k(I.pdl, factor_kernel<T, true>, grid, 256, 0, I.stream, I.p, I.g, nullptr);
}
template <typename T> static void sweeps(Inst<T> &I, T *phi, bool box)
{
    const int warps = I.exact_warps;
    const size_t smem = I.line_smem;
    if (I.order == AMCFD_ORDER_EXACT) {
        Status *st = I.g.st;
        if (box)
            sweep_exact_kernel<T, true><<<I.exact_grid, 32 * warps, smem, I.stream>>>(
                I.p, I.g, phi, I.flags_mom, I.g.tickets_mom, 0, &st->seq_mom, &st->done_mom,
                &st->ticket_mom);
        else
            sweep_exact_kernel<T, false><<<I.exact_grid, 32 * warps, smem, I.stream>>>(
                I.p, I.g, phi, I.g.flags, I.g.tickets_energy, I.g.ntickets_energy,
                &st->seq_energy, &st->done_energy, &st->ticket_energy);
    } else if (box) {
        int grid = std::max(1, std::min((I.max_lines / 2 + warps - 1) / warps + 1, I.sm_count));
        for (int sweep = 0; sweep < 4; ++sweep)
            for (int color = 0; color < 2; ++color)
                launch_k(I.pdl, sweep_rb_kernel<T, true>, grid, 32 * warps, smem, I.stream, I.p, I.g, phi, color);
    } else if (I.pipe_grid > 0) {
        // whole domain, the eight passes in one pipelined launch
        Status *st = I.g.st;
        launch_k(I.pdl, sweep_rb_pipe_kernel<T>, I.pipe_grid, 32 * I.pipe_warps, I.pipe_smem, I.stream, I.p, I.g, phi,
                 1, I.pipe_stride, I.flags_pipe, &st->seq_pipe, &st->done_pipe, &st->ticket_pipe);
    } else {
        // whole domain: one line per warp, sweep_warps warps per CTA
        const int w = I.sweep_warps;
        const int lines = ((I.p.nj - 2 + 1) / 2) * (I.p.nk - 2);
        const int grid = std::max(1, (lines + w - 1) / w);
        const size_t rs = rounds_smem<T>(I.p, w);
        for (int color = 0; color < 2; ++color)
            launch_k(I.pdl, sweep_rb_rounds_kernel<T, true>, grid, 32 * w, rs, I.stream, I.p, I.g, phi, color,
                     color == 0);
        for (int sweep = 1; sweep < 4; ++sweep)
            for (int color = 0; color < 2; ++color)
                launch_k(I.pdl, sweep_rb_rounds_kernel<T, false>, grid, 32 * w, rs, I.stream, I.p, I.g, phi, color, 0);
    }
}
template <typename T> void launch_energy_sweeps(Inst<T> &I) { sweeps<T>(I, I.g.h, false); }

// One red-black pass of both kinds (the factorising first pass and a plain one) on
// `phi` with `warps` warps per CTA: what the autotuner times (phi is a scratch copy).
template <typename T> void launch_sweep_probe(Inst<T> &I, T *phi, int warps)
{
    const int lines = ((I.p.nj - 2 + 1) / 2) * (I.p.nk - 2);
    const int grid = std::max(1, (lines + warps - 1) / warps);
    const size_t rs = rounds_smem<T>(I.p, warps);
    launch_k(I.pdl, sweep_rb_rounds_kernel<T, true>, grid, 32 * warps, rs, I.stream, I.p, I.g, phi, 0, 0);
    launch_k(I.pdl, sweep_rb_rounds_kernel<T, false>, grid, 32 * warps, rs, I.stream, I.p, I.g, phi, 1, 0);
}

// ---------------------------------------------------------------------------
// Defect correction of the energy solve (AMCFD_PREC_FP32_DC).  The assembly left
// FP32 coefficients and the FP64 defect r = su + sum a_nb h_nb - ap h in the DC
// buffers; the red-black passes solve A delta = r in FP32 with delta starting at
// the block correction delphi, which in exact arithmetic are the iterates the
// FP64 passes would reach for h (the system is linear), and h += delta is then
// applied in FP64.  The rounding error is that of delta, not of h.
// ---------------------------------------------------------------------------
void launch_dc_sweeps(Inst<double> &I)
{
    Fields<float> f;
    memset(&f, 0, sizeof(f));
    const DcBuf &d = I.dc;
    f.an = d.an; f.as = d.as; f.ae = d.ae; f.aw = d.aw; f.at = d.at; f.ab = d.ab; f.ap = d.ap; f.su = d.su;
    f.pr = d.pr; f.cf = d.cf; f.iden = d.iden;
    f.delphi = I.g.delphi;
    f.st = I.g.st;
    if (I.pipe_grid_dc > 0) {
        Status *st = I.g.st;
        launch_k(I.pdl, sweep_rb_pipe_kernel<float>, I.pipe_grid_dc, 32 * I.pipe_warps, I.pipe_smem_dc, I.stream, I.p,
                 f, d.delta, 2, I.pipe_stride, I.flags_pipe, &st->seq_pipe, &st->done_pipe, &st->ticket_pipe);
        return;
    }
    const int w = I.sweep_warps;
    const int lines = ((I.p.nj - 2 + 1) / 2) * (I.p.nk - 2);
    const int grid = std::max(1, (lines + w - 1) / w);
    const size_t rs = rounds_smem<float>(I.p, w);
    for (int color = 0; color < 2; ++color)
        launch_k(I.pdl, sweep_rb_rounds_kernel<float, true>, grid, 32 * w, rs, I.stream, I.p, f, d.delta, color,
                                                                             color == 0 ? 2 : 0);
    for (int sweep = 1; sweep < 4; ++sweep)
        for (int color = 0; color < 2; ++color)
            launch_k(I.pdl, sweep_rb_rounds_kernel<float, false>, grid, 32 * w, rs, I.stream, I.p, f, d.delta, color,
                     0);
}

// One factorising and one plain pass of the defect-correction sweeps with `warps`
// lines per CTA (the autotuner's probe; it overwrites only the correction).
void launch_dc_sweep_probe(Inst<double> &I, int warps)
{
    Fields<float> f;
    memset(&f, 0, sizeof(f));
    const DcBuf &d = I.dc;
    f.an = d.an; f.as = d.as; f.ae = d.ae; f.aw = d.aw; f.at = d.at; f.ab = d.ab; f.ap = d.ap; f.su = d.su;
    f.pr = d.pr; f.cf = d.cf; f.iden = d.iden;
    f.delphi = I.g.delphi;
    f.st = I.g.st;
    const int lines = ((I.p.nj - 2 + 1) / 2) * (I.p.nk - 2);
    const int grid = std::max(1, (lines + warps - 1) / warps);
    const size_t rs = rounds_smem<float>(I.p, warps);
    launch_k(I.pdl, sweep_rb_rounds_kernel<float, true>, grid, 32 * warps, rs, I.stream, I.p, f, d.delta, 0, 2);
    launch_k(I.pdl, sweep_rb_rounds_kernel<float, false>, grid, 32 * warps, rs, I.stream, I.p, f, d.delta, 1, 0);
}

// h += delta over the interior (delta is zero elsewhere), 16-byte vectors of
// delta: four FP32 corrections onto two FP64 vectors of h.
__global__ void __launch_bounds__(256) dc_apply_kernel(double *h, const float *delta, size_t n4)
{
    pdl_enter();
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (size_t)gridDim.x * blockDim.x) {
        const float4 d = reinterpret_cast<const float4 *>(delta)[q];
        double2 *hp = reinterpret_cast<double2 *>(h) + 2 * q;
        double2 a = hp[0], b = hp[1];
        a.x += (double)d.x; a.y += (double)d.y; b.x += (double)d.z; b.y += (double)d.w;
        hp[0] = a;
        hp[1] = b;
    }
}

void launch_dc_apply(Inst<double> &I)
{
    // the padded pitch is a multiple of 32, so the array is a whole number of 4-vectors
    const size_t n4 = (size_t)I.p.nk * I.p.nj * I.p.nip / 4;
    launch_k(I.pdl, dc_apply_kernel, I.grid_1d, 256, 0, I.stream, I.g.h, I.dc.delta, n4);
}
template <typename T> void launch_phi_sweeps(Inst<T> &I, T *phi) { sweeps<T>(I, phi, false); }
template <typename T> void launch_box_sweeps(Inst<T> &I, int ivar)
{
    T *phi = ivar == 1 ? I.g.uvel : ivar == 2 ? I.g.vvel : ivar == 3 ? I.g.wvel : I.g.pp;
    sweeps<T>(I, phi, true);
}
template <typename T> void launch_box_tickets(Inst<T> &I)
{
    launch_k(I.pdl, box_tickets_kernel, 1, 1024, 0, I.stream, I.p, I.g.tickets_mom, I.g.ntickets_mom, I.g.st);
}

// Occupancy of the persistent sweep (host helper used at context creation).
template <typename T> int exact_sweep_blocks_per_sm(int warps, size_t smem)
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sweep_exact_kernel<T, false>, 32 * warps, smem);
    int nb2 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, sweep_exact_kernel<T, true>, 32 * warps, smem);
    return std::max(1, std::min(nb, nb2));
}
template <typename T> void set_sweep_smem_limit(size_t smem)
{
    raise_smem_limit((const void *)sweep_exact_kernel<T, false>, smem);
    raise_smem_limit((const void *)sweep_exact_kernel<T, true>, smem);
    raise_smem_limit((const void *)sweep_rb_kernel<T, true>, smem);
}
// The whole-domain red-black kernel's buffer (qr and pr of each warp's line): the
// most warps per CTA (8, 4 or 2) whose buffers fit 200 KiB, with the limit raised
// for them; 0 when not even 2 fit.
template <typename T> int set_rounds_smem_limit(const Params &p)
{
    for (int w = 8; w >= 2; w /= 2) {
        const size_t need = rounds_smem<T>(p, w);
        if (need > 200 * 1024) continue;
        if (raise_smem_limit((const void *)sweep_rb_rounds_kernel<T, false>, need) == cudaSuccess &&
            raise_smem_limit((const void *)sweep_rb_rounds_kernel<T, true>, need) == cudaSuccess)
            return w;
    }
    return 0;
}

// Launch shape of the pipelined sweep: `warps` lines per CTA, as many CTAs as are
// resident at once (the kernel needs none of them to be: its tickets come in
// dependency order); 0 when a CTA's line buffers do not fit.
template <typename T> int setup_pipe_sweep(const Params &p, int warps, int sm_count, size_t &smem)
{
    smem = rounds_smem<T>(p, warps);
    if (smem > 200 * 1024 || raise_smem_limit((const void *)sweep_rb_pipe_kernel<T>, smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sweep_rb_pipe_kernel<T>, 32 * warps, smem) != cudaSuccess ||
        nb < 1)
        return 0;
    return nb * sm_count;
}

#define AMCFD_INST(T)                                                     \
    template int setup_pipe_sweep<T>(const Params &, int, int, size_t &); \
    template void launch_energy_factor<T>(Inst<T> &);                    \
    template void launch_box_factor<T>(Inst<T> &);                       \
    template void launch_energy_sweeps<T>(Inst<T> &);                    \
    template void launch_sweep_probe<T>(Inst<T> &, T *, int);            \
    template void launch_phi_factor<T>(Inst<T> &, T *);                  \
    template void launch_phi_sweeps<T>(Inst<T> &, T *);                  \
    template void launch_box_sweeps<T>(Inst<T> &, int);                  \
    template void launch_box_tickets<T>(Inst<T> &);                      \
    template int exact_sweep_blocks_per_sm<T>(int, size_t);              \
    template void set_sweep_smem_limit<T>(size_t);                       \
    template int set_rounds_smem_limit<T>(const Params &);
AMCFD_INST(double)
AMCFD_INST(float)
#undef AMCFD_INST

}  // namespace amcfd
