// Line-solve primitives shared by the energy sweeps (k_linesolve.cu) and the
// momentum-box solves (k_momentum.cu): per-warp staging of an x-line's
// coefficient rows, the warp-scan Thomas recurrences of one line, the box
// extents, and the grid barrier of the cooperative box solve.
#pragma once
#include "kernels.cuh"
#include "amcfd.h"
#include "async.cuh"

namespace amcfd {

// Load of a value another warp may have just written (bypasses L1).
template <typename T> __device__ __forceinline__ T ld_shared_row(const T *ptr) { return __ldcg(ptr); }

// Explicitly rounded operations: the right-hand side of a line's cell is formed
// by the same sequence of roundings whichever code forms it (left to the
// compiler, which product fuses into which sum may depend on where the operands
// come from).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
// e = (at phi_t + ab phi_b + an phi_n + as phi_s + su) / den, with 1/den given
template <typename T>
__device__ __forceinline__ T line_rhs(T at, T vt, T ab, T vb, T an, T vn, T as, T vs, T su, T id)
{
    return mul_rn(add_rn(fma_rn(as, vs, fma_rn(an, vn, fma_rn(ab, vb, mul_rn(at, vt)))), su), id);
}

// ---------------------------------------------------------------------------
// Per-warp staging of one x-line.  The eight pass-invariant coefficient rows of
// the line (at ab an as su cf pr iden) are brought into shared memory with
// TMA bulk copies completing on a per-warp mbarrier; the copies are issued
// before the exact-order kernel waits on its neighbours, so their latency
// overlaps the wait.  Rows start 16-byte aligned: the copy starts at the
// aligned cell ib <= i0 and is rounded up to whole 16-byte units (never past
// the padded row, nip being a multiple of 32 cells).
// ---------------------------------------------------------------------------
enum { S_AT = 0, S_AB, S_AN, S_AS, S_SU, S_CF, S_PR, S_ID, S_N, S_Q = S_N };

template <typename T>
__device__ __forceinline__ void stage_line(const Fields<T> &g, size_t row, int ib, int ie, T *sl,
                                           int nmax, uint64_t *bar)
{
    // lane 0 only.  Previous generic-proxy use of this shared buffer is ordered
    // before the asynchronous copies by the proxy fence.
    fence_proxy_async();
    const uint32_t bytes = (uint32_t)((ie - ib) * sizeof(T));
    mbar_expect_tx(bar, bytes * S_N);
    const T *src[S_N] = {g.at, g.ab, g.an, g.as, g.su, g.cf, g.pr, g.iden};
#pragma unroll
    for (int q = 0; q < S_N; ++q) bulk_load(sl + (size_t)q * nmax, src[q] + row + ib, bytes, bar);
}

// ---------------------------------------------------------------------------
// Thomas recurrences of one line by one warp, from shared-memory rows indexed
// by i - i0: e (right-hand side / den on entry, the solution on exit), cf and
// pr.  Each lane owns a contiguous chunk; the chunks are chained by warp scans
// of affine maps (x -> A x + B), forward for qr_i = cf_i qr_{i-1} + e_i and
// backward for phi_i = pr_i phi_{i+1} + qr_i; then the line is stored.  lo and
// hi are the fixed end values phi_{i0-1} and phi_{i1+1}.
template <typename T>
__device__ __forceinline__ void scan_line(T *phi, size_t row, int i0, int i1, T *se, const T *sc,
                                          const T *sp, T lo, T hi)
{
    const int lane = threadIdx.x & 31;
    const int n = i1 - i0 + 1;
    const int L = (n + 31) >> 5;
    const int a = lane * L;
    const int b = min(a + L, n);
    T A = T(1), B = T(0);
    for (int i = a; i < b; ++i) {
        const T cfi = sc[i];
        B = fma_rn(cfi, B, se[i]);
        A = mul_rn(cfi, A);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T A2 = __shfl_up_sync(0xffffffffu, A, o);
        T B2 = __shfl_up_sync(0xffffffffu, B, o);
        if (lane >= o) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    T Ae = __shfl_up_sync(0xffffffffu, A, 1);
    T Be = __shfl_up_sync(0xffffffffu, B, 1);
    if (lane == 0) { Ae = T(1); Be = T(0); }
    T q = fma_rn(Ae, lo, Be);
    for (int i = a; i < b; ++i) {
        q = fma_rn(sc[i], q, se[i]);
        se[i] = q;
    }
    A = T(1);
    B = T(0);
    for (int i = b - 1; i >= a; --i) {
        const T pri = sp[i];
        B = fma_rn(pri, B, se[i]);
        A = mul_rn(pri, A);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T A2 = __shfl_down_sync(0xffffffffu, A, o);
        T B2 = __shfl_down_sync(0xffffffffu, B, o);
        if (lane + o < 32) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    Ae = __shfl_down_sync(0xffffffffu, A, 1);
    Be = __shfl_down_sync(0xffffffffu, B, 1);
    if (lane == 31) { Ae = T(1); Be = T(0); }
    T x = fma_rn(Ae, hi, Be);
    for (int i = b - 1; i >= a; --i) {
        x = fma_rn(sp[i], x, se[i]);
        se[i] = x;
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) phi[row + i0 + i] = se[i];
}

// One x-line solved by one warp from its staged rows.  `row` is the offset of
// node (0, j, k); cells i0..i1 are unknowns, phi[i0-1] and phi[i1+1] the fixed
// ends; sl holds the line from cell ib on.  The right-hand side and the forward
// recurrence go to row `qrow` of sl: the source row S_SU itself (consumed), or
// the scratch row S_Q of a buffer that keeps the line's rows for later passes.
template <typename T, bool COHERENT>
__device__ __forceinline__ void solve_staged(T *phi, size_t row, int i0, int i1, int ib,
                                             size_t sj, size_t sk, T *sl, int nmax, int qrow = S_SU)
{
    const int lane = threadIdx.x & 31;
    const T *sat = sl + S_AT * nmax, *sab = sl + S_AB * nmax, *san = sl + S_AN * nmax,
            *sas = sl + S_AS * nmax, *ssu = sl + S_SU * nmax, *sc = sl + S_CF * nmax,
            *sp = sl + S_PR * nmax, *sid = sl + S_ID * nmax;
    T *se = sl + (size_t)qrow * nmax;
    auto ldp = [&](size_t c) -> T { return COHERENT ? ld_shared_row<T>(phi + c) : phi[c]; };
    // the line's fixed ends, loaded with the neighbour rows rather than in the
    // middle of the recurrences
    const T lo = ldp(row + i0 - 1), hi = ldp(row + i1 + 1);
    // right-hand side e_i = d_i / den_i, coalesced neighbour rows; four
    // iterations' neighbour loads are issued before any result is stored
    constexpr int U = 4;
    for (int i = ib + lane; i <= i1; i += 32 * U) {
        T nt[U], nb[U], nn[U], ns[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int iu = i + 32 * u;
            const bool ok = iu >= i0 && iu <= i1;
            const size_t c = row + (ok ? iu : i0);
            nt[u] = ok ? ldp(c + sk) : T(0);
            nb[u] = ok ? ldp(c - sk) : T(0);
            nn[u] = ok ? ldp(c + sj) : T(0);
            ns[u] = ok ? ldp(c - sj) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int iu = i + 32 * u;
            if (iu < i0 || iu > i1) continue;
            const int s = iu - ib;
            se[s] = line_rhs(sat[s], nt[u], sab[s], nb[u], san[s], nn[u], sas[s], ns[u], ssu[s], sid[s]);
        }
    }
    __syncwarp();
    const int o = i0 - ib;
    scan_line<T>(phi, row, i0, i1, se + o, sc + o, sp + o, lo, hi);
}

// ---------------------------------------------------------------------------
// A line's coefficient rows and factorisation held in registers across passes:
// lane l keeps cells a = l L .. a + L - 1 of the line (relative to i0), the
// chunk that scan_line gives a lane on a line of n cells when L = (n + 31) / 32.
// ---------------------------------------------------------------------------
template <typename T, int L>
struct LineRegs {
    T at[L], ab[L], an[L], as[L], su[L], cf[L], pr[L], id[L];
};
// One pass over a line of n <= 32 L cells from its registers: solve_staged and
// scan_line with the same expressions on the same per-lane chunks (so the same
// bits), the right-hand side and both recurrences in registers; only the four
// neighbouring rows and the two fixed ends are read (through L2: other CTAs
// write them), and the lane's cells are stored.
template <typename T, int L>
__device__ __forceinline__ void solve_line_regs(T *phi, size_t row, int i0, int n, size_t sj, size_t sk,
                                                const LineRegs<T, L> &r)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int a = lane * L;
    const T lo = ld_shared_row<T>(phi + row + i0 - 1), hi = ld_shared_row<T>(phi + row + i0 + n);
    T nt[L], nb[L], nn[L], ns[L], e[L];
#pragma unroll
    for (int v = 0; v < L; ++v) {
        const bool ok = a + v < n;
        const size_t c = row + i0 + (ok ? a + v : 0);
        nt[v] = ok ? ld_shared_row<T>(phi + c + sk) : T(0);
        nb[v] = ok ? ld_shared_row<T>(phi + c - sk) : T(0);
        nn[v] = ok ? ld_shared_row<T>(phi + c + sj) : T(0);
        ns[v] = ok ? ld_shared_row<T>(phi + c - sj) : T(0);
    }
#pragma unroll
    for (int v = 0; v < L; ++v)
        e[v] = line_rhs(r.at[v], nt[v], r.ab[v], nb[v], r.an[v], nn[v], r.as[v], ns[v], r.su[v], r.id[v]);
    T A = T(1), B = T(0);
#pragma unroll
    for (int v = 0; v < L; ++v)
        if (a + v < n) {
            B = fma_rn(r.cf[v], B, e[v]);
            A = mul_rn(r.cf[v], A);
        }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T A2 = __shfl_up_sync(full, A, o);
        T B2 = __shfl_up_sync(full, B, o);
        if (lane >= o) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    T Ae = __shfl_up_sync(full, A, 1);
    T Be = __shfl_up_sync(full, B, 1);
    if (lane == 0) { Ae = T(1); Be = T(0); }
    T q = fma_rn(Ae, lo, Be);
#pragma unroll
    for (int v = 0; v < L; ++v)
        if (a + v < n) {
            q = fma_rn(r.cf[v], q, e[v]);
            e[v] = q;
        }
    A = T(1);
    B = T(0);
#pragma unroll
    for (int v = L - 1; v >= 0; --v)
        if (a + v < n) {
            B = fma_rn(r.pr[v], B, e[v]);
            A = mul_rn(r.pr[v], A);
        }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T A2 = __shfl_down_sync(full, A, o);
        T B2 = __shfl_down_sync(full, B, o);
        if (lane + o < 32) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    Ae = __shfl_down_sync(full, A, 1);
    Be = __shfl_down_sync(full, B, 1);
    if (lane == 31) { Ae = T(1); Be = T(0); }
    T x = fma_rn(Ae, hi, Be);
#pragma unroll
    for (int v = L - 1; v >= 0; --v)
        if (a + v < n) {
            x = fma_rn(r.pr[v], x, e[v]);
            phi[row + i0 + a + v] = x;
        }
}

// ---------------------------------------------------------------------------
// One pass over an FP32 line of n <= 32 L cells from its registers, exchanging
// values with the neighbouring lines through a tagged copy: each cell's entry
// in `xc` is one 64-bit word, the value's bits low and a version tag high,
// stored in one access, so a reader sees a whole (value, tag) pair.  The pass
// reads the four neighbours of each of its cells: from `xc`, waiting (bounded)
// until the tag is `expect`, where the neighbouring line lies in the box (in_t,
// in_b, in_n, in_s), else from phi (fixed during the solve); the fixed ends
// from phi.  It stores its cells to `xc` with tag `expect` + 1 and, on the
// line's last pass (`last`), to phi.  No fence or flag: a value and its version
// travel together.  The arithmetic is solve_line_regs's.  False (for the whole
// warp) when a wait gave up or an error is raised.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long xtag(float v, unsigned tag)
{
    return ((unsigned long long)tag << 32) | __float_as_uint(v);
}
template <int L>
__device__ __forceinline__ bool solve_line_tagged(float *phi, unsigned long long *xc, size_t row, int i0, int n,
                                                  size_t sj, size_t sk, const LineRegs<float, L> &r, bool in_t,
                                                  bool in_b, bool in_n, bool in_s, unsigned expect, bool last,
                                                  Status *st, long long polls)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int a = lane * L;
    const float lo = ld_shared_row<float>(phi + row + i0 - 1), hi = ld_shared_row<float>(phi + row + i0 + n);
    const bool in[4] = {in_t, in_b, in_n, in_s};
    const long long off[4] = {(long long)sk, -(long long)sk, (long long)sj, -(long long)sj};
    unsigned long long q[4][L];
    float nv[4][L];
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
        for (int v = 0; v < L; ++v) {
            const bool ok = a + v < n;
            const size_t c = row + i0 + (ok ? a + v : 0) + off[d];
            q[d][v] = (ok && in[d]) ? __ldcg(xc + c) : xtag(0.f, expect);
            nv[d][v] = (ok && !in[d]) ? ld_shared_row<float>(phi + c) : 0.f;
        }
    // the whole warp polls together (a lane whose values have arrived waits for
    // the others in the vote), so that it leaves the loop converged: lanes
    // leaving one by one would run the scans below in as many divergent groups
    for (long long it = 0;; ++it) {
        bool ready = true;
#pragma unroll
        for (int d = 0; d < 4; ++d)
#pragma unroll
            for (int v = 0; v < L; ++v) ready = ready && (unsigned)(q[d][v] >> 32) == expect;
        if (__all_sync(full, ready)) break;
        if ((it & 63) == 63 && __any_sync(full, *(volatile int *)&st->error != 0)) return false;
        if (it > polls) {
            if (lane == 0 && atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = -5;
            return false;
        }
#pragma unroll
        for (int d = 0; d < 4; ++d)
#pragma unroll
            for (int v = 0; v < L; ++v)
                if ((unsigned)(q[d][v] >> 32) != expect) {
                    const size_t c = row + i0 + a + v + off[d];
                    q[d][v] = __ldcg(xc + c);
                }
    }
    float e[L];
#pragma unroll
    for (int v = 0; v < L; ++v) {
        float w[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) w[d] = in[d] ? __uint_as_float((unsigned)q[d][v]) : nv[d][v];
        e[v] = line_rhs(r.at[v], w[0], r.ab[v], w[1], r.an[v], w[2], r.as[v], w[3], r.su[v], r.id[v]);
    }
    float A = 1.f, B = 0.f;
#pragma unroll
    for (int v = 0; v < L; ++v)
        if (a + v < n) {
            B = fma_rn(r.cf[v], B, e[v]);
            A = mul_rn(r.cf[v], A);
        }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float A2 = __shfl_up_sync(full, A, o), B2 = __shfl_up_sync(full, B, o);
        if (lane >= o) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    float Ae = __shfl_up_sync(full, A, 1), Be = __shfl_up_sync(full, B, 1);
    if (lane == 0) { Ae = 1.f; Be = 0.f; }
    float x = fma_rn(Ae, lo, Be);
#pragma unroll
    for (int v = 0; v < L; ++v)
        if (a + v < n) {
            x = fma_rn(r.cf[v], x, e[v]);
            e[v] = x;
        }
    A = 1.f;
    B = 0.f;
#pragma unroll
    for (int v = L - 1; v >= 0; --v)
        if (a + v < n) {
            B = fma_rn(r.pr[v], B, e[v]);
            A = mul_rn(r.pr[v], A);
        }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float A2 = __shfl_down_sync(full, A, o), B2 = __shfl_down_sync(full, B, o);
        if (lane + o < 32) {
            B = fma_rn(A, B2, B);
            A = mul_rn(A, A2);
        }
    }
    Ae = __shfl_down_sync(full, A, 1);
    Be = __shfl_down_sync(full, B, 1);
    if (lane == 31) { Ae = 1.f; Be = 0.f; }
    x = fma_rn(Ae, hi, Be);
#pragma unroll
    for (int v = L - 1; v >= 0; --v)
        if (a + v < n) {
            x = fma_rn(r.pr[v], x, e[v]);
            const size_t c = row + i0 + a + v;
            xc[c] = xtag(x, expect + 1u);
            if (last) phi[c] = x;
        }
    return true;
}

// ---------------------------------------------------------------------------
// Thomas factorisation of one line by one warp: den_i = ap_i - aw_i pr_{i-1},
// pr_i = ae_i / den_i, cf_i = aw_i / den_i, iden_i = 1 / den_i from pr = 0
// before the first cell, with solveLiquidDomain's guard on |den|
// (CFDSolverManager.cpp:2438-2439).  The pivots follow the projective map
// x -> ae / (ap - aw x), the matrix [[0, ae], [-aw, ap]] on (x, 1): each lane
// multiplies the matrices of its chunk of L = (n + 31) / 32 cells (rescaled by
// powers of two, which is exact), an exclusive warp scan gives it the product of
// the lanes below, whose map applied to 0 is its entry pivot, and the lane then
// runs the recurrence over its own cells.  The guard acts in that recurrence, on
// the cell where it fires and the rest of its lane's chunk; the prefixes of the
// later lanes do not see it (it fires only on degenerate coefficients).  Every
// operation is explicitly rounded: the register and the memory forms below give
// the same bits.
// ---------------------------------------------------------------------------
template <typename T>
struct PMat {
    T a, b, c, d;  // [[a, b], [c, d]]
};
// Scale by the power of two that brings the largest entry into [1, 2): the
// exponent field of the largest magnitude gives it directly (entries that are
// zero, subnormal, infinite or NaN, or too large for the scale to be normal,
// are left alone).
__device__ __forceinline__ float pow2_inverse_scale(float mx, bool &ok)
{
    const unsigned eb = (__float_as_uint(mx) >> 23) & 0xffu;
    ok = eb >= 1u && eb <= 253u;
    return __uint_as_float((254u - eb) << 23);
}
__device__ __forceinline__ double pow2_inverse_scale(double mx, bool &ok)
{
    const unsigned long long eb = (unsigned long long)(__double_as_longlong(mx) >> 52) & 0x7ffull;
    ok = eb >= 1ull && eb <= 2045ull;
    return __longlong_as_double((long long)((2046ull - eb) << 52));
}
template <typename T>
__device__ __forceinline__ void pmat_rescale(PMat<T> &m)
{
    const T mx = fmax(fmax(fabs(m.a), fabs(m.b)), fmax(fabs(m.c), fabs(m.d)));
    bool ok;
    const T s = pow2_inverse_scale(mx, ok);
    if (ok) {
        m.a *= s; m.b *= s; m.c *= s; m.d *= s;
    }
}
// m <- [[0, e], [-w, p]] m
template <typename T>
__device__ __forceinline__ void pmat_cell(PMat<T> &m, T w, T e, T p)
{
    const PMat<T> r{mul_rn(e, m.c), mul_rn(e, m.d), fma_rn(p, m.c, mul_rn(-w, m.a)), fma_rn(p, m.d, mul_rn(-w, m.b))};
    m = r;
    pmat_rescale(m);
}
// The entry pivot of this lane: the product of the lanes below applied to 0.
template <typename T>
__device__ __forceinline__ T pmat_entry(PMat<T> m)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T ba = __shfl_up_sync(full, m.a, o), bb = __shfl_up_sync(full, m.b, o);
        const T bc = __shfl_up_sync(full, m.c, o), bd = __shfl_up_sync(full, m.d, o);
        if (lane >= o) {  // own x lower
            const PMat<T> r{fma_rn(m.a, ba, mul_rn(m.b, bc)), fma_rn(m.a, bb, mul_rn(m.b, bd)),
                            fma_rn(m.c, ba, mul_rn(m.d, bc)), fma_rn(m.c, bb, mul_rn(m.d, bd))};
            m = r;
            pmat_rescale(m);
        }
    }
    const T eb = __shfl_up_sync(full, m.b, 1), ed = __shfl_up_sync(full, m.d, 1);
    return lane == 0 ? T(0) : eb / ed;
}
// One cell of the recurrence from the previous pivot x (updated to this cell's pr).
template <typename T>
__device__ __forceinline__ void factor_cell(T w, T e, T p, T &x, T &pr, T &cf, T &id)
{
    T den = fma_rn(-w, x, p);
    if (fabs(den) <= T(1e-12)) den += T(kSmall);
    id = T(1) / den;
    pr = mul_rn(e, id);
    cf = mul_rn(w, id);
    x = pr;
}
// The warp's line from registers: lane l holds cells l L .. l L + L - 1 (n <= 32 L).
template <typename T, int L>
__device__ __forceinline__ void factor_line_regs(int n, const T (&w)[L], const T (&e)[L], const T (&p)[L],
                                                 T (&pr)[L], T (&cf)[L], T (&id)[L])
{
    const int a = (threadIdx.x & 31) * L;
    PMat<T> m{T(1), T(0), T(0), T(1)};
#pragma unroll
    for (int v = 0; v < L; ++v)
        if (a + v < n) pmat_cell(m, w[v], e[v], p[v]);
    T x = pmat_entry(m);
#pragma unroll
    for (int v = 0; v < L; ++v) {
        pr[v] = cf[v] = id[v] = T(0);
        if (a + v < n) factor_cell(w[v], e[v], p[v], x, pr[v], cf[v], id[v]);
    }
}
// A line's coefficients from global memory (cell i0 of the line at offset c0)
// into the registers of its warp; aw, ae, ap into `f` for the factorisation
// (factor_line_regs), which the caller runs once the loads of all its lines are
// in flight.
template <typename T, int L>
struct LineFetch {
    T w[L], e[L], p[L];
};
template <typename T, int L>
__device__ __forceinline__ void load_line_regs(LineRegs<T, L> &r, LineFetch<T, L> &f, const Fields<T> &g,
                                               size_t c0, int n)
{
    const int a = (threadIdx.x & 31) * L;
    T (&w)[L] = f.w;
    T (&e)[L] = f.e;
    T (&p)[L] = f.p;
#pragma unroll
    for (int v = 0; v < L; ++v) {
        const bool ok = a + v < n;
        const size_t c = c0 + (ok ? a + v : 0);
        r.at[v] = ok ? g.at[c] : T(0);
        r.ab[v] = ok ? g.ab[c] : T(0);
        r.an[v] = ok ? g.an[c] : T(0);
        r.as[v] = ok ? g.as[c] : T(0);
        r.su[v] = ok ? g.su[c] : T(0);
        w[v] = ok ? g.aw[c] : T(0);
        e[v] = ok ? g.ae[c] : T(0);
        p[v] = ok ? g.ap[c] : T(1);
    }
}

// The warp's line through accessors: get(i, aw, ae, ap) reads cell i (0-based),
// put(i, pr, cf, iden) writes it.  The same operations as factor_line_regs.
template <typename T, class Get, class Put>
__device__ __forceinline__ void factor_line_mem(int n, Get get, Put put)
{
    const int L = (n + 31) >> 5;
    const int a = min((threadIdx.x & 31) * L, n), b = min(a + L, n);
    PMat<T> m{T(1), T(0), T(0), T(1)};
    for (int i = a; i < b; ++i) {
        T w, e, p;
        get(i, w, e, p);
        pmat_cell(m, w, e, p);
    }
    T x = pmat_entry(m);
    for (int i = a; i < b; ++i) {
        T w, e, p, pr, cf, id;
        get(i, w, e, p);
        factor_cell(w, e, p, x, pr, cf, id);
        put(i, pr, cf, id);
    }
}

// Aligned staging window [ib, ie) of cells i0..i1 (16-byte units).
template <typename T>
__device__ __forceinline__ void stage_window(int i0, int i1, int &ib, int &ie)
{
    constexpr int V = 16 / sizeof(T);
    ib = i0 & ~(V - 1);
    ie = (i1 + 1 + V - 1) & ~(V - 1);
}

template <bool BOX>
__device__ __forceinline__ void box_of(const Params &p, const Status *st, int &i0, int &i1,
                                       int &j0, int &j1, int &k0, int &k1)
{
    if (BOX) {
        i0 = st->istatp1; i1 = st->iendm1; j0 = st->jstat; j1 = st->jend; k0 = st->kstat; k1 = p.nkm2;
    } else {
        i0 = 1; i1 = p.nim2; j0 = 1; j1 = p.njm2; k0 = 1; k1 = p.nkm2;
    }
}

// GPU-scope acquire / release accesses of the grid barrier's words.
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned *p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(unsigned *p, unsigned v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// Barrier over the first n CTAs of a cooperative launch (all co-resident).
// Thread 0 of each CTA arrives with an acquire-release add on the count; the
// last to arrive resets the count and publishes generation `target` with a
// release store; the others poll the generation with acquire loads, at most
// `limit` times, then record AMCFD_E_TIMEOUT (detail `where`).  Each CTA counts
// the generations itself (the value at its start plus the barriers it has
// passed).  Writes of a CTA before the barrier are visible to every CTA after
// it: the CTA barrier orders them before thread 0's release, the chain of
// read-modify-writes on the count carries every arrival to the last one, and
// its release of the generation to every acquire that reads it.  False once a
// device error is raised; a context whose device wait gave up stays failed, so
// the count left behind by an abandoned barrier is never used again.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *gen, unsigned target, unsigned n,
                                             Status *st, long long limit, int where)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        if (atom_add_acq_rel_gpu(count, 1u) == n - 1) {
            st_relaxed_gpu(count, 0u);
            st_release_gpu(gen, target);
        } else {
            long long it = 0;
            while ((int)(ld_acquire_gpu(gen) - target) < 0) {
                if ((it & 63) == 63 && *(volatile int *)&st->error) { ok = 0; break; }
                if (++it > limit) {
                    if (atomicCAS(&st->error, 0, AMCFD_E_TIMEOUT) == 0) st->error_where = where;
                    ok = 0;
                    break;
                }
            }
        }
        ok_s = ok;
    }
    __syncthreads();
    __syncwarp();  // thread 0's warp leaves converged
    return ok_s != 0;
}

// A kernel's dynamic shared-memory limit is one value per process, shared by every
// context: it is only ever raised, so that a context with a smaller grid never
// lowers it under what another context's launches need.
static inline cudaError_t raise_smem_limit(const void *func, size_t need)
{
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, func);
    if (e != cudaSuccess) return e;
    if ((int)need <= a.maxDynamicSharedSizeBytes) return cudaSuccess;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
}

}  // namespace amcfd
