// Device-side data layout and helpers shared by the solver kernels.
//
// Layout: every 3-D field is a structure-of-arrays buffer indexed
// (k*nj + j)*nip + i, i fastest, with the i-pitch nip padded to a multiple of
// 32 elements so that every x-line starts on a 256-byte boundary (FP64).
// The reference uses the same [k][j][i] order with an unpadded pitch
// (CFDSolverManager.cpp:249).  Geometry is kept as 1-D FP64 metrics; volumes
// and face areas are recomputed in the kernels with the reference's own
// products (CFDSolverManager.cpp:243-286), so they are bit-identical to the
// reference arrays.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace amcfd {

constexpr double kSmall = 1.0e-6;  // CFDSolverManager.h:143
constexpr double kLarge = 1.0e20;  // CFDSolverManager.h:144

// std::max / std::min with the reference's NaN behaviour.
__host__ __device__ __forceinline__ double maxd(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double mind(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float maxd(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float mind(float a, float b) { return (b < a) ? b : a; }

// Scalar parameters of one instance (DomainManager/Mesh fields read by the hot path).
struct Params {
    int ni, nj, nk, nip;
    int nim1, njm1, nkm1, nim2, njm2, nkm2;
    double dens, denl, viscos, tsolid, tliquid, hsmelt, hlcal, hlatnt, acpa, acpb, acpl;
    double thconsa, thconsb, thconsc, thconla, thconlb;
    double urfu, urfv, urfw, urfp, urfh;
    double htci, htcj, htckn, emiss, sigm, tempamb;
    double beta, grav, dgdtp, darcyKo, a_oxygen;
    double alaspow, alaseta, alasrb, alasfact;
    double pressamb, gasconst, evaplatent, evaptemp, evapfact, molarmass;
    int isevap, scheme, steady, navierstokes;
    int nheattable;
    int volsrc;  // a volumetric source is configured (scalar form with heatthick > 0, or a table)
    double avolpow, apowseta, heatthick, heatrb, avolfact;  // scalar volumetric source
    int species;  // *SOLVE_SPECIES: the ivar = 6 equation is solved
    double initconc, massdiff, kp, urfc;
    // *POWDER_BED_MODE: effective powder properties (powderMaterialProps); nk above
    // is the active domain, nk_alloc the planes every 3-D array holds
    int powder, nk_alloc;
    double powderden, powdercpa, powdercpb, powderthcona, powderthconb;
    // polls of one bounded wait on another warp's line counter before the wait
    // gives up with AMCFD_E_TIMEOUT (exact-order sweeps)
    long long wait_polls;
};

// Device status block: per-step inputs written by the host, per-iteration
// results written by the kernels (reductions are FP64).
struct Status {
    // per step
    double timet, delt, beamposx, beamposy, scanvel;
    // device-driven outer loop: iterations run in this step, momentum-box cells of
    // the last one (-1: none yet), momentum path of the current one (1: small box)
    // and iterations that took the small-box path
    int lp_niter, lp_box, lp_mode, lp_small;
    int powerindicator, istart, jstart, heat_iter;
    double heatinlaser;
    // current volumetric-source parameters (advanced per outer iteration)
    double avolpow, apowseta, heatthick, heatrb, avolfact;
    // per outer iteration
    double ahtoploss, resorh, tpeak, alen, depth, width, ratio, accul, heatvol, heatout;
    double fluxwest, fluxeast, fluxtop, fluxbottom, fluxnorth, fluxsouth;
    double resoru, resorv, resorw, resorm, refmom, umaxt, mass_denom;
    double resorc;  // species residual (0 without *SOLVE_SPECIES)
    int istat, iend, jstat, jend, kstat, istatp1, iendm1;
    int imin, imax, jmin, jmax, kmin, kmax;
    int momentum_active, box_cells;
    int mp_imax, mp_imin;  // melt-pool length scan candidates, gathered by h2t_kernel
    int niter, itertot, converged;
    int error;         // 0, or an AMCFD_E_* code set by a kernel
    int error_where;   // kernel-specific detail (e.g. the line that timed out)
    int nonfinite;     // a reduction produced NaN/Inf
    unsigned long long seq_energy, done_energy, ticket_energy;
    unsigned long long seq_mom, done_mom, ticket_mom;
    // grid barrier of the cooperative momentum-box solve: arrivals, generation;
    // its line-flag epochs: launch sequence number, CTAs done with the passes
    unsigned gbar_count, gbar_gen, gflag_seq, gflag_done;
    // pipelined red-black sweep (all passes in one launch): launch sequence number,
    // CTAs done, next work ticket
    unsigned long long seq_pipe, done_pipe, ticket_pipe;
};

// Outer-loop control of a step captured as one CUDA graph (a chain of
// conditional nodes): the convergence kernel of iteration k sets whether
// iteration k+1 runs and which momentum path it takes.  active = 0 outside such
// a graph; has_next = 0 for the last iteration of the chain.
struct LoopCtl {
    cudaGraphConditionalHandle cont, mode_next;
    int active, has_next, maxit, cap;  // cap: small-box capacity in cells, -1 when disabled
};

// Fixed-size reduction slots written per CTA and reduced in a fixed order.
enum RedSlot {
    R_SUMD = 0, R_SUMH, R_AHTOP, R_ACCUL, R_HEATVOL, R_FW, R_FE, R_FB, R_FT, R_FS, R_FN,
    R_HEATIN, R_MSUMD, R_MDENOM, R_MRESORM, R_UMAX, R_TPEAK, R_NSLOTS
};

template <typename T>
struct Fields {
    // 1-D metrics (FP64)
    const double *x, *y, *z, *xu, *yv, *zw, *dxpwinv, *dypsinv, *dzpbinv, *fracx, *fracy, *fracz;
    // 3-D fields
    T *uvel, *vvel, *wvel, *unot, *vnot, *wnot, *pressure, *pp;
    T *h, *hnot, *temp, *fracl, *fraclnot, *sourceinput;
    T *diff_cur, *rho_cur, *vis_cur, *diff_nxt, *rho_nxt, *vis_nxt;
    // coefficients (shared by all equations, as in the reference)
    T *an, *as, *ae, *aw, *at, *ab, *ap, *su, *apnot, *sp;
    // pass-invariant line factorisation: pr = ae/den, cf = aw/den, iden = 1/den
    T *pr, *cf, *iden;
    T *dux, *dvy, *dwz;
    // species (null without *SOLVE_SPECIES): avgconcentration, its previous-step
    // value and the liquid concentration of updateSolutions
    T *conc, *concnot, *concn;
    // powder bed (null otherwise): consolidated fraction, solidified-track marker and
    // the track id of the last solid / liquid pass (updateSolutions)
    T *csfrac, *solfrac, *mpphase, *mpliq;
    // solidification parameters (null otherwise): temperature gradient G and growth rate R
    T *grad, *rate;
    // energy-balance free surface (null otherwise): deflection fi and its iterate
    // ([j][nip], FP64), deformed heights zr and the temperatures on them
    double *fs_fi, *fs_zz;
    T *fs_zr, *fs_tempr;
    double *heatin;     // nj*nip, Gaussian surface flux of the current step
    double *heattable;  // nheattable x 6
    // reductions
    double *red;        // [nblocks][R_NSLOTS] per-CTA partials
    double *bc;         // block correction: [npart][4][nip] per-CTA partial sums
    double *bcsum;      // [4][nip] reduced sums
    double *delphi;     // nip
    int npart;          // number of block-correction partial rows
    // melt-pool column scans (getMeltPoolShape), gathered with integer atomics by
    // h2t_kernel: per column i the deepest k with T < Ts on the beam plane, and the
    // first/last j around the beam with T < Ts on the top plane
    int *mp_kb, *mp_jup, *mp_jdn;
    // exact-order line sweep scheduling
    int *flags;         // (nk*nj) per-line visit counters (monotone across calls)
    int2 *tickets_energy;  // precomputed topological order of the energy visits
    int ntickets_energy;
    int2 *tickets_mom;     // regenerated on the device for each momentum box
    int *ntickets_mom;
    Status *st;
};

__host__ __device__ __forceinline__ size_t cidx(int i, int j, int k, int nj, int nip)
{
    return ((size_t)k * nj + j) * (size_t)nip + i;
}

// Division in the bulk precision: IEEE in FP64 (the parity build), the fast
// approximate reciprocal form in FP32 (about 2 ulp; the FP32 build is checked
// against the FP64 oracle, not bit for bit).
__device__ __forceinline__ double bdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float bdiv(float a, float b) { return __fdividef(a, b); }

// Discretisation scheme A(|Pe|) (CFDSolverManager.cpp:3071-3101).
template <typename R>
__device__ __forceinline__ R scheme_fn(int scheme, R pe)
{
    if (scheme == 1) {
        R base = R(1) - R(0.1) * pe;
        R out = base;
#pragma unroll
        for (int q = 1; q < 5; q++) out *= base;
        return maxd(R(0), out);
    }
    if (scheme == 2) return pe / (exp(pe) - R(1));
    return R(1);
}

// a_nb pair for one face: plus = D*A(|F|/D) + max(0,-F), minus = D*A(|F|/D) + max(0,F).
template <typename R>
__device__ __forceinline__ void face_coef(int scheme, R d, R f, R &plus, R &minus)
{
    R a = d * scheme_fn<R>(scheme, bdiv(fabs(f), d));
    plus = a + maxd(R(0), -f);
    minus = a + maxd(R(0), f);
}

// Warp sum / max of doubles with a fixed shuffle tree (deterministic).
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block reduction of up to 8 values into red[blk*R_NSLOTS + slot[q]] (sum or max).
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], const int (&slot)[NV],
                                                   const bool (&is_max)[NV], double *red,
                                                   int blk)
{
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31;
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = is_max[q] ? warp_max(v[q]) : warp_sum(v[q]);
    if ((tid & 31) == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) sh[warp][q] = v[q];
    }
    __syncthreads();
    if (tid < 32) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = (lane < nwarps) ? sh[lane][q] : (is_max[q] ? -INFINITY : 0.0);
            x = is_max[q] ? warp_max(x) : warp_sum(x);
            if (lane == 0) red[(size_t)blk * R_NSLOTS + slot[q]] = x;
        }
    }
    (void)tid;
}

// N sums of per-CTA partials (item q: slot slot[q] of the nb entries at base[q]) in
// one pass, each in the order of a one-slot reduction with one CTA: strided
// partial sums per thread, a warp shuffle tree, then warp 0 over the warps' sums.
// The loads of all items are in flight together.  scr holds N * 33 doubles.
template <int N>
__device__ void reduce_sums(const double *const (&base)[N], const int (&slot)[N], int nb, double (&out)[N],
                            double *scr)
{
    double acc[N];
#pragma unroll
    for (int q = 0; q < N; ++q) acc[q] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < N; ++q) acc[q] = acc[q] + base[q][(size_t)b * R_NSLOTS + slot[q]];
    }
#pragma unroll
    for (int q = 0; q < N; ++q) acc[q] = warp_sum(acc[q]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < N; ++q) scr[q * 33 + warp] = acc[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < N; ++q) {
            double r = lane < nw ? scr[q * 33 + lane] : 0.0;
            r = warp_sum(r);
            if (lane == 0) scr[q * 33 + 32] = r;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; ++q) out[q] = scr[q * 33 + 32];
    __syncthreads();
}

// One aligned 16-byte vector of a field (4 FP32 or 2 FP64 elements): the unit of
// the coalesced row loads of the line-sweep, factorisation and H->T kernels.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

template <typename T>
__device__ __forceinline__ void ld16(const T *ptr, T (&o)[16 / sizeof(T)])
{
    const typename Vec16<T>::type v = *reinterpret_cast<const typename Vec16<T>::type *>(ptr);
    memcpy(o, &v, 16);
}

// Bounded spin budget for every device-side wait (about one second).
constexpr long long kSpinLimit = 1ll << 24;

// Programmatic dependent launch.  Every kernel of the outer iteration calls this
// before it touches memory.  Launched with programmatic stream serialisation
// (launch_k), it waits here until the kernel before it in the stream has
// completed and that kernel's writes are visible, then releases the launch of
// the kernel after it, whose CTAs become resident and wait in their own
// pdl_enter: a launch's latency overlaps the run of the kernel before it instead
// of following its drain.  Launched without the attribute, both instructions
// return at once.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace amcfd
