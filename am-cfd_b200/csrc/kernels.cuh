// Geometry helpers, the host-side instance record and the kernel launchers.
#pragma once
#include <cuda.h>
#include <cstdio>
#include <utility>
#include "dev.cuh"

namespace amcfd {

// Face areas and control volumes (CFDSolverManager.cpp:243-286), recomputed
// from the 1-D metrics with the reference's products.  The reference arrays
// are only filled for interior indices and are zero elsewhere; so are these.
template <typename T>
__device__ __forceinline__ double area_ij(const Params &p, const Fields<T> &g, int i, int j)
{
    if (i < 1 || i > p.nim2 || j < 1 || j > p.njm2) return 0.0;
    return (g.xu[i + 1] - g.xu[i]) * (g.yv[j + 1] - g.yv[j]);
}
template <typename T>
__device__ __forceinline__ double area_ik(const Params &p, const Fields<T> &g, int i, int k)
{
    if (i < 1 || i > p.nim2 || k < 1 || k > p.nkm2) return 0.0;
    return (g.xu[i + 1] - g.xu[i]) * (g.zw[k + 1] - g.zw[k]);
}
template <typename T>
__device__ __forceinline__ double area_jk(const Params &p, const Fields<T> &g, int j, int k)
{
    if (j < 1 || j > p.njm2 || k < 1 || k > p.nkm2) return 0.0;
    return (g.yv[j + 1] - g.yv[j]) * (g.zw[k + 1] - g.zw[k]);
}
template <typename T>
__device__ __forceinline__ double volume_p(const Params &p, const Fields<T> &g, int i, int j, int k)
{
    return (g.xu[i + 1] - g.xu[i]) * (g.yv[j + 1] - g.yv[j]) * (g.zw[k + 1] - g.zw[k]);
}
// staggered-cell areas/volumes of the momentum equations
template <typename T>
__device__ __forceinline__ double area_uij(const Fields<T> &g, int i, int j)
{ return (g.x[i] - g.x[i - 1]) * (g.yv[j + 1] - g.yv[j]); }
template <typename T>
__device__ __forceinline__ double area_vij(const Fields<T> &g, int i, int j)
{ return (g.xu[i + 1] - g.xu[i]) * (g.y[j] - g.y[j - 1]); }
template <typename T>
__device__ __forceinline__ double area_uik(const Fields<T> &g, int i, int k)
{ return (g.x[i] - g.x[i - 1]) * (g.zw[k + 1] - g.zw[k]); }
template <typename T>
__device__ __forceinline__ double area_wik(const Fields<T> &g, int i, int k)
{ return (g.xu[i + 1] - g.xu[i]) * (g.z[k] - g.z[k - 1]); }
template <typename T>
__device__ __forceinline__ double area_vjk(const Fields<T> &g, int j, int k)
{ return (g.y[j] - g.y[j - 1]) * (g.zw[k + 1] - g.zw[k]); }
template <typename T>
__device__ __forceinline__ double area_wjk(const Fields<T> &g, int j, int k)
{ return (g.yv[j + 1] - g.yv[j]) * (g.z[k] - g.z[k - 1]); }
template <typename T>
__device__ __forceinline__ double volume_u(const Fields<T> &g, int i, int j, int k)
{ return (g.x[i] - g.x[i - 1]) * (g.yv[j + 1] - g.yv[j]) * (g.zw[k + 1] - g.zw[k]); }
template <typename T>
__device__ __forceinline__ double volume_v(const Fields<T> &g, int i, int j, int k)
{ return (g.xu[i + 1] - g.xu[i]) * (g.y[j] - g.y[j - 1]) * (g.zw[k + 1] - g.zw[k]); }
template <typename T>
__device__ __forceinline__ double volume_w(const Fields<T> &g, int i, int j, int k)
{ return (g.xu[i + 1] - g.xu[i]) * (g.yv[j + 1] - g.yv[j]) * (g.z[k] - g.z[k - 1]); }

// TMA tensor maps of the fields the energy assembly stages (k_assemble.cu).
struct AsmMaps {
    CUtensorMap diff, h, fracl, rho, w, u, v, temp, hnot, flnot;
};

// Defect-correction buffers (AMCFD_PREC_FP32_DC, FP64 instances only): the
// energy coefficients rounded to FP32, with `su` holding the FP64 defect
// su + sum a_nb h_nb - ap h of the current enthalpy instead of the source; the
// FP32 line factorisation; and the FP32 enthalpy correction `delta` the line
// sweeps solve for (zero on every boundary node, never written there).
struct DcBuf {
    float *an, *as, *ae, *aw, *at, *ab, *ap, *su, *pr, *cf, *iden, *delta;
};

// Host-side record of one instance on the device.
template <typename T>
struct Inst {
    Params p;
    Fields<T> g;
    cudaStream_t stream = nullptr;
    int sm_count = 148;
    int order = 0;
    int check_finite = 0;
    // reduction regions (per-CTA partials)
    double *red_las = nullptr, *red_bc = nullptr, *red_asm = nullptr, *red_h2t = nullptr,
           *red_mom = nullptr;
    int nb_las = 0, nb_bc = 0, nb_asm = 0, nb_h2t = 0, nb_mom = 0;
    dim3 asm_grid;
    int grid_1d = 0;          // grid of the pointwise kernels
    int exact_grid = 0;       // CTAs of the persistent exact-order line sweep
    int exact_warps = 4;      // warps per CTA in the line sweeps
    size_t line_smem = 0;     // dynamic smem of a line-sweep CTA
    int *flags_mom = nullptr;
    int max_lines = 0;        // (nj-2)*(nk-2)
    AsmMaps asm_maps[2];      // by property parity
    T *mom_scratch = nullptr; // one field: line-solve scratch of the small-box momentum path
    size_t mom_small_smem = 0;  // its dynamic shared memory
    int mom_cluster = 0;        // CTAs of the cluster that takes boxes past one CTA's shared memory
                                // (set by setup_mom_small from the request here: 0 = default)
    // launch shapes picked by the autotuner (or pinned by the options)
    int asm_kseg = 0;           // planes per CTA of the energy assembly (0: the default rule)
    int sweep_warps = 4;        // warps (lines) per CTA of the whole-domain red-black sweeps
    int sweep_warps_max = 4;    // the most whose line buffers fit a CTA's shared memory
    const T *asm_diff_a = nullptr;  // diff_cur at parity 0
    // updateSolutions inputs of the current step (powder bed)
    double trackindx = 1.0;
    int trackid = 0;
    // defect correction of the energy line solves (FP64 instances only)
    bool dc_on = false;
    DcBuf dc{};
    // launches of the outer iteration overlap the end of the kernel before them
    // (programmatic dependent launch, launch_k)
    bool pdl = true;
    // cooperative red-black line solve of the momentum box (box_grid 0: the
    // multi-launch form): CTAs, warps per CTA, dynamic shared memory
    int box_grid = 0, box_warps = 4;
    size_t box_smem = 0;
    // FP32 box lines' values exchanged between passes with a version tag (one
    // 64-bit word per node of the grid)
    unsigned long long *xchg = nullptr;
    // the whole-domain red-black passes of a solve as one pipelined launch
    // (pipe_grid 0: a launch per pass): CTAs, warps per CTA, planes between the
    // passes in the work order, dynamic shared memory, per-line pass flags;
    // pipe_*_dc: the FP32 correction sweeps of defect correction.  Measured on the
    // 400x200x100 deck (FP32, ms per solve): stride 2: 0.567, 4: 0.386, 6: 0.338,
    // 8: 0.320, 12-32: 0.312-0.315, 128: 0.317; a launch per pass 0.344
    int pipe_grid = 0, pipe_warps = 8, pipe_grid_dc = 0, pipe_stride = 16;
    size_t pipe_smem = 0, pipe_smem_dc = 0;
    int *flags_pipe = nullptr;
};

// Launch of a kernel that begins with pdl_enter().  With `pdl` the launch carries
// programmatic stream serialisation: it may start while the kernel before it in
// the stream drains (the kernel's pdl_enter waits for that kernel's completion).
template <typename... K, typename... A>
inline void launch_k(bool pdl, void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                     A &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    if (pdl) {
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
    }
    cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// launchers (k_energy.cu)
template <typename T> void launch_laser(Inst<T> &I);
template <typename T> void launch_energy_bc(Inst<T> &I);
template <typename T> void launch_energy_assemble(Inst<T> &I);
template <typename T> int make_assemble_maps(Inst<T> &I, T *diff_a, T *diff_b, T *rho_a, T *rho_b);
template <typename T> void launch_block_correct(Inst<T> &I, int ivar = 5);
template <typename T> void launch_h2t(Inst<T> &I);
template <typename T> void launch_meltpool(Inst<T> &I);
template <typename T> void launch_converge(Inst<T> &I, double tol, const LoopCtl &lc = LoopCtl{});
void launch_loop_init(Status *st, const LoopCtl &lc, cudaStream_t s);
template <typename T> void launch_update_solutions(Inst<T> &I);
// line solvers (k_linesolve.cu)
template <typename T> void launch_energy_factor(Inst<T> &I);
template <typename T> void launch_energy_sweeps(Inst<T> &I);
template <typename T> void launch_sweep_probe(Inst<T> &I, T *phi, int warps);
template <typename T> void launch_phi_factor(Inst<T> &I, T *phi);   // whole-domain phi
template <typename T> void launch_phi_sweeps(Inst<T> &I, T *phi);
template <typename T> void launch_box_factor(Inst<T> &I);
template <typename T> void launch_box_sweeps(Inst<T> &I, int ivar);
template <typename T> void setup_box_solve(Inst<T> &I, bool enable);
template <typename T> void launch_box_tickets(Inst<T> &I);
// defect correction: the energy line sweeps in FP32 on the correction, and h += delta
void launch_dc_sweeps(Inst<double> &I);
void launch_dc_sweep_probe(Inst<double> &I, int warps);
void launch_dc_apply(Inst<double> &I);
// momentum (k_momentum.cu)
template <typename T> void launch_momentum(Inst<T> &I, bool small);
template <typename T> int mom_small_capacity(const Inst<T> &I);
template <typename T> void setup_mom_small(Inst<T> &I);
// species (k_species.cu)
template <typename T> void launch_species(Inst<T> &I);
template <typename T> void launch_species_update(Inst<T> &I);
// moving mesh and solidification parameters (k_mesh.cu)
template <typename T> void launch_remap(Inst<T> &I, const double *oldx, const double *oldy, int dirx, int diry);
template <typename T> void launch_solidification(Inst<T> &I, double scanvel);
// energy-balance free surface (k_freesurf.cu)
struct FsIn {
    double lam1, lam2, gamma, c1, urf, tol_e, tol_b, vd;
    int maxit_e, maxit_b;
};
struct FsOut {
    double xmid, fmid, fimin, fimax;
    int niter, bracketed;
};
template <typename T> void launch_free_surface(Inst<T> &I, const FsIn &a, FsOut *out_dev);

}  // namespace amcfd
