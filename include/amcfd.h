/*
 * amcfd.h -- C ABI of the B200 melt-pool solver (libamcfd_b200.so).
 *
 * The reference AM-CFD exposes no library API: its boundary is the
 * `AM-CFD <deck.k>` process (src/main.cpp:25-52) and, in-process, the public
 * methods of CFDSolverManager (src/headers/CFDSolverManager.h:96-104) that
 * main() calls once per time step.  Each entry point below names the
 * reference interface it replaces.  All functions return 0 on success and a
 * negative AMCFD_E* code on failure; amcfd_last_error() gives the message.
 * Host buffers belong to the caller, device memory to the context; a context
 * is used from one host thread and owns one CUDA stream.
 */
#ifndef AMCFD_H
#define AMCFD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AMCFD_OK 0
#define AMCFD_E_ARG -1        /* invalid argument or unsupported option */
#define AMCFD_E_IO -2         /* deck, mesh or toolpath file missing/unreadable */
#define AMCFD_E_PARSE -3      /* malformed deck row */
#define AMCFD_E_CUDA -4       /* CUDA runtime error */
#define AMCFD_E_NONFINITE -5  /* NaN/Inf detected in a residual or field reduction */
#define AMCFD_E_TIMEOUT -6    /* a bounded device-side wait gave up */
#define AMCFD_E_NOMEM -7      /* device allocation failed */
#define AMCFD_E_CAPACITY -8   /* size beyond a fixed capacity */

#define AMCFD_MAX_ZONES 32

/* Discretisation scheme, *SELECT_DISCRETIZATION (Mesh.cpp:378-392). */
#define AMCFD_SCHEME_UPWIND 0
#define AMCFD_SCHEME_POWER_LAW 1
#define AMCFD_SCHEME_EXPONENTIAL 2

/*
 * Solver parameters: the DomainManager / Mesh fields that the hot path reads
 * (DomainManager.h:25-72, Mesh.h:22-71), already mapped from the deck by
 * DomainManager::assignInputValues (DomainManager.cpp:29-263).
 */
typedef struct amcfd_params {
    /* grid zones (DomainManager.cpp:33-46): length, control volumes, exponent */
    int nzx, nzy, nzz;
    double xzone[AMCFD_MAX_ZONES], ncvx[AMCFD_MAX_ZONES], powrx[AMCFD_MAX_ZONES];
    double yzone[AMCFD_MAX_ZONES], ncvy[AMCFD_MAX_ZONES], powry[AMCFD_MAX_ZONES];
    double zzone[AMCFD_MAX_ZONES], ncvz[AMCFD_MAX_ZONES], powrz[AMCFD_MAX_ZONES];
    /* material (DomainManager.cpp:59-73) */
    double dens, denl, viscos, tsolid, tliquid, hsmelt, hlfriz, acpa, acpb, acpl;
    double thconsa, thconsb, thconsc, thconla, thconlb;
    /* under-relaxation (:76-80) */
    double urfu, urfv, urfw, urfp, urfh;
    /* energy boundary conditions and boundary temperatures (:83-94) */
    double htci, htcj, htck1, htckn, emiss;
    double tempwest, tempeast, tempnorth, tempbottom, temppreheat;
    /* momentum boundary conditions (:97-100) */
    double beta, dgdtp, darcyKo, a_oxygen;
    /* *PARAMETERS (Mesh.cpp:440-470) */
    double grav, sigm, tempamb, pressamb, gasconst;
    /* Gaussian surface source (:105-108) */
    double alaspow, alaseta, alasrb, alasfact;
    /* single track (:51-54): laser-on time, start point, scan speed */
    double lasertime, xstart, ystart, scanvel;
    /* scalar volumetric source (:169-173); heatthick = 0 disables it */
    double avolpow, apowseta, heatthick, heatrb, avolfact;
    /* *BOUNDARY_EVAPORATION (DomainManager.cpp:113-120); isevap = 0 when absent */
    int isevap;
    double evaplatent, evaptemp, evapfact, molarmass;
    /* time control (Mesh.cpp:284-299) */
    double delt, outtime, finaltime, nonlintol;
    int maxit;
    int scheme;          /* AMCFD_SCHEME_* */
    int navierstokes;    /* 0 when *FLUID_FLOW_OFF */
    int steady;          /* delt >= 100 (DomainManager.cpp:203-210) */
    /* *TOOLPATH_FILE rows (DomainManager.cpp:276-286); udtoolpath = 0 for a single track */
    int udtoolpath;
    int ntool;
    const double *tool_txyz; /* ntool x 4: t, x, y, z */
    const int *tool_on;      /* ntool: laser-on flag of the segment ending at the row */
    const int *tool_id;      /* ntool: track id */
    /* *VOLUMETRIC_HEAT_SOURCE_TABLE rows (t, avolpow, apowseta, heatthick, heatrb, avolfact),
     * read per outer iteration by calculateSource(5) (CFDSolverManager.cpp:1707-1717) */
    int nheattable;
    const double *heattable; /* nheattable x 6 */
    /* *CONTROL_TIMESTEP_VARIABLE rows (t, delt, outtime), applied per step (main.cpp:125-134) */
    int nvardt;
    const double *vardt;     /* nvardt x 3 */
    /* optional features (all solved) */
    int powderbed, movingmesh, species, freesurface;
    /* *SOLVE_SPECIES row (DomainManager.cpp:123-129): initial concentration, mass
     * diffusivity, partition coefficient kp, under-relaxation factor urfc */
    double initconc, massdiff, kp, urfc;
    /* *POWDER_BED_MODE row (DomainManager.cpp:147-158): layers, control volumes per
     * layer, layer height, powder density, cp = powdercpa*T + powdercpb,
     * k = powderthcona*T + powderthconb.  The deck parser has already added the
     * layers to the last z-zone (:160-161). */
    int numlayers, ncvzlayer;
    double layerheight, powderden, powdercpa, powdercpb, powderthcona, powderthconb;
    /* *ACTIVATE_MOVING_MESH row (Mesh.cpp:364-370): 0-based x and y zones that follow the
     * beam (their neighbours grow and shrink, CFDSolverManager.cpp:72-124) */
    int xmoveindex, ymoveindex;
    /* *CALCULATE_SOLIDIFICATION_PARAMETERS (Mesh.cpp:58-61): G and R after every step */
    int solidification;
    /* *TRACK_ENERGY_BASED_FREE_SURFACE row (DomainManager.cpp:133-143): bisection interval
     * of the pressure multiplier, surface tension, energy-balance iterations and
     * tolerance, bisection iterations and tolerance, under-relaxation */
    double fs_lam1, fs_lam2, fs_surftens, fs_maxiterenergy, fs_tolenergy, fs_maxiterbisect,
        fs_tolbisect, fs_urfree;
} amcfd_params;

/* Per-step results, the scalars main() and PrintManager read after
 * iterativeLoopSolve (CFDSolverManager.h:81-90, BoundCondManager.h:331-342). */
typedef struct amcfd_step_report {
    double timet;
    int niter, itertot;
    double resorh, resorm, resoru, resorv, resorw;
    double tpeak, alen, depth, width, ratio;
    double heatinlaser, ahtoploss, accul, heatout, heatvol;
    double beamposx, beamposy, scanvel;
    int istat, iend, jstat, jend, kstat, jstart, powerindicator;
    int momentum_cells;  /* cells of the momentum box solved in the last outer iteration */
    int fallback;        /* 1 when the step's warm-start guess was rejected */
    double resorc;       /* species residual (calculateResiduals(6)); 0 without *SOLVE_SPECIES */
    int nk_active;       /* nodes in z of the active domain (grows per powder layer) */
    int trackindx;       /* BoundCondManager::trackindx_ */
    int steadylength;    /* BoundCondManager::steadylength_ (moving mesh) */
} amcfd_step_report;

/* Line-sweep ordering of the line-by-line solver. */
#define AMCFD_ORDER_EXACT 0    /* the reference's lexicographic Gauss-Seidel order (parity mode) */
#define AMCFD_ORDER_REDBLACK 1 /* red-black line ordering over (j,k): fully parallel sweeps */

/* Arithmetic of the bulk fields and coefficients. */
#define AMCFD_PREC_FP64 0
#define AMCFD_PREC_FP32 1      /* FP32 bulk, FP64 reductions and H->T inversion */
/* FP64 fields, properties, reductions and momentum; the energy line solves (the
 * bulk of the bandwidth) in FP32 on the correction: each outer iteration forms the
 * FP64 defect of the enthalpy equation, solves for the correction with FP32
 * coefficients and adds it to the FP64 enthalpy (mixed-precision defect
 * correction).  Red-black order only. */
#define AMCFD_PREC_FP32_DC 2

typedef struct amcfd_options {
    int device;          /* CUDA device ordinal */
    int order;           /* AMCFD_ORDER_* */
    int precision;       /* AMCFD_PREC_* */
    int use_graphs;      /* capture the fixed-shape part of an outer iteration */
    int check_finite;    /* fail with AMCFD_E_NONFINITE when a reduction is not finite */
    int no_small_box;    /* the momentum chain of a melt-pool box small enough for one CTA's
                            shared memory (red-black order only): 0 lets the solver choose (the
                            cooperative box solve where it is available, which measured as fast
                            or faster for every box size, else the one-CTA chain); 1 never runs
                            the one-CTA chain; -1 runs it whenever the box fits */
    int host_loop;       /* 1: with use_graphs, still launch one graph per outer iteration and
                            test convergence on the host (0: one graph per step, the
                            iterations chained on the device) */
    int wait_polls;      /* polls (about 64 ns each) a warp of a line sweep (the exact-order
                            wavefront, the pipelined red-black passes, the cooperative
                            momentum-box solve) waits for a neighbouring line before the step fails with
                            AMCFD_E_TIMEOUT; 0 = the default 2^24 (about one second).  The
                            reference has no such wait (its sweeps are sequential). */
    int autotune;        /* 1: at creation, time the candidate launch shapes of the energy
                            assembly (planes per CTA) and of the red-black line sweeps (lines
                            per CTA) on this grid and keep the fastest (amcfd_tuning reports
                            them); 0: the fixed defaults.  The assembly's shape sets the order
                            of its FP64 partial sums, so contexts whose results must agree bit
                            for bit pin it (asm_kseg). */
    int asm_kseg;        /* planes per CTA of the energy assembly: 4, 8 or 16; 0 = default/tuned */
    int sweep_warps;     /* lines (warps) per CTA of the red-black sweeps: 2, 4 or 8; 0 = default/tuned */
    int mom_cluster;     /* CTAs of the cluster that solves a momentum box larger than one CTA's
                            shared memory (red-black order): 2, 4, 8 or 16, at most what the
                            device schedules; 1 = no cluster (such boxes take the multi-kernel
                            path); 0 = the default, 1 (the multi-kernel path measured faster
                            on the benchmark decks' boxes) */
    int serial_launch;   /* 1: every kernel of an outer iteration is launched only after the
                            kernel before it has finished; 0: a kernel's launch overlaps the
                            end of the one before it (programmatic dependent launch: it
                            still waits for that kernel's completion before it reads
                            anything, so the results are the same bits); 1 also solves the
                            momentum box's lines of an equation with a launch per colour pass
                            instead of one cooperative launch */
    int box_ctas;        /* CTAs of the cooperative momentum-box line solve (capped at what the
                            largest box needs and what is resident at once); 0 = that cap
                            (fewer make each warp take several lines of a colour, restaging
                            them every pass) */
    int pass_launch;     /* 1: the whole-domain red-black line sweeps (enthalpy, species,
                            the defect correction) take one launch per colour pass; 0: the
                            eight passes of a solve run in one launch, pipelined along k so
                            that later passes find a plane's coefficient rows in L2 (the
                            same bits: each line still reads its neighbours after exactly
                            the passes the per-pass order gives it).  serial_launch = 1
                            implies 1. */
} amcfd_options;

typedef struct amcfd_deck amcfd_deck;
typedef struct amcfd_ctx amcfd_ctx;

/* Deck parsing: replaces Mesh::getDomainInfo / assignParameters / readMeshFile
 * (Mesh.h:74-84) and DomainManager::assignInputValues / getToolpath
 * (DomainManager.h:256-258).  The returned params point into the deck's own
 * storage (toolpath rows) and stay valid until amcfd_deck_free. */
int amcfd_deck_load(const char *path, amcfd_deck **out);
int amcfd_deck_params(const amcfd_deck *deck, amcfd_params *out);
const char *amcfd_deck_error(void);
void amcfd_deck_free(amcfd_deck *deck);
/* "keyword_id", "directory", "geometry_file" (NULL unless *OUTPUT_FINAL_GEOMETRY),
 * "mesh_file": the names PrintManager derives its output files from;
 * "scalar_out", "vector_out": the requested output fields, space-separated. */
const char *amcfd_deck_string(const amcfd_deck *deck, const char *what);
/* sizeof(amcfd_params) / sizeof(amcfd_step_report), for bindings that mirror the structs */
size_t amcfd_sizeof_params(void);
size_t amcfd_sizeof_report(void);

/* Context creation: replaces CFDSolverManager::generateGrid + initializeSolver
 * and BoundCondManager::initializeBoundaries (CFDSolverManager.cpp:34-590,
 * BoundCondManager.cpp:27-63).  opts may be NULL (FP64, exact order, device 0). */
int amcfd_create(const amcfd_params *params, const amcfd_options *opts, amcfd_ctx **out);
void amcfd_destroy(amcfd_ctx *ctx);
const char *amcfd_last_error(const amcfd_ctx *ctx);

/* One time step: main.cpp:136-162 -- timet += delt, BoundCondManager::updateLaser,
 * CFDSolverManager::iterativeLoopSolve, CFDSolverManager::updateSolutions. */
int amcfd_step(amcfd_ctx *ctx, amcfd_step_report *report);

/* Field access by the reference's registry key (CFDSolverManager.cpp:528-541):
 * "temp","uvel","vvel","wvel","pressure","pp","enthalpy","fracl","fraclnot",
 * "hnot","diff","rho","vis","sourceinput"; with *SOLVE_SPECIES also "avgconcentration",
 * "avgconcentrationnot","concentration"; with *POWDER_BED_MODE also "csfrac","solfrac",
 * "mpPhase","mpLiqPhase"; with *CALCULATE_SOLIDIFICATION_PARAMETERS also "grad","rate";
 * with *TRACK_ENERGY_BASED_FREE_SURFACE also "zr","tempr" (as of the last amcfd_free_surface);
 * grid arrays "x","y","z","xu","yv","zw" (the current ones under a moving mesh).  Arrays
 * cover the whole grid (every powder layer, active or not). 
 * host buffers hold ni*nj*nk doubles in [k][j][i] order (i fastest). */
int amcfd_get_field(amcfd_ctx *ctx, const char *name, double *host_out);
/* amcfd_get_field that returns as soon as the copy is queued (no counterpart in the
 * reference, whose writers read host arrays in place).  The field is packed on the
 * solver's stream, so later steps may change it at once, and copied to host_out on a
 * second stream while the caller goes on; with pinned host_out the copy overlaps the
 * next step.  host_out must stay valid and is complete only after amcfd_wait_reads.
 * Any later read of a field waits for the copy before it reuses the staging. */
int amcfd_get_field_async(amcfd_ctx *ctx, const char *name, double *host_out);
/* Blocks until the last amcfd_get_field_async copy has landed in host memory. */
int amcfd_wait_reads(amcfd_ctx *ctx);
int amcfd_set_field(amcfd_ctx *ctx, const char *name, const double *host_in);
int amcfd_get_grid(amcfd_ctx *ctx, const char *name, double *host_out);
int amcfd_dims(const amcfd_ctx *ctx, int *ni, int *nj, int *nk);

/* Kernel-level entry points for parity tests: run one phase of an outer
 * iteration on the current device state (the reference function each phase
 * replaces is listed in amcfd_phase_name). */
/* 1: main.cpp:136-141, timet += delt and BoundCondManager::updateLaser */
#define AMCFD_PHASE_LASER 1
/* 2: applyBCs(5), discretizeEquations(5), calculateSource(5), calculateResiduals(5),
 *    bareplateMaterialProps (into "diff_next"/"rho_next"/"vis_next") and the
 *    block-correction solve of enhanceConvergenceSpeed(5) (CFDSolverManager.cpp:619-626) */
#define AMCFD_PHASE_ENERGY_ASSEMBLE 2
/* 3: the block-correction update and solveEntireDomain(5) (:626-642) */
#define AMCFD_PHASE_ENERGY_SOLVE 3
/* 4: convertEnthalpyToTemp (:643) */
#define AMCFD_PHASE_H2T 4
/* 5: getMeltPoolShape (:657) */
#define AMCFD_PHASE_MELTPOOL 5
/* 6: cleanVelocities and the u, v, w, p' chain (:660-675) */
#define AMCFD_PHASE_MOMENTUM 6
/* 7: calculateFluxes and the convergence test (:689-716); the new properties become current */
#define AMCFD_PHASE_CONVERGE 7
/* 8: CFDSolverManager::updateSolutions */
#define AMCFD_PHASE_UPDATE 8
/* 9: the species equation, applyBCs(6) ... solveEntireDomain(6) (:678-687); a no-op
 *    without *SOLVE_SPECIES */
#define AMCFD_PHASE_SPECIES 9
int amcfd_run_phase(amcfd_ctx *ctx, int phase, amcfd_step_report *report);
const char *amcfd_phase_name(int phase);

/* Device time of the last amcfd_step split by kernel family (ms); n entries. */
int amcfd_last_timing(const amcfd_ctx *ctx, double *ms, int n);
/* Enable (1) or disable (0) the per-phase CUDA-event timing read by amcfd_last_timing;
 * clears the accumulated times. */
int amcfd_profile(amcfd_ctx *ctx, int enable);

/* nsteps calls of amcfd_step bracketed by CUDA events on the context stream;
 * *device_ms receives the device time between the events.  (main.cpp:123-201) */
int amcfd_run_steps(amcfd_ctx *ctx, int nsteps, amcfd_step_report *report, double *device_ms);

/* Number of kernels the context has launched since creation. */
long long amcfd_kernel_launches(const amcfd_ctx *ctx);

/* Launch shapes in use (no counterpart in the reference): planes per CTA of the
 * energy assembly (*asm_kseg, 0 = the default rule) and lines per CTA of the
 * red-black sweeps (*sweep_warps); with amcfd_options.autotune, the measured times
 * of the candidates in ms (times[0..2]: assembly with 4, 8, 16 planes; times[3..5]:
 * a factorising and a plain sweep pass with 2, 4, 8 lines, or, when the red-black
 * passes run as one pipelined launch, that launch with its passes 8, 16, 32 planes
 * apart in its work order; 0 when not timed). */
int amcfd_tuning(const amcfd_ctx *ctx, int *asm_kseg, int *sweep_warps, double *times);
/* The planes between successive passes in the work order of the pipelined red-black
 * line solve (autotuned among 8, 16, 32; default 16), or 0 when the passes take a
 * launch each.  No counterpart in the reference (its sweeps are sequential loops). */
int amcfd_pipe_stride(const amcfd_ctx *ctx, int *stride);

/* Parameter sweep over independent instances: runs nsteps time steps of every
 * context in ctxs[0..n), each on its own stream, spread over nthreads host threads
 * (0 = one per context, at most 64).  A thread takes the next context in array
 * order and runs all its steps, so pass the contexts largest first.  The first
 * step of the first context of each kind (precision, order, graph use) runs on the
 * calling thread before the others start: it loads every kernel that kind
 * launches, so that no thread loads a kernel while another captures a graph.  reports[q]
 * receives the last step's report of ctxs[q] and status[q] its return code (0, or
 * a negative AMCFD_E_* code; that context's amcfd_last_error says why); either may
 * be NULL.  Returns 0 when every context succeeded, else the first failing code in
 * array order.  The reference runs one instance per process (main.cpp:25-233); a
 * sweep is many such runs. */
int amcfd_run_batch(amcfd_ctx *const *ctxs, int n, int nsteps, int nthreads,
                    amcfd_step_report *reports, int *status);

/* Energy-balance free surface (FreeSurfaceManager::execute, FreeSurfaceManager.cpp:74-209):
 * the surface deflection of the molten top nodes that balances gravity, surface
 * tension and a pressure multiplier found by bisection so that the deflected volume
 * matches the evaporated volume; then the deformed node heights "zr" and the
 * temperatures interpolated onto them, "tempr".  The reference runs it before each
 * output (main.cpp:174-176, 210-212); the output writer does the same.  Decks without
 * *TRACK_ENERGY_BASED_FREE_SURFACE: AMCFD_E_ARG. */
typedef struct amcfd_free_surface_report {
    double lambda;     /* the last multiplier tried (xmid) */
    double residual;   /* its volume residual (fmid) */
    double fi_min, fi_max;  /* extremes of the deflection over the surface */
    double volume;     /* the target volume vd */
    int iterations;    /* bisection iterations run */
    int bracketed;     /* 0 where the initial interval did not bracket the root (the reference warns) */
} amcfd_free_surface_report;
int amcfd_free_surface(amcfd_ctx *ctx, amcfd_free_surface_report *out);

/* ---- Output writer (main.cpp:92-226, PrintManager.cpp, vtsBinWriter.cpp) ------
 * Writes what the reference's transient run writes, in its formats:
 * <directory>/<keyword_id>_<n>.vts (VTK StructuredGrid, appended raw Float64
 * point data of the deck's *SCALAR_OUT fields, uvel/vvel/wvel as the cell-centred
 * auvel/avvel/awvel), <keyword_id>.pvd, <keyword_id>_Residuals.txt and, with
 * *OUTPUT_FINAL_GEOMETRY, the final-geometry file; paths relative to `root`
 * (NULL or "" = the working directory).  Create it before the first step: like
 * the reference it writes the initial state as <keyword_id>_0.vts. */
typedef struct amcfd_writer amcfd_writer;
int amcfd_writer_create(amcfd_ctx *ctx, const amcfd_deck *deck, const char *root, amcfd_writer **out);
/* after each amcfd_step: 1 when the output interval has passed and an output
 * was written, 0 when not, a negative AMCFD_E_* code on failure */
int amcfd_writer_step(amcfd_writer *w);
/* the final output and final-geometry file (after the last step) */
int amcfd_writer_finish(amcfd_writer *w);
const char *amcfd_writer_last_error(const amcfd_writer *w);
void amcfd_writer_destroy(amcfd_writer *w);

/* ---- Learned warm start: a 4-layer 3x3x3 convolutional network --------------
 * No counterpart in the reference.  Layers 16->32->32->32->16 channels (9 input
 * features and 2 outputs used), ReLU between layers, BF16 operands on the tensor
 * cores with FP32 accumulation, FP32 master parameters laid out per layer as
 * W[27][cout][cin] then b[cout] (tap = 9(dk+1) + 3(dj+1) + (di+1)).  Inputs and
 * outputs are device arrays over a full ni x nj x nk node grid, channels last;
 * boundary nodes are held at zero (a zero-padded convolution over the interior). */
typedef struct amcfd_net amcfd_net;
size_t amcfd_net_param_count(void);
int amcfd_net_create(int device, unsigned long long seed, amcfd_net **out);
void amcfd_net_destroy(amcfd_net *net);
const char *amcfd_net_last_error(const amcfd_net *net);
int amcfd_net_get_params(amcfd_net *net, float *host, size_t n);
int amcfd_net_set_params(amcfd_net *net, const float *host, size_t n);
int amcfd_net_get_grads(amcfd_net *net, float *host, size_t n);
/* Overwrites the gradients that amcfd_net_adam applies next (data-parallel training
 * averages them over the ranks in between).  No counterpart in the reference. */
int amcfd_net_set_grads(amcfd_net *net, const float *host, size_t n);
/* feat_dev: [ncell][11] FP32; y_dev (nullable): [ncell][2] FP32 */
int amcfd_net_forward(amcfd_net *net, const float *feat_dev, int ni, int nj, int nk, float *y_dev);
/* MSE of the last forward pass against target_dev [ncell][2] over interior cells;
 * all parameter gradients into the net's gradient buffer */
int amcfd_net_backward(amcfd_net *net, const float *target_dev, double *loss);
int amcfd_net_adam(amcfd_net *net, float lr);
/* device ms (CUDA events) of the last forward and backward passes */
int amcfd_net_last_ms(const amcfd_net *net, float *fwd_ms, float *bwd_ms);

/* Attach a warm-start network to a solver context (same device).  Modes:
 * AMCFD_WS_OFF; AMCFD_WS_PREDICT: each step starts from the network's predicted
 * enthalpy and pressure increments, kept only if they lower the step's initial
 * energy residual (the report's `fallback` is 1 when they were rejected);
 * AMCFD_WS_PREDICT_H: the same with the enthalpy increment only;
 * AMCFD_WS_RECORD: no prediction.  In all active modes every step leaves its
 * features ([ncell][11]) and realised scaled increments ([ncell][2]) in device
 * buffers (amcfd_ws_buffers) for training with amcfd_net_forward/backward.
 * Decks with a volumetric heat-source table are refused. */
#define AMCFD_WS_OFF 0
#define AMCFD_WS_PREDICT 1
#define AMCFD_WS_RECORD 2
#define AMCFD_WS_PREDICT_H 3
int amcfd_ws_attach(amcfd_ctx *ctx, amcfd_net *net, int mode);
int amcfd_ws_buffers(amcfd_ctx *ctx, float **feat_dev, float **target_dev);
int amcfd_ws_stats(const amcfd_ctx *ctx, long long *accepted, long long *rejected);

/* Energy residual without any device allocation.  No counterpart in the reference:
 * it exists for callers that cannot let a library allocate device memory (an
 * application that owns all device memory through its own pool, or one under a
 * fixed memory budget).  The caller passes device arrays an..su and the enthalpy h,
 * laid out [nk][nj][pitch] (i fastest, pitch >= ni), and a device double for the
 * result; resorh = sum|(sum a_nb h_nb + su)/ap - h| / (sum|h| + 1e-6) over the
 * interior, as calculateResiduals(5) computes it.  Scratch is a file-scope device
 * array held by every GPU that loads the library (64 KiB) that supports at most
 * 4096 interior k-planes (nk - 2); larger grids get AMCFD_E_CAPACITY.  The first
 * call on a device looks up that array's address (make it before any stream
 * capture); a call under a new context of the device (after cudaDeviceReset) looks
 * it up again.  Calls share the array: calls that overlap on the GPU race.  Work is
 * queued on `stream` (a cudaStream_t, NULL for the default stream).  A CUDA error
 * already pending from the caller's own earlier work makes the call return
 * AMCFD_E_CUDA without launching and without clearing that error. */
int amcfd_energy_residual_noalloc(const double *an, const double *as, const double *ae,
                                  const double *aw, const double *at, const double *ab,
                                  const double *ap, const double *su, const double *h,
                                  int ni, int nj, int nk, int pitch,
                                  double *resorh_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AMCFD_H */
