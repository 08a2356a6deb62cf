// Host driver and C ABI of the solver (include/amcfd.h).
//
// A context owns one instance on one GPU: the device arrays, a CUDA stream and
// the host copy of the grid and laser state.  amcfd_step() reproduces one pass
// of the reference time loop (src/main.cpp:125-162): variable time step,
// timet += delt, BoundCondManager::updateLaser (beam position on the host,
// heat flux on the device), the SIMPLE outer loop of
// CFDSolverManager::iterativeLoopSolve (CFDSolverManager.cpp:595-722) as a
// chain of kernels per outer iteration, and updateSolutions.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <string>
#include <vector>

#include "amcfd.h"
#include "async.cuh"
#include "kernels.cuh"

namespace amcfd {
template <typename T> int exact_sweep_blocks_per_sm(int warps, size_t smem);
template <typename T> void set_sweep_smem_limit(size_t smem);
template <typename T> int set_rounds_smem_limit(const Params &p);
template <typename T> int setup_pipe_sweep(const Params &p, int warps, int sm_count, size_t &smem);
dim3 energy_assemble_grid(const Params &p, int kseg);
template <typename T> int h2t_blocks_per_sm();
template <typename T> void launch_pack_field(const T *src, double *dst, int ni, int nip,
                                             long long rows, int sm_count, cudaStream_t s);
template <typename T> void launch_centre_velocity(Inst<T> &I, int comp, double *dst);
template <typename T> void ws_features(Inst<T> &I, float *feat, const float *prev, double bx, double by,
                                       double power);
template <typename T> void ws_copy(Inst<T> &I, T *const *save, int dir);
template <typename T> void ws_apply(Inst<T> &I, const float *y, double alpha, int with_p);
template <typename T> void ws_target(Inst<T> &I, T *const *save, float *target);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
int encode_tiled_3d(CUtensorMap *map, CUtensorMapDataType dtype, const void *base, const uint64_t dims[3],
                    const uint64_t strides[2], const uint32_t box[3], int swizzle_bytes)
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &qr) !=
                cudaSuccess ||
            qr != cudaDriverEntryPointSuccess || !ptr)
            return -1;
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }
    const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
    const cuuint64_t st[2] = {strides[0], strides[1]};
    const cuuint32_t bx[3] = {box[0], box[1], box[2]};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, dtype, 3, const_cast<void *>(base), d, st, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swizzle_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                    : swizzle_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                    : swizzle_bytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                          : CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

int encode_field_map(CUtensorMap *map, const void *base, int elem, int nip, int nj, int nk, int bx,
                     int by)
{
    const uint64_t dims[3] = {(uint64_t)nip, (uint64_t)nj, (uint64_t)nk};
    const uint64_t strides[2] = {(uint64_t)nip * elem, (uint64_t)nip * nj * elem};
    const uint32_t box[3] = {(uint32_t)bx, (uint32_t)by, 1};
    return encode_tiled_3d(map, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           base, dims, strides, box, 0);
}
}  // namespace amcfd

using namespace amcfd;

struct amcfd_ctx {
    std::string err;
    amcfd_params prm;
    std::vector<double> tool, heattable, vardt;
    std::vector<int> tool_on, tool_id;
    int precision = AMCFD_PREC_FP64;  // FP64 also under defect correction (FP64 instance)
    bool dc = false;                   // AMCFD_PREC_FP32_DC: energy line solves on the FP32 correction
    int order = AMCFD_ORDER_EXACT;
    int device = 0;
    int ni = 0, nj = 0, nk = 0, nip = 0;  // nk: planes of every 3-D array (all powder layers)
    int nk_active = 0;                     // DomainManager::nk_ (grows per powder layer)
    double hlcal = 0, hlatnt = 0;
    std::vector<double> x, y, z, xu, yv, zw, dxpwinv, dypsinv, dzpbinv, fracx, fracy, fracz;
    // laser / time state (BoundCondManager.h:339-349, DomainManager::timet_)
    double timet = 0, delt = 0, outtime = 0, scanvel = 0;
    double beamposx = 0, beamposy = 0, beamposz = 0, oldbeamposx = 0, oldbeamposy = 0,
           oldbeamposz = 0;
    int powerindicator = 1, init = 1, trackindx = 1, istart = 0, jstart = 0, vardt_state = 0;
    int itertot = 0, niter = 0;
    int steadylength = 0;          // BoundCondManager::steadylength_ (moving mesh)
    double *dmetric[12] = {};      // device copies of x y z xu yv zw dxpwinv dypsinv dzpbinv fracx fracy fracz
    double *mesh_old = nullptr;    // moving mesh: centres before the move, x (ni) then y (nj)
    double *mesh_pinned = nullptr; // moving mesh: pinned staging of the new metrics and old centres
    FsOut *fs_out = nullptr;       // free surface: the bisection's results (device)
    Inst<double> I64;
    Inst<float> I32;
    std::vector<void *> allocs;
    cudaStream_t stream = nullptr;
    Status *st_dev = nullptr;
    Status *st_host = nullptr;  // pinned
    cudaEvent_t ev[16] = {};
    double last_ms[16] = {0};
    bool events = false;
    long long launches = 0;  // kernels launched since creation
    // CUDA graphs of one outer iteration, by [timing events recorded][property parity]:
    // the iteration swaps the current/next property buffers, so two graphs alternate.
    bool use_graphs = false;
    cudaGraphExec_t gexec[2][2][2] = {};  // [events][parity][small-box momentum]
    // the whole outer loop of a step as one graph, by property parity at its start
    cudaGraphExec_t gloop[2] = {};
    bool host_loop = false;        // drive the outer iterations from the host even with graphs
    long long wait_polls = 0;      // budget of the exact-order sweep's line waits (0: default)
    int autotune = 0, asm_kseg = 0, sweep_warps = 0;  // launch shapes: tuned, or pinned (0: default)
    double tune_ms[6] = {0};       // the autotuner's measured candidates
    int mom_cluster = 1;           // CTAs of the cluster momentum path (1: none)
    int mom_cluster_req = 0;       // as requested by the options (0: default)
    int serial_launch = 0;         // 1: no programmatic dependent launch, box solve per pass
    int pass_launch = 0;           // 1: the whole-domain red-black sweeps take a launch per pass
    int box_ctas = 0;              // CTAs of the cooperative box solve (0: what the box needs)
    int last_box = -1;             // momentum box cells seen by the last outer iteration
    int small_mode = 0;            // one-CTA momentum chain: 0 auto, 1 never, -1 whenever the box fits
    const void *diff_a = nullptr;  // the current-property buffer of parity 0
    double *pack = nullptr;        // FP64 read-out staging (ni*nj*nk), made on first use
    // asynchronous read-out: the staging is copied to the host on its own stream
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_packed = nullptr, ev_copied = nullptr;
    bool copy_pending = false;     // a copy out of the staging may still be running
    int sm_count = 0;
    // learned warm start (amcfd_ws_attach)
    amcfd_net *net = nullptr;
    int ws_mode = 0;
    float *ws_feat = nullptr, *ws_y = nullptr, *ws_target = nullptr;
    void *ws_save[4] = {};         // h, p, T, f_l at the start of the step
    long long ws_accepted = 0, ws_rejected = 0;
    int ws_fallback = 0;           // the last step's prediction was rejected
};

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return AMCFD_E_CUDA;                                                          \
        }                                                                                 \
    } while (0)

static int fail(amcfd_ctx *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

// ---- grid: CFDSolverManager::generateGrid (CFDSolverManager.cpp:126-240) -------------
static void zone_faces(int nz, const double *len, const double *ncv, const double *powr,
                       std::vector<double> &face)
{
    face[0] = 0.0;
    face[1] = 0.0;
    int ist = 2;
    double statloc = 0.0;
    for (int zi = 0; zi < nz; zi++) {
        for (int q = 0; q < ncv[zi]; q++) {
            double term;
            if (powr[zi] >= 0.0)
                term = std::pow((double)(q + 1) / ncv[zi], powr[zi]);
            else
                term = 1.0 - std::pow(1.0 - (double)(q + 1) / ncv[zi], -powr[zi]);
            face[q + ist] = statloc + len[zi] * term;
        }
        ist += (int)ncv[zi];
        statloc += len[zi];
    }
}

// nkz: the z nodes whose centres are (re)computed -- every node at start-up, the
// active ones when a moving mesh regenerates a powder-bed grid (the reference
// then loops to nk_, leaving the planes above as they were).
static void build_grid(amcfd_ctx *c, int nkz)
{
    const amcfd_params &p = c->prm;
    auto axis = [](int n, int na, int nz, const double *len, const double *ncv, const double *powr,
                   std::vector<double> &face, std::vector<double> &cen, std::vector<double> &inv,
                   std::vector<double> &frac) {
        if (face.size() != (size_t)n + 1) {
            face.assign(n + 1, 0.0);
            cen.assign(n + 1, 0.0);
            inv.assign(n + 1, 0.0);
            frac.assign(n + 1, 0.0);
        }
        zone_faces(nz, len, ncv, powr, face);
        for (int q = 0; q < na - 1; q++) cen[q] = (face[q + 1] + face[q]) * 0.5;
        cen[na - 1] = face[na - 1];
        for (int q = 1; q < na; q++) inv[q] = 1.0 / (cen[q] - cen[q - 1]);
        for (int q = 0; q < na - 1; q++) frac[q] = (cen[q + 1] - face[q + 1]) / (cen[q + 1] - cen[q]);
    };
    axis(c->ni, c->ni, p.nzx, p.xzone, p.ncvx, p.powrx, c->xu, c->x, c->dxpwinv, c->fracx);
    axis(c->nj, c->nj, p.nzy, p.yzone, p.ncvy, p.powry, c->yv, c->y, c->dypsinv, c->fracy);
    axis(c->nk, nkz, p.nzz, p.zzone, p.ncvz, p.powrz, c->zw, c->z, c->dzpbinv, c->fracz);
}

// ---- laser position: BoundCondManager::getLaserCoords / updateLaser (:68-275) ----------
static void laser_coords(amcfd_ctx *c)
{
    const amcfd_params &p = c->prm;
    if (p.steady) {
        c->beamposx = p.xstart;
    } else if (!p.udtoolpath) {
        c->oldbeamposx = c->beamposx;
        if (c->timet <= p.lasertime) {
            c->beamposx = p.xstart + c->timet * c->scanvel;
            if (c->init) {
                c->oldbeamposx = c->beamposx;
                c->init = 0;
            }
        } else {
            c->beamposx = p.xstart + p.lasertime * c->scanvel;
            c->powerindicator = 0;
        }
        c->beamposy = p.ystart;
    } else {
        double tx = 0.0, ty = 0.0, tz = 0.0, deltaty = 0.0;
        const double small = 1.0e-8;
        c->oldbeamposx = c->beamposx;
        c->oldbeamposy = c->beamposy;
        c->oldbeamposz = c->beamposz;
        int oldpower = c->powerindicator;
        const int n = (int)c->tool_on.size();
        for (int ii = 1; ii < n; ii++) {
            const double *b = &c->tool[4 * ii];
            if (c->timet <= b[0] + small) {
                const double *a = &c->tool[4 * (ii - 1)];
                double ratio = (c->timet - a[0]) / (b[0] - a[0]);
                double dx = b[1] - a[1];
                deltaty = b[2] - a[2];
                double dz = b[3] - a[3];
                tx = ratio * dx + a[1];
                ty = ratio * deltaty + a[2];
                tz = ratio * dz + a[3];
                c->powerindicator = c->tool_on[ii];
                if (c->init) {
                    c->oldbeamposx = a[1];
                    c->oldbeamposy = a[2];
                    c->oldbeamposz = a[3];
                    oldpower = c->tool_on[ii - 1];
                    c->init = 0;
                }
                break;
            }
        }
        c->beamposx = tx;
        c->beamposy = ty;
        c->beamposz = tz;
        double dist = std::sqrt((c->beamposx - c->oldbeamposx) * (c->beamposx - c->oldbeamposx) +
                                (c->beamposy - c->oldbeamposy) * (c->beamposy - c->oldbeamposy) +
                                (c->beamposz - c->oldbeamposz) * (c->beamposz - c->oldbeamposz));
        c->scanvel = dist / c->delt;
        if (oldpower - c->powerindicator > 0 && deltaty > small) c->trackindx++;
        // powder bed: the beam switching on activates the next layer (:266-272)
        if (c->powerindicator - oldpower > 0 && p.powderbed) {
            c->trackindx++;
            c->nk_active += p.ncvzlayer;
        }
    }
    // nearest node to the beam (:92-126)
    int iout = 0, jout = 0;
    for (int i = 1; i < c->ni - 1; i++) {
        if (c->beamposx <= c->x[i]) break;
        iout = i;
    }
    if (std::fabs(c->beamposx - c->x[iout + 1]) < std::fabs(c->beamposx - c->x[iout])) iout++;
    c->istart = iout;
    for (int j = 1; j < c->nj - 1; j++) {
        if (c->beamposy <= c->y[j]) break;
        jout = j;
    }
    if (std::fabs(c->beamposy - c->y[jout + 1]) < std::fabs(c->beamposy - c->y[jout])) jout++;
    c->jstart = jout;
}

// ---- device setup ----------------------------------------------------------------------
template <typename T>
static int alloc3(amcfd_ctx *ctx, T **ptr, size_t n)
{
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return AMCFD_E_NOMEM;
    }
    ctx->allocs.push_back(p);
    cudaMemsetAsync(p, 0, n * sizeof(T), ctx->stream);
    *ptr = (T *)p;
    return 0;
}

template <typename T>
static int upload(amcfd_ctx *ctx, T *dst, const std::vector<double> &src)
{
    std::vector<T> tmp(src.begin(), src.end());
    CK(cudaMemcpy(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

// (t, m, s) order of the visits (ks, k, s, j) of solveEntireDomain over M planes
// and J rows (k_linesolve.cu explains the wave index t).
static std::vector<int2> energy_tickets(int M, int J)
{
    std::vector<int2> tk;
    tk.reserve((size_t)4 * M * J);
    const int Tw = 3 * (2 * M - 1) + (J - 1) + 2 + 1;
    for (int t = 0; t < Tw; ++t)
        for (int m = std::max(0, (t - 2 - (J - 1)) / 3 - 1); m <= std::min(2 * M - 1, t / 3); ++m)
            for (int s = 0; s < 2; ++s) {
                int jj = t - 3 * m - 2 * s;
                if (jj >= 0 && jj < J) tk.push_back(make_int2(m, (s << 16) | jj));
            }
    return tk;
}

static void drop_graphs(amcfd_ctx *ctx);

// Resize the active domain to nk planes (powder-bed layer activation,
// BoundCondManager.cpp:266-272; PrintManager.cpp:67-73 at start-up): the launch
// shapes that depend on nk, the exact-order ticket list and the captured graphs
// (their kernel arguments hold the old extents) follow.
template <typename T>
static int set_active_nk(amcfd_ctx *ctx, Inst<T> &I, int nk)
{
    Params &p = I.p;
    if (nk == p.nk) return 0;
    if (nk < 3 || nk > p.nk_alloc)
        return fail(ctx, AMCFD_E_CAPACITY, "powder layer activation beyond the generated grid (nk " +
                                               std::to_string(nk) + " of " + std::to_string(p.nk_alloc) + ")");
    CK(cudaStreamSynchronize(ctx->stream));
    p.nk = nk; p.nkm1 = nk - 1; p.nkm2 = nk - 2;
    I.asm_grid = energy_assemble_grid(p, I.asm_kseg);
    I.nb_asm = I.asm_grid.x * I.asm_grid.y * I.asm_grid.z;
    I.g.npart = I.asm_grid.y * I.asm_grid.z;
    I.max_lines = (p.nj - 2) * (p.nk - 2);
    const std::vector<int2> tk = energy_tickets(p.nk - 2, p.nj - 2);
    CK(cudaMemcpy(I.g.tickets_energy, tk.data(), tk.size() * sizeof(int2), cudaMemcpyHostToDevice));
    I.g.ntickets_energy = (int)tk.size();
    drop_graphs(ctx);
    return 0;
}

template <typename T>
static int setup_instance(amcfd_ctx *ctx, Inst<T> &I)
{
    const amcfd_params &q = ctx->prm;
    Params &p = I.p;
    memset(&p, 0, sizeof(p));
    p.ni = ctx->ni; p.nj = ctx->nj; p.nk = ctx->nk; p.nip = ctx->nip;
    p.nim1 = p.ni - 1; p.njm1 = p.nj - 1; p.nkm1 = p.nk - 1;
    p.nim2 = p.ni - 2; p.njm2 = p.nj - 2; p.nkm2 = p.nk - 2;
    p.dens = q.dens; p.denl = q.denl; p.viscos = q.viscos; p.tsolid = q.tsolid;
    p.tliquid = q.tliquid; p.hsmelt = q.hsmelt; p.hlcal = ctx->hlcal; p.hlatnt = ctx->hlatnt;
    p.acpa = q.acpa; p.acpb = q.acpb; p.acpl = q.acpl;
    p.thconsa = q.thconsa; p.thconsb = q.thconsb; p.thconsc = q.thconsc;
    p.thconla = q.thconla; p.thconlb = q.thconlb;
    p.urfu = q.urfu; p.urfv = q.urfv; p.urfw = q.urfw; p.urfp = q.urfp; p.urfh = q.urfh;
    p.htci = q.htci; p.htcj = q.htcj; p.htckn = q.htckn; p.emiss = q.emiss; p.sigm = q.sigm;
    p.tempamb = q.tempamb; p.beta = q.beta; p.grav = q.grav; p.dgdtp = q.dgdtp;
    p.darcyKo = q.darcyKo; p.a_oxygen = q.a_oxygen;
    p.alaspow = q.alaspow; p.alaseta = q.alaseta; p.alasrb = q.alasrb; p.alasfact = q.alasfact;
    p.pressamb = q.pressamb; p.gasconst = q.gasconst; p.evaplatent = q.evaplatent;
    p.evaptemp = q.evaptemp; p.evapfact = q.evapfact; p.molarmass = q.molarmass;
    p.isevap = q.isevap; p.scheme = q.scheme; p.steady = q.steady; p.navierstokes = q.navierstokes;
    p.nheattable = q.nheattable;
    p.volsrc = (q.nheattable > 0 || q.heatthick > 0.0) ? 1 : 0;
    p.avolpow = q.avolpow; p.apowseta = q.apowseta; p.heatthick = q.heatthick;
    p.heatrb = q.heatrb; p.avolfact = q.avolfact;
    p.species = q.species ? 1 : 0;
    p.initconc = q.initconc; p.massdiff = q.massdiff; p.kp = q.kp; p.urfc = q.urfc;
    p.powder = q.powderbed ? 1 : 0;
    p.nk_alloc = ctx->nk;
    p.powderden = q.powderden; p.powdercpa = q.powdercpa; p.powdercpb = q.powdercpb;
    p.powderthcona = q.powderthcona; p.powderthconb = q.powderthconb;

    const size_t n3 = (size_t)p.nk * p.nj * p.nip;
    Fields<T> &g = I.g;
    memset(&g, 0, sizeof(g));
    int rc;
    double *m1[12];
    const std::vector<double> *src1[12] = {&ctx->x, &ctx->y, &ctx->z, &ctx->xu, &ctx->yv, &ctx->zw,
                                           &ctx->dxpwinv, &ctx->dypsinv, &ctx->dzpbinv,
                                           &ctx->fracx, &ctx->fracy, &ctx->fracz};
    for (int a = 0; a < 12; a++) {
        if ((rc = alloc3<double>(ctx, &m1[a], src1[a]->size()))) return rc;
        if ((rc = upload<double>(ctx, m1[a], *src1[a]))) return rc;
    }
    g.x = m1[0]; g.y = m1[1]; g.z = m1[2]; g.xu = m1[3]; g.yv = m1[4]; g.zw = m1[5];
    g.dxpwinv = m1[6]; g.dypsinv = m1[7]; g.dzpbinv = m1[8]; g.fracx = m1[9]; g.fracy = m1[10];
    g.fracz = m1[11];
    for (int a = 0; a < 12; a++) ctx->dmetric[a] = m1[a];
    if (q.movingmesh) {
        if ((rc = alloc3<double>(ctx, &ctx->mesh_old, (size_t)p.ni + p.nj))) return rc;
        size_t nst = (size_t)p.ni + p.nj;
        for (int a = 0; a < 12; a++) nst += src1[a]->size();
        CK(cudaMallocHost(&ctx->mesh_pinned, nst * sizeof(double)));
    }
    T **f3[] = {&g.uvel, &g.vvel, &g.wvel, &g.unot, &g.vnot, &g.wnot, &g.pressure, &g.pp,
                &g.h, &g.hnot, &g.temp, &g.fracl, &g.fraclnot, &g.sourceinput,
                &g.diff_cur, &g.rho_cur, &g.vis_cur, &g.diff_nxt, &g.rho_nxt, &g.vis_nxt,
                &g.an, &g.as, &g.ae, &g.aw, &g.at, &g.ab, &g.ap, &g.su, &g.pr, &g.cf, &g.iden,
                &g.dux, &g.dvy, &g.dwz};
    for (auto f : f3)
        if ((rc = alloc3<T>(ctx, f, n3))) return rc;
    if (p.species)
        for (T **f : {&g.conc, &g.concnot, &g.concn})
            if ((rc = alloc3<T>(ctx, f, n3))) return rc;
    if (p.powder)
        for (T **f : {&g.csfrac, &g.solfrac, &g.mpphase, &g.mpliq})
            if ((rc = alloc3<T>(ctx, f, n3))) return rc;
    if (q.solidification)  // CFDSolverManager.cpp:469-472: zero until first written
        for (T **f : {&g.grad, &g.rate})
            if ((rc = alloc3<T>(ctx, f, n3))) return rc;
    if (q.freesurface) {
        if ((rc = alloc3<double>(ctx, &g.fs_fi, (size_t)p.nj * p.nip)) ||
            (rc = alloc3<double>(ctx, &g.fs_zz, (size_t)p.nj * p.nip)) || (rc = alloc3<T>(ctx, &g.fs_zr, n3)) ||
            (rc = alloc3<T>(ctx, &g.fs_tempr, n3)))
            return rc;
        double *o = nullptr;
        if ((rc = alloc3<double>(ctx, &o, (sizeof(FsOut) + 7) / 8))) return rc;
        ctx->fs_out = reinterpret_cast<FsOut *>(o);
    }
    if ((rc = alloc3<double>(ctx, &g.heatin, (size_t)p.nj * p.nip))) return rc;
    if (q.nheattable > 0) {
        if ((rc = alloc3<double>(ctx, &g.heattable, ctx->heattable.size()))) return rc;
        if ((rc = upload<double>(ctx, g.heattable, ctx->heattable))) return rc;
    }
    // reduction regions
    I.sm_count = 148;
    cudaDeviceGetAttribute(&I.sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    I.stream = ctx->stream;
    I.order = ctx->order;
    I.pdl = !ctx->serial_launch;
    I.nb_las = std::max(1, std::min(I.sm_count * 2, (p.ni * p.nj + 255) / 256));
    I.nb_bc = std::max(1, std::min(I.sm_count * 2, (p.ni * p.nj + 2 * p.nk * (p.ni + p.nj) + 255) / 256));
    I.asm_kseg = ctx->asm_kseg;
    I.sweep_warps = ctx->sweep_warps > 0 ? ctx->sweep_warps : 4;
    I.asm_grid = energy_assemble_grid(p, I.asm_kseg);
    I.nb_asm = I.asm_grid.x * I.asm_grid.y * I.asm_grid.z;
    // the assembly's per-CTA buffers hold the largest grid of any active height and
    // of any shape the autotuner may pick
    int nb_asm_max = I.nb_asm, npart_max = I.asm_grid.y * I.asm_grid.z;
    for (int nka = ctx->nk_active; nka <= p.nk; nka += std::max(1, q.ncvzlayer)) {
        if (!p.powder) nka = p.nk;
        const int cand[4] = {I.asm_kseg, 4, 8, 16};
        for (int c = 0; c < 4; ++c) {
            const int seg = cand[c];
            if (c > 0 && !ctx->autotune) continue;
            Params pa = p;
            pa.nk = nka;
            const dim3 ga = energy_assemble_grid(pa, seg);
            nb_asm_max = std::max(nb_asm_max, (int)(ga.x * ga.y * ga.z));
            npart_max = std::max(npart_max, (int)(ga.y * ga.z));
        }
        if (!p.powder) break;
    }
    I.nb_h2t = std::max(1, std::min(I.sm_count * h2t_blocks_per_sm<T>(), (int)((n3 + 255) / 256)));
    I.nb_mom = I.sm_count * 2;
    I.grid_1d = std::max(1, std::min(I.sm_count * 8, (int)((n3 + 255) / 256)));
    double *red;
    size_t nred = (size_t)(I.nb_las + I.nb_bc + nb_asm_max + I.nb_h2t + 5 * I.nb_mom) * R_NSLOTS;
    if ((rc = alloc3<double>(ctx, &red, nred))) return rc;
    I.red_las = red;
    I.red_bc = I.red_las + (size_t)I.nb_las * R_NSLOTS;
    I.red_asm = I.red_bc + (size_t)I.nb_bc * R_NSLOTS;
    I.red_h2t = I.red_asm + (size_t)nb_asm_max * R_NSLOTS;
    I.red_mom = I.red_h2t + (size_t)I.nb_h2t * R_NSLOTS;
    g.red = red;
    if (make_assemble_maps<T>(I, g.diff_cur, g.diff_nxt, g.rho_cur, g.rho_nxt))
        return fail(ctx, AMCFD_E_CUDA, "tensor-map encoding for the energy assembly failed");
    g.npart = I.asm_grid.y * I.asm_grid.z;
    if ((rc = alloc3<double>(ctx, &g.bc, (size_t)npart_max * 4 * p.nip))) return rc;
    if ((rc = alloc3<double>(ctx, &g.delphi, (size_t)p.nip))) return rc;
    if ((rc = alloc3<double>(ctx, &g.bcsum, (size_t)4 * p.nip))) return rc;
    if ((rc = alloc3<int>(ctx, &g.mp_kb, (size_t)p.nip))) return rc;
    if ((rc = alloc3<int>(ctx, &g.mp_jdn, (size_t)p.nip))) return rc;
    if ((rc = alloc3<int>(ctx, &g.mp_jup, (size_t)p.nip))) return rc;
    {
        std::vector<int> jup(p.nip, p.njm1);  // "no cell below Ts" sentinel
        CK(cudaMemcpy(g.mp_jup, jup.data(), jup.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // exact-order scheduling
    I.max_lines = (p.nj - 2) * (p.nk - 2);
    if ((rc = alloc3<int>(ctx, &g.flags, (size_t)p.nk * p.nj))) return rc;
    if ((rc = alloc3<int>(ctx, &I.flags_mom, (size_t)p.nk * p.nj))) return rc;
    {
        const int M = p.nk - 2, J = p.nj - 2;
        const std::vector<int2> tk = energy_tickets(M, J);
        if (tk.size() != (size_t)4 * M * J) return fail(ctx, AMCFD_E_ARG, "ticket enumeration mismatch");
        int2 *d;
        if ((rc = alloc3<int2>(ctx, &d, tk.size()))) return rc;
        CK(cudaMemcpy(d, tk.data(), tk.size() * sizeof(int2), cudaMemcpyHostToDevice));
        g.tickets_energy = d;
        g.ntickets_energy = (int)tk.size();
        if ((rc = alloc3<int2>(ctx, &g.tickets_mom, tk.size()))) return rc;
        if ((rc = alloc3<int>(ctx, &g.ntickets_mom, 1))) return rc;
        if ((rc = alloc3<T>(ctx, &I.mom_scratch, n3))) return rc;
        I.mom_cluster = ctx->mom_cluster_req;
        setup_mom_small<T>(I);
        ctx->mom_cluster = I.mom_cluster;
    }
    g.st = ctx->st_dev;
    p.wait_polls = ctx->wait_polls > 0 ? ctx->wait_polls : kSpinLimit;
    if (ctx->dc) {
        // FP32 coefficients, defect, factorisation and correction of the energy solve
        DcBuf &d = I.dc;
        for (float **f : {&d.an, &d.as, &d.ae, &d.aw, &d.at, &d.ab, &d.ap, &d.su, &d.pr, &d.cf, &d.iden,
                          &d.delta})
            if ((rc = alloc3<float>(ctx, f, n3))) return rc;
        I.sweep_warps_max = std::min(I.sweep_warps_max, set_rounds_smem_limit<float>(p));
        if (I.sweep_warps_max < 2) return fail(ctx, AMCFD_E_CAPACITY, "x-lines too long for the red-black sweep");
        I.dc_on = true;
    }
    I.check_finite = 0;
    I.exact_warps = 4;
    // per warp: 8 staged coefficient rows + one mbarrier (k_linesolve.cu)
    I.line_smem = (size_t)I.exact_warps * 8 * p.nip * sizeof(T) + (size_t)I.exact_warps * 8;
    set_sweep_smem_limit<T>(I.line_smem);
    setup_box_solve<T>(I, !ctx->serial_launch);
    if (ctx->box_ctas > 0 && I.box_grid > 0) I.box_grid = std::min(ctx->box_ctas, I.box_grid);
    if (sizeof(T) == 4 && I.box_grid > 0)  // the FP32 box solve's tagged exchange of line values
        if ((rc = alloc3<unsigned long long>(ctx, &I.xchg, n3))) return rc;
    I.sweep_warps_max = set_rounds_smem_limit<T>(p);
    if (I.sweep_warps_max < 2) return fail(ctx, AMCFD_E_CAPACITY, "x-lines too long for the red-black sweep");
    if (ctx->sweep_warps > I.sweep_warps_max)
        return fail(ctx, AMCFD_E_CAPACITY, "sweep_warps beyond what the x-lines leave room for");
    I.sweep_warps = std::min(I.sweep_warps, I.sweep_warps_max);
    if (I.order == AMCFD_ORDER_REDBLACK && !ctx->serial_launch && !ctx->pass_launch) {
        // the eight passes of a whole-domain solve in one pipelined launch (k_linesolve.cu)
        if ((rc = alloc3<int>(ctx, &I.flags_pipe, (size_t)p.nk * p.nj))) return rc;
        I.pipe_grid = setup_pipe_sweep<T>(p, I.pipe_warps, I.sm_count, I.pipe_smem);
        if (I.dc_on) I.pipe_grid_dc = setup_pipe_sweep<float>(p, I.pipe_warps, I.sm_count, I.pipe_smem_dc);
    }
    int bps = exact_sweep_blocks_per_sm<T>(I.exact_warps, I.line_smem);
    // A wave of the exact-order sweep holds about 2(nj-2)/3 lines; about three
    // waves of lines in flight keep the dependency chain fed without flooding L2
    // with flag polls from warps that are waves ahead.
    I.exact_grid = std::max(1, std::min(I.sm_count * bps, (2 * (p.nj - 2) + I.exact_warps - 1) /
                                                              I.exact_warps));

    // initializeSolver (CFDSolverManager.cpp:402-525)
    std::vector<double> hv(n3, 0.0);
    auto enth = [&](double t) { return 0.5 * q.acpa * t * t + q.acpb * t; };
    const double hpre = enth(q.temppreheat);
    const double diff0 = (q.thconsa * q.temppreheat * q.temppreheat + q.thconsb * q.temppreheat +
                          q.thconsc) / (q.acpa * q.temppreheat + q.acpb);
    auto fill = [&](T *dst, double v) {
        std::vector<double> a(n3, v);
        return upload<T>(ctx, dst, a);
    };
    // both buffers of each property pair: planes outside the active domain (unbuilt
    // powder layers) keep these values until they become active, as in the
    // reference's single arrays
    if ((rc = fill(g.vis_cur, q.viscos)) || (rc = fill(g.rho_cur, q.dens)) ||
        (rc = fill(g.diff_cur, diff0)) || (rc = fill(g.vis_nxt, q.viscos)) ||
        (rc = fill(g.rho_nxt, q.dens)) || (rc = fill(g.diff_nxt, diff0)) || (rc = fill(g.hnot, hpre)) ||
        (rc = fill(g.temp, q.temppreheat)))
        return rc;
    // species (CFDSolverManager.cpp:474-479): every node at the initial concentration
    if (p.species && ((rc = fill(g.conc, q.initconc)) || (rc = fill(g.concnot, q.initconc)) ||
                      (rc = fill(g.concn, q.initconc))))
        return rc;
    if (q.freesurface) {
        // FreeSurfaceManager::initializeFreeSurface (:34-69): zr = z, tempr = T, fi = 0
        std::vector<double> zr(n3);
        for (int k = 0; k < p.nk; k++)
            std::fill(zr.begin() + (size_t)k * p.nj * p.nip, zr.begin() + (size_t)(k + 1) * p.nj * p.nip, ctx->z[k]);
        if ((rc = upload<T>(ctx, g.fs_zr, zr)) || (rc = fill(g.fs_tempr, q.temppreheat))) return rc;
    }
    if (p.powder) {
        // CFDSolverManager.cpp:482-492: the base plate is consolidated, the build
        // layers are powder (csfrac 0); solfrac, mpPhase, mpLiqPhase start at 0
        std::vector<double> cs(n3, 0.0);
        const double top = ctx->z[p.nk - 1] - (double)q.numlayers * q.layerheight;
        for (int k = 0; k < p.nk; k++)
            if (ctx->z[k] < top)
                for (size_t c = (size_t)k * p.nj * p.nip; c < (size_t)(k + 1) * p.nj * p.nip; ++c) cs[c] = 1.0;
        if ((rc = upload<T>(ctx, g.csfrac, cs))) return rc;
    }
    for (int k = 0; k < p.nk; k++)
        for (int j = 0; j < p.nj; j++)
            for (int i = 0; i < p.ni; i++) hv[cidx(i, j, k, p.nj, p.nip)] = hpre;
    for (int k = 0; k < p.nk; k++)
        for (int j = 0; j < p.nj; j++) {
            hv[cidx(0, j, k, p.nj, p.nip)] = enth(q.tempwest);
            hv[cidx(p.nim1, j, k, p.nj, p.nip)] = enth(q.tempeast);
        }
    for (int j = 0; j < p.nj; j++)
        for (int i = 0; i < p.ni; i++) hv[cidx(i, j, 0, p.nj, p.nip)] = enth(q.tempbottom);
    for (int k = 0; k < p.nk; k++)
        for (int i = 0; i < p.ni; i++) hv[cidx(i, p.njm1, k, p.nj, p.nip)] = enth(q.tempnorth);
    if ((rc = upload<T>(ctx, g.h, hv))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    // powder bed: only the first layer starts active (PrintManager.cpp:67-73)
    return set_active_nk<T>(ctx, I, ctx->nk_active);
}

static bool phase_ok(int phase) { return phase >= 1 && phase <= AMCFD_PHASE_SPECIES; }

// The track id updateSolutions tags melted cells with (CFDSolverManager.cpp:2638-2644):
// that of the first toolpath row not earlier than the current time.  The
// reference leaves it undefined without a toolpath or past the last row; 0 here.
static int track_id(const amcfd_ctx *ctx)
{
    int id = 0;
    for (int i = (int)ctx->tool_id.size(); i > 0; i--)
        if (ctx->timet <= ctx->tool[4 * (i - 1)]) id = ctx->tool_id[i - 1];
    return id;
}

static void drop_graphs(amcfd_ctx *ctx)
{
    for (auto &plane : ctx->gexec)
        for (auto &row : plane)
            for (auto &ge : row)
                if (ge) {
                    cudaGraphExecDestroy(ge);
                    ge = nullptr;
                }
    for (auto &ge : ctx->gloop)
        if (ge) {
            cudaGraphExecDestroy(ge);
            ge = nullptr;
        }
}

// ---- one outer iteration -----------------------------------------------------------------
template <typename T>
static void swap_props(Inst<T> &I)
{
    std::swap(I.g.diff_cur, I.g.diff_nxt);
    std::swap(I.g.rho_cur, I.g.rho_nxt);
    std::swap(I.g.vis_cur, I.g.vis_nxt);
}

// The one-CTA momentum chain serves red-black runs whose melt-pool box, as of
// the last outer iteration, fits its shared memory (it stays correct, only
// slower, if the box has grown past that since).
// In the automatic mode the one-CTA chain is taken only where the cooperative box
// solve is unavailable: on the 400x200x100 deck the cooperative path took 0.099
// against 0.139 ms an outer iteration for boxes of 1300-2200 cells and 0.100
// against 0.176 for 2600-3100 cells; on the 120x60x40 deck 0.093 against 0.101
// (1400-1600 cells) and the same 0.090 for 800-1000 cells.
template <typename T>
static bool small_allowed(const amcfd_ctx *ctx, const Inst<T> &I)
{
    if (ctx->order != AMCFD_ORDER_REDBLACK || ctx->small_mode == 1) return false;
    return ctx->small_mode == -1 || I.box_grid == 0;
}
template <typename T>
static bool mom_small(const amcfd_ctx *ctx, const Inst<T> &I)
{
    return small_allowed(ctx, I) && ctx->last_box >= 0 && ctx->last_box <= mom_small_capacity<T>(I);
}

// The energy line solve: with defect correction the FP32 passes on the correction.
template <typename T>
static void energy_sweeps(Inst<T> &I)
{
    if constexpr (sizeof(T) == sizeof(double)) {
        if (I.dc_on) {
            launch_dc_sweeps(I);
            return;
        }
    }
    launch_energy_sweeps<T>(I);
}

// H->T; with defect correction the correction is added to the FP64 enthalpy first.
template <typename T>
static void h2t(Inst<T> &I)
{
    if constexpr (sizeof(T) == sizeof(double))
        if (I.dc_on) launch_dc_apply(I);
    launch_h2t<T>(I);
}

template <typename T>
static void run_phase_impl(amcfd_ctx *ctx, Inst<T> &I, int phase)
{
    switch (phase) {
    case AMCFD_PHASE_ENERGY_ASSEMBLE:
        launch_energy_bc<T>(I);
        launch_energy_assemble<T>(I);
        launch_block_correct<T>(I);
        break;
    case AMCFD_PHASE_ENERGY_SOLVE:
        launch_energy_factor<T>(I);
        energy_sweeps<T>(I);
        break;
    case AMCFD_PHASE_H2T: h2t<T>(I); break;
    case AMCFD_PHASE_MELTPOOL: launch_meltpool<T>(I); break;
    case AMCFD_PHASE_MOMENTUM: launch_momentum<T>(I, mom_small<T>(ctx, I)); break;
    case AMCFD_PHASE_CONVERGE:
        launch_converge<T>(I, ctx->prm.nonlintol);
        swap_props<T>(I);
        break;
    case AMCFD_PHASE_UPDATE:
        I.trackindx = (double)ctx->trackindx;
        I.trackid = track_id(ctx);
        launch_update_solutions<T>(I);
        launch_species_update<T>(I);
        break;
    case AMCFD_PHASE_SPECIES: launch_species<T>(I); break;
    default: break;
    }
}

// CFDSolverManager::generateGrid with the mesh following the beam (:72-124, 345-346):
// the moving zones shift by the beam's displacement of this step, the grid is
// rebuilt, its metrics replace the device copies and the fields are remapped.
// Runs after the step's laser update, whose surface flux used the old grid.
template <typename T>
static int move_mesh(amcfd_ctx *ctx, Inst<T> &I)
{
    amcfd_params &p = ctx->prm;
    const double dx = ctx->beamposx - ctx->oldbeamposx, dy = ctx->beamposy - ctx->oldbeamposy;
    const int dirx = dx < 0 ? -1 : 1, diry = dy < 0 ? -1 : 1;
    const int ix = p.xmoveindex, iy = ctx->steadylength ? p.ymoveindex : p.xmoveindex;
    p.xzone[ix - 1] += dx;
    p.xzone[ix + 1] -= dx;
    p.yzone[iy - 1] += dy;
    p.yzone[iy + 1] -= dy;
    // staged in pinned memory so that the copies stay asynchronous; event 8 marks
    // the end of the previous step's copies out of the staging
    CK(cudaEventSynchronize(ctx->ev[8]));
    double *st = ctx->mesh_pinned;
    std::copy(ctx->x.begin(), ctx->x.begin() + ctx->ni, st);
    std::copy(ctx->y.begin(), ctx->y.begin() + ctx->nj, st + ctx->ni);
    CK(cudaMemcpyAsync(ctx->mesh_old, st, ((size_t)ctx->ni + ctx->nj) * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    st += (size_t)ctx->ni + ctx->nj;
    build_grid(ctx, ctx->nk_active);
    const std::vector<double> *src[12] = {&ctx->x, &ctx->y, &ctx->z, &ctx->xu, &ctx->yv, &ctx->zw,
                                          &ctx->dxpwinv, &ctx->dypsinv, &ctx->dzpbinv,
                                          &ctx->fracx, &ctx->fracy, &ctx->fracz};
    for (int a = 0; a < 12; a++) {
        std::copy(src[a]->begin(), src[a]->end(), st);
        CK(cudaMemcpyAsync(ctx->dmetric[a], st, src[a]->size() * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
        st += src[a]->size();
    }
    CK(cudaEventRecord(ctx->ev[8], ctx->stream));
    launch_remap<T>(I, ctx->mesh_old, ctx->mesh_old + ctx->ni, dirx, diry);
    ctx->launches += 2;
    return 0;
}

static int begin_step(amcfd_ctx *ctx)
{
    const amcfd_params &p = ctx->prm;
    if (p.nvardt > 0) {
        const int n = p.nvardt;
        if (ctx->timet > ctx->vardt[3 * ctx->vardt_state] && ctx->vardt_state < n - 1)
            ctx->vardt_state += 1;
        ctx->delt = ctx->vardt[3 * ctx->vardt_state + 1];
        ctx->outtime = ctx->vardt[3 * ctx->vardt_state + 2];
    }
    ctx->timet += ctx->delt;
    if (!p.steady) laser_coords(ctx);
    if (p.powderbed) {
        const int rc = ctx->precision == AMCFD_PREC_FP64 ? set_active_nk<double>(ctx, ctx->I64, ctx->nk_active)
                                                         : set_active_nk<float>(ctx, ctx->I32, ctx->nk_active);
        if (rc) return rc;
    }
    Status *h = ctx->st_host;
    h->timet = ctx->timet;
    h->delt = ctx->delt;
    h->beamposx = ctx->beamposx;
    h->beamposy = ctx->beamposy;
    h->scanvel = ctx->scanvel;
    h->powerindicator = ctx->powerindicator;
    h->istart = ctx->istart;
    h->jstart = ctx->jstart;
    h->lp_niter = 0;
    h->lp_box = ctx->last_box;
    h->lp_mode = 0;
    h->lp_small = 0;
    // the per-step block is the leading members of Status, up to heat_iter
    CK(cudaMemcpyAsync(ctx->st_dev, h, offsetof(Status, heat_iter), cudaMemcpyHostToDevice,
                       ctx->stream));
    if (ctx->events) cudaEventRecord(ctx->ev[10], ctx->stream);
    if (ctx->precision == AMCFD_PREC_FP64)
        launch_laser<double>(ctx->I64);
    else
        launch_laser<float>(ctx->I32);
    if (ctx->events) {
        cudaEventRecord(ctx->ev[11], ctx->stream);
        cudaEventSynchronize(ctx->ev[11]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[10], ctx->ev[11]);
        ctx->last_ms[6] += ms;
    }
    ctx->launches += 1;
    ctx->niter = 0;
    if (p.movingmesh) {
        const int rc = ctx->precision == AMCFD_PREC_FP64 ? move_mesh<double>(ctx, ctx->I64)
                                                         : move_mesh<float>(ctx, ctx->I32);
        if (rc) return rc;
    }
    return 0;
}

static int read_status(amcfd_ctx *ctx)
{
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st_dev, sizeof(Status), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    const Status *s = ctx->st_host;
    if (s->error) {
        char buf[160];
        snprintf(buf, sizeof buf, "device wait gave up (code %d, line %d)", s->error, s->error_where);
        ctx->err = buf;
        return s->error;
    }
    if (s->nonfinite) return fail(ctx, AMCFD_E_NONFINITE, "non-finite residual or temperature");
    return 0;
}

// Kernel launches issued by one phase (the launch counter of the bench).
static long long phase_launches(const amcfd_ctx *ctx, int phase, bool small)
{
    const long long sweeps = ctx->order == AMCFD_ORDER_EXACT ? 1 : 8;
    // whole-domain red-black solves: one pipelined launch, or one per pass
    const bool fp64 = ctx->precision == AMCFD_PREC_FP64;
    const long long phi_sweeps = (fp64 ? ctx->I64.pipe_grid : ctx->I32.pipe_grid) > 0 ? 1 : sweeps;
    const long long energy_sweeps = (ctx->dc ? ctx->I64.pipe_grid_dc > 0 : phi_sweeps == 1) ? 1 : sweeps;
    switch (phase) {
    case AMCFD_PHASE_LASER: return 1;
    case AMCFD_PHASE_ENERGY_ASSEMBLE: return 3;
    case AMCFD_PHASE_ENERGY_SOLVE: return ctx->order == AMCFD_ORDER_EXACT ? 1 + sweeps : energy_sweeps;
    case AMCFD_PHASE_H2T: return ctx->dc ? 2 : 1;
    case AMCFD_PHASE_MELTPOOL: return 1;
    case AMCFD_PHASE_MOMENTUM: {
        // cooperative: cleanVelocities, applyBCs(1), then per equation its assembly and
        // one launch for the solve and what follows it; otherwise per equation
        // applyBCs, assembly, factorisation and sweeps, then correctPressure
        const bool coop = (ctx->precision == AMCFD_PREC_FP64 ? ctx->I64.box_grid : ctx->I32.box_grid) > 0;
        const int tickets = ctx->order == AMCFD_ORDER_EXACT ? 1 : 0;
        if (small) return ctx->mom_cluster > 1 ? 14 : 9;
        return coop ? 2 + 4 * 2 : tickets + 1 + 4 * (3 + sweeps) + 2 + 1;
    }
    case AMCFD_PHASE_CONVERGE: return 1;
    case AMCFD_PHASE_UPDATE: return ctx->prm.species ? 2 : 1;
    case AMCFD_PHASE_SPECIES: return ctx->prm.species ? (ctx->order == AMCFD_ORDER_EXACT ? 4 : 3) + phi_sweeps : 0;
    default: return 0;
    }
}

// Timing slots of amcfd_last_timing (accumulated device ms while profiling):
// 0 energy BC+assembly+block correction, 1 line factorisation, 2 energy line
// sweeps, 3 H->T + melt pool, 4 momentum chain, 5 convergence, 6 laser,
// 7 push-back, 8 outer iterations run, 9 energy-sweep launches, 10 species.
// Event record; under stream capture it must become an event node of the graph
// (the external flag is only valid while capturing).
static inline void rec(amcfd_ctx *ctx, int q, bool capturing)
{
    if (capturing)
        cudaEventRecordWithFlags(ctx->ev[q], ctx->stream, cudaEventRecordExternal);
    else
        cudaEventRecord(ctx->ev[q], ctx->stream);
}

// The launch sequence of one outer iteration (iterativeLoopSolve body,
// CFDSolverManager.cpp:601-719); ends with the property-buffer swap.
template <typename T>
static void launch_iteration(amcfd_ctx *ctx, Inst<T> &I, bool capturing)
{
    const bool ev = ctx->events;
    if (ev) rec(ctx, 0, capturing);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_ENERGY_ASSEMBLE);
    if (ev) rec(ctx, 1, capturing);
    launch_energy_factor<T>(I);
    if (ev) rec(ctx, 2, capturing);
    energy_sweeps<T>(I);
    if (ev) rec(ctx, 3, capturing);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_H2T);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_MELTPOOL);
    if (ev) rec(ctx, 4, capturing);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_MOMENTUM);
    if (ev) rec(ctx, 5, capturing);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_SPECIES);
    if (ev) rec(ctx, 7, capturing);
    run_phase_impl<T>(ctx, I, AMCFD_PHASE_CONVERGE);
    if (ev) rec(ctx, 6, capturing);
}

// Graph captures of all contexts of the process, one at a time: a capture must
// not overlap anything that loads a kernel module (a first launch of a kernel),
// which a capture in another thread may do.
static std::mutex g_capture_mu;

// One outer iteration replayed from a CUDA graph.  Every launch of an iteration
// has a fixed grid and reads its data-dependent extents (the momentum box, the
// sweep tickets) from the device status block, so the graph captured on the
// first iteration of each parity is valid for every later one.
template <typename T>
static int launch_iteration_graph(amcfd_ctx *ctx, Inst<T> &I)
{
    const int par = (const void *)I.g.diff_cur == ctx->diff_a ? 0 : 1;
    cudaGraphExec_t &ge = ctx->gexec[ctx->events ? 1 : 0][par][mom_small<T>(ctx, I) ? 1 : 0];
    if (!ge) {
        std::lock_guard<std::mutex> lock(g_capture_mu);
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        launch_iteration<T>(ctx, I, true);  // swaps the property buffers
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (e != cudaSuccess || !graph) {
            cudaGetLastError();
            ctx->err = std::string("graph capture: ") + cudaGetErrorString(e);
            return AMCFD_E_CUDA;
        }
        e = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ge = nullptr;
            ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(e);
            return AMCFD_E_CUDA;
        }
    } else {
        swap_props<T>(I);
    }
    CK(cudaGraphLaunch(ge, ctx->stream));
    return 0;
}

// ---- the outer loop of a step as one CUDA graph ----------------------------------------
// Outer iterations 1..maxit are chained by conditional if-nodes: iteration k+1
// runs when the convergence kernel of iteration k sets its condition (the host
// loop's test: not converged, finite, no device error, fewer than maxit
// iterations), and an if/else node in each iteration takes the momentum path
// that the host would have chosen from the previous iteration's box.  The chain
// has no loop node, so a condition that is never set only ends the step early.
// Iterations alternate the property parity, so the graph is built per parity of
// its first iteration.  The host launches it once per step and reads the status
// once.
constexpr int kMaxChain = 64;  // longer maxit: the host drives the loop

template <typename T>
static int build_loop_graph(amcfd_ctx *ctx, Inst<T> &I, cudaGraphExec_t &ge)
{
    std::lock_guard<std::mutex> lock(g_capture_mu);
    const int maxit = ctx->prm.maxit;
    const int cap = small_allowed(ctx, I) ? mom_small_capacity<T>(I) : -1;
    const double tol = ctx->prm.nonlintol;
    std::vector<cudaGraph_t> parts;  // captured pieces; child nodes hold copies
    cudaGraph_t top = nullptr;
    cudaError_t err = cudaSuccess;
    auto keep = [&](cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
        return err == cudaSuccess;
    };
    auto capture = [&](auto &&launch) -> cudaGraph_t {
        if (!keep(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal))) return nullptr;
        launch();
        cudaGraph_t g = nullptr;
        if (!keep(cudaStreamEndCapture(ctx->stream, &g))) return nullptr;
        parts.push_back(g);
        return g;
    };
    auto child = [&](cudaGraph_t parent, cudaGraphNode_t dep, cudaGraph_t g) -> cudaGraphNode_t {
        cudaGraphNode_t n = nullptr;
        if (err == cudaSuccess) keep(cudaGraphAddChildGraphNode(&n, parent, dep ? &dep : nullptr, dep ? 1 : 0, g));
        return n;
    };
    auto cond = [&](cudaGraph_t parent, cudaGraphNode_t dep, cudaGraphConditionalHandle h, unsigned size,
                    cudaGraph_t *bodies) -> cudaGraphNode_t {
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = size;
        cudaGraphNode_t n = nullptr;
        if (err == cudaSuccess && keep(cudaGraphAddNode(&n, parent, dep ? &dep : nullptr, dep ? 1 : 0, &np)))
            for (unsigned q = 0; q < size; ++q) bodies[q] = np.conditional.phGraph_out[q];
        return n;
    };
    keep(cudaGraphCreate(&top, 0));
    std::vector<cudaGraphConditionalHandle> hc(maxit + 1), hm(maxit + 1);
    for (int k = 1; k <= maxit && err == cudaSuccess; ++k) {
        keep(cudaGraphConditionalHandleCreate(&hm[k], top, 0, cudaGraphCondAssignDefault));
        if (k < maxit) keep(cudaGraphConditionalHandleCreate(&hc[k], top, 0, cudaGraphCondAssignDefault));
    }
    // the energy part and the momentum paths depend only on the parity
    cudaGraph_t energy[2] = {}, mom_small_g[2] = {}, mom_grid_g[2] = {};
    for (int q = 0; q < 2; ++q) {
        energy[q] = capture([&] {
            run_phase_impl<T>(ctx, I, AMCFD_PHASE_ENERGY_ASSEMBLE);
            run_phase_impl<T>(ctx, I, AMCFD_PHASE_ENERGY_SOLVE);
            run_phase_impl<T>(ctx, I, AMCFD_PHASE_H2T);
            run_phase_impl<T>(ctx, I, AMCFD_PHASE_MELTPOOL);
        });
        if (cap >= 0) mom_small_g[q] = capture([&] { launch_momentum<T>(I, true); });
        mom_grid_g[q] = capture([&] { launch_momentum<T>(I, false); });
        swap_props<T>(I);
    }
    cudaGraph_t g_init = capture([&] {
        const LoopCtl lc{0, hm[1], 1, 1, maxit, cap};
        launch_loop_init(ctx->st_dev, lc, I.stream);
    });
    // top: init, iteration 1, then iterations 2..maxit in sequence, each inside an
    // if-node on the condition its predecessor sets (a skipped iteration leaves the
    // next condition at its default 0, so the rest of the chain is skipped too)
    cudaGraphNode_t last = child(top, nullptr, g_init);
    for (int k = 1; k <= maxit && err == cudaSuccess; ++k) {
        const int q = (k - 1) & 1;  // parity relative to the first iteration
        cudaGraph_t g = top;
        cudaGraphNode_t n = last;
        if (k > 1) {
            cudaGraph_t body[1] = {};
            last = cond(top, last, hc[k - 1], 1, body);
            g = body[0];
            n = nullptr;
        }
        if (err != cudaSuccess) break;
        n = child(g, n, energy[q]);
        cudaGraph_t br[2] = {};
        n = cond(g, n, hm[k], 2, br);
        if (err != cudaSuccess) break;
        if (cap >= 0) child(br[0], nullptr, mom_small_g[q]);
        child(br[1], nullptr, mom_grid_g[q]);
        // species and the convergence test, with the loop control of iteration k
        const LoopCtl lc{k < maxit ? hc[k] : 0, k < maxit ? hm[k + 1] : 0, 1, k < maxit ? 1 : 0, maxit, cap};
        if (q) swap_props<T>(I);
        cudaGraph_t tail = capture([&] {
            run_phase_impl<T>(ctx, I, AMCFD_PHASE_SPECIES);
            launch_converge<T>(I, tol, lc);
        });
        if (q) swap_props<T>(I);
        n = child(g, n, tail);
        if (k == 1) last = n;
    }
    if (err == cudaSuccess) keep(cudaGraphInstantiate(&ge, top, 0));
    for (cudaGraph_t g : parts)
        if (g) cudaGraphDestroy(g);
    if (top) cudaGraphDestroy(top);
    if (err != cudaSuccess) {
        cudaGetLastError();
        ge = nullptr;
        ctx->err = std::string("outer-loop graph: ") + cudaGetErrorString(err);
        return AMCFD_E_CUDA;
    }
    return 0;
}

// Kernel launches of one outer iteration on the small-box or the grid momentum path.
static long long iteration_launches(const amcfd_ctx *ctx, bool small)
{
    long long n = 0;
    for (int ph = AMCFD_PHASE_ENERGY_ASSEMBLE; ph <= AMCFD_PHASE_CONVERGE; ++ph) n += phase_launches(ctx, ph, small);
    return n + phase_launches(ctx, AMCFD_PHASE_SPECIES, small);
}

template <typename T>
static int outer_loop_graph(amcfd_ctx *ctx, Inst<T> &I)
{
    const int par = (const void *)I.g.diff_cur == ctx->diff_a ? 0 : 1;
    cudaGraphExec_t &ge = ctx->gloop[par];
    int rc;
    if (!ge && (rc = build_loop_graph<T>(ctx, I, ge))) return rc;
    CK(cudaGraphLaunch(ge, ctx->stream));
    rc = read_status(ctx);
    const Status *s = ctx->st_host;
    const int n = s->lp_niter;
    ctx->niter = n;
    ctx->itertot += n;
    ctx->launches += 1 + (long long)s->lp_small * iteration_launches(ctx, true) +
                     (long long)(n - s->lp_small) * iteration_launches(ctx, false);
    ctx->last_box = s->lp_box;
    if (n & 1) swap_props<T>(I);
    return rc;
}

// Timing slots of amcfd_last_timing (accumulated device ms while profiling):
// 0 energy BC+assembly+block correction, 1 line factorisation, 2 energy line
// sweeps, 3 H->T + melt pool, 4 momentum chain, 5 convergence, 6 laser,
// 7 push-back, 8 outer iterations run, 9 energy-sweep launches.
template <typename T>
static int outer_loop(amcfd_ctx *ctx, Inst<T> &I)
{
    const int maxit = ctx->prm.maxit;
    int rc;
    if (ctx->use_graphs && !ctx->events && !ctx->host_loop && ctx->niter == 0 && maxit >= 1 &&
        maxit <= kMaxChain)
        return outer_loop_graph<T>(ctx, I);
    while (ctx->niter < maxit) {
        ctx->niter++;
        ctx->itertot++;
        const bool ev = ctx->events;
        const bool small = mom_small<T>(ctx, I);
        if (ctx->use_graphs) {
            if ((rc = launch_iteration_graph<T>(ctx, I))) return rc;
        } else {
            launch_iteration<T>(ctx, I, false);
        }
        for (int ph = AMCFD_PHASE_ENERGY_ASSEMBLE; ph <= AMCFD_PHASE_CONVERGE; ++ph)
            ctx->launches += phase_launches(ctx, ph, small);
        ctx->launches += phase_launches(ctx, AMCFD_PHASE_SPECIES, small);
        if ((rc = read_status(ctx))) return rc;
        ctx->last_box = ctx->st_host->momentum_active ? ctx->st_host->box_cells : 0;
        if (ev) {
            // events 0..5 bound slots 0..4; the species solve runs between events 5
            // and 7, the convergence test between 7 and 6
            for (int q = 0; q < 5; q++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ctx->ev[q], ctx->ev[q + 1]);
                ctx->last_ms[q] += ms;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev[5], ctx->ev[7]);
            ctx->last_ms[10] += ms;
            ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev[7], ctx->ev[6]);
            ctx->last_ms[5] += ms;
            ctx->last_ms[8] += 1.0;
            ctx->last_ms[9] += ctx->order == AMCFD_ORDER_EXACT
                                   ? 1.0
                                   : (double)phase_launches(ctx, AMCFD_PHASE_ENERGY_SOLVE, small);
        }
        if (ctx->st_host->converged) break;
    }
    return 0;
}

static void fill_report(amcfd_ctx *ctx, amcfd_step_report *r)
{
    if (!r) return;
    const Status *s = ctx->st_host;
    memset(r, 0, sizeof(*r));
    r->timet = ctx->timet;
    r->niter = ctx->niter;
    r->itertot = ctx->itertot;
    r->resorh = s->resorh; r->resorm = s->resorm; r->resoru = s->resoru;
    r->resorv = s->resorv; r->resorw = s->resorw;
    r->tpeak = s->tpeak; r->alen = s->alen; r->depth = s->depth; r->width = s->width;
    r->ratio = s->ratio; r->heatinlaser = s->heatinlaser; r->ahtoploss = s->ahtoploss;
    r->accul = s->accul; r->heatout = s->heatout; r->heatvol = s->heatvol;
    r->beamposx = ctx->beamposx; r->beamposy = ctx->beamposy; r->scanvel = ctx->scanvel;
    r->istat = s->istat; r->iend = s->iend; r->jstat = s->jstat; r->jend = s->jend;
    r->kstat = s->kstat; r->jstart = ctx->jstart; r->powerindicator = ctx->powerindicator;
    r->momentum_cells = s->box_cells;
    r->fallback = ctx->ws_fallback;
    r->resorc = s->resorc;
    r->nk_active = ctx->nk_active;
    r->trackindx = ctx->trackindx;
    r->steadylength = ctx->steadylength;
}

// ---- learned warm start ----------------------------------------------------------------
// Energy residual of the current state (assembly + calculateResiduals(5),
// CFDSolverManager.cpp:2073-2101) without touching the step's BC or source
// state; a non-finite value comes back as +inf and clears the device flag.
template <typename T>
static int ws_residual(amcfd_ctx *ctx, Inst<T> &I, double &r)
{
    launch_energy_assemble<T>(I);
    launch_block_correct<T>(I);
    CK(cudaMemcpyAsync(ctx->st_host, ctx->st_dev, sizeof(Status), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    if (ctx->st_host->error) return read_status(ctx);
    r = ctx->st_host->resorh;
    if (ctx->st_host->nonfinite || !std::isfinite(r)) {
        const int zero = 0;
        CK(cudaMemcpyAsync(&ctx->st_dev->nonfinite, &zero, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        r = INFINITY;
    }
    ctx->launches += 3;
    return 0;
}

// Start of a step (after the laser moved): features of the current state,
// snapshot of h, p, T, f_l; in predict mode the network's increments (full,
// then half) are applied and the first that lowers the energy residual of the
// start of the step is kept.
template <typename T>
static int ws_before(amcfd_ctx *ctx, Inst<T> &I)
{
    T *const *save = reinterpret_cast<T *const *>(ctx->ws_save);
    const double power = ctx->prm.alaspow * (double)ctx->powerindicator;
    ws_features<T>(I, ctx->ws_feat, ctx->ws_target, ctx->beamposx, ctx->beamposy, power);
    ws_copy<T>(I, save, 0);
    ctx->launches += 2;
    ctx->ws_fallback = 0;
    if (ctx->ws_mode != AMCFD_WS_PREDICT && ctx->ws_mode != AMCFD_WS_PREDICT_H) return 0;
    int rc;
    double r0, r1;
    if ((rc = ws_residual<T>(ctx, I, r0))) return rc;
    if ((rc = amcfd_net_forward(ctx->net, ctx->ws_feat, ctx->ni, ctx->nj, ctx->nk, ctx->ws_y)))
        return fail(ctx, rc, std::string("warm-start network: ") + amcfd_net_last_error(ctx->net));
    for (double alpha : {1.0, 0.5}) {
        ws_apply<T>(I, ctx->ws_y, alpha, ctx->ws_mode == AMCFD_WS_PREDICT ? 1 : 0);
        if ((rc = ws_residual<T>(ctx, I, r1))) return rc;
        ctx->launches += 1;
        if (r1 < r0) {
            ctx->ws_accepted++;
            return 0;
        }
        ws_copy<T>(I, save, 1);
        ctx->launches += 1;
    }
    ctx->ws_rejected++;
    ctx->ws_fallback = 1;
    return 0;
}

template <typename T>
static void ws_after(amcfd_ctx *ctx, Inst<T> &I)
{
    ws_target<T>(I, reinterpret_cast<T *const *>(ctx->ws_save), ctx->ws_target);
    ctx->launches += 1;
}

// ---- autotuner ------------------------------------------------------------------------
// At creation (opt-in): the energy assembly with 4, 8 and 16 planes per CTA and a
// factorising plus a plain red-black pass with 2, 4 and 8 lines per CTA, each timed
// with CUDA events on the context stream (one untimed round, then the minimum of
// three rounds in rotated order) on this grid; the fastest of each is kept unless
// the options pin it.  The assembly runs in place (everything it writes is formed
// again by the first outer iteration); the sweep passes run on a scratch field.
template <typename T>
static int autotune(amcfd_ctx *ctx, Inst<T> &I)
{
    cudaEvent_t e0 = ctx->ev[14], e1 = ctx->ev[15];
    const int segs[3] = {4, 8, 16}, warps[3] = {2, 4, 8}, strides[3] = {8, 16, 32};
    // the line sweeps: with the passes pipelined in one launch, the planes between
    // passes in its work order; otherwise the lines per CTA of the per-pass launches
    bool pipe = I.pipe_grid > 0;
    if constexpr (sizeof(T) == sizeof(double))
        if (I.dc_on) pipe = I.pipe_grid_dc > 0;
    float best_asm[3], best_sw[3];
    for (int c = 0; c < 3; ++c) best_asm[c] = best_sw[c] = INFINITY;
    auto set_seg = [&](int seg) {
        I.asm_kseg = seg;
        I.asm_grid = energy_assemble_grid(I.p, seg);
        I.nb_asm = I.asm_grid.x * I.asm_grid.y * I.asm_grid.z;
        I.g.npart = I.asm_grid.y * I.asm_grid.z;
    };
    auto sweep_probe = [&](int c) {
        if (pipe) I.pipe_stride = strides[c];
        if constexpr (sizeof(T) == sizeof(double)) {
            if (I.dc_on) {
                if (pipe)
                    launch_dc_sweeps(I);  // overwrites only the correction
                else
                    launch_dc_sweep_probe(I, warps[c]);
                return;
            }
        }
        if (pipe)
            launch_phi_sweeps<T>(I, I.mom_scratch);  // a scratch field
        else
            launch_sweep_probe<T>(I, I.mom_scratch, warps[c]);
    };
    const bool tune_sweep = ctx->order == AMCFD_ORDER_REDBLACK && (pipe || !ctx->sweep_warps);
    for (int round = 0; round < 4; ++round)
        for (int q = 0; q < 3; ++q) {
            const int c = (q + round) % 3;
            float ms = 0.f;
            if (!ctx->asm_kseg) {
                set_seg(segs[c]);
                CK(cudaEventRecord(e0, ctx->stream));
                launch_energy_assemble<T>(I);
                CK(cudaEventRecord(e1, ctx->stream));
                CK(cudaEventSynchronize(e1));
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (round > 0) best_asm[c] = std::min(best_asm[c], ms);
            }
            if (tune_sweep && (pipe || warps[c] <= I.sweep_warps_max)) {
                CK(cudaEventRecord(e0, ctx->stream));
                sweep_probe(c);
                CK(cudaEventRecord(e1, ctx->stream));
                CK(cudaEventSynchronize(e1));
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (round > 0) best_sw[c] = std::min(best_sw[c], ms);
            }
        }
    CK(cudaGetLastError());
    if (!ctx->asm_kseg) {
        const int c = (int)(std::min_element(best_asm, best_asm + 3) - best_asm);
        set_seg(segs[c]);
        ctx->asm_kseg = segs[c];
        for (int q = 0; q < 3; ++q) ctx->tune_ms[q] = best_asm[q];
    }
    if (tune_sweep) {
        const int c = (int)(std::min_element(best_sw, best_sw + 3) - best_sw);
        if (pipe) {
            I.pipe_stride = strides[c];
        } else {
            I.sweep_warps = warps[c];
            ctx->sweep_warps = warps[c];
        }
        for (int q = 0; q < 3; ++q) ctx->tune_ms[3 + q] = best_sw[q];
    }
    ctx->launches += 4 * 3 * 3;
    return 0;
}

// =========================================================================================
extern "C" {

int amcfd_tuning(const amcfd_ctx *ctx, int *asm_kseg, int *sweep_warps, double *times)
{
    if (!ctx) return AMCFD_E_ARG;
    const int seg = ctx->precision == AMCFD_PREC_FP64 ? ctx->I64.asm_kseg : ctx->I32.asm_kseg;
    const int w = ctx->precision == AMCFD_PREC_FP64 ? ctx->I64.sweep_warps : ctx->I32.sweep_warps;
    if (asm_kseg) *asm_kseg = seg;
    if (sweep_warps) *sweep_warps = w;
    if (times)
        for (int q = 0; q < 6; ++q) times[q] = ctx->tune_ms[q];
    return 0;
}

int amcfd_pipe_stride(const amcfd_ctx *ctx, int *stride)
{
    if (!ctx || !stride) return AMCFD_E_ARG;
    const bool fp64 = ctx->precision == AMCFD_PREC_FP64;
    const int grid = fp64 ? (ctx->dc ? ctx->I64.pipe_grid_dc : ctx->I64.pipe_grid) : ctx->I32.pipe_grid;
    *stride = grid > 0 ? (fp64 ? ctx->I64.pipe_stride : ctx->I32.pipe_stride) : 0;
    return 0;
}

int amcfd_create(const amcfd_params *params, const amcfd_options *opts, amcfd_ctx **out)
{
    if (!params || !out) return AMCFD_E_ARG;
    *out = nullptr;
    amcfd_ctx *ctx = new amcfd_ctx();
    *out = ctx;
    ctx->prm = *params;
    amcfd_params &p = ctx->prm;
    if (p.freesurface && (p.fs_maxiterenergy < 0 || p.fs_maxiterbisect < 0))
        return fail(ctx, AMCFD_E_ARG, "*TRACK_ENERGY_BASED_FREE_SURFACE iteration counts must not be negative");
    if (p.movingmesh) {
        // the zones either side of the moving one change length; before the melt pool
        // reaches a steady length the y shift uses the x zone index (CFDSolverManager.cpp:108-115)
        const int ix = p.xmoveindex, iy = p.ymoveindex;
        if (ix < 1 || ix > p.nzx - 2 || iy < 1 || iy > p.nzy - 2 || ix > p.nzy - 2)
            return fail(ctx, AMCFD_E_ARG, "*ACTIVATE_MOVING_MESH zones need a zone on either side");
    }
    if (p.nzx < 1 || p.nzy < 1 || p.nzz < 1 || p.nzx > AMCFD_MAX_ZONES || p.nzy > AMCFD_MAX_ZONES ||
        p.nzz > AMCFD_MAX_ZONES)
        return fail(ctx, AMCFD_E_ARG, "bad zone counts");
    if (p.acpa == 0.0) return fail(ctx, AMCFD_E_ARG, "acpa must be non-zero (H->T divides by it)");
    if (opts) {
        ctx->device = opts->device;
        ctx->order = opts->order;
        ctx->precision = opts->precision;
        ctx->use_graphs = opts->use_graphs != 0;
        if (opts->no_small_box < -1 || opts->no_small_box > 1)
            return fail(ctx, AMCFD_E_ARG, "no_small_box must be -1, 0 or 1");
        ctx->small_mode = opts->no_small_box;
        ctx->host_loop = opts->host_loop != 0;
        if (opts->wait_polls < 0) return fail(ctx, AMCFD_E_ARG, "wait_polls must not be negative");
        ctx->wait_polls = opts->wait_polls;
        if (opts->asm_kseg != 0 && opts->asm_kseg != 4 && opts->asm_kseg != 8 && opts->asm_kseg != 16)
            return fail(ctx, AMCFD_E_ARG, "asm_kseg must be 0, 4, 8 or 16");
        if (opts->sweep_warps != 0 && opts->sweep_warps != 2 && opts->sweep_warps != 4 && opts->sweep_warps != 8)
            return fail(ctx, AMCFD_E_ARG, "sweep_warps must be 0, 2, 4 or 8");
        if (opts->mom_cluster != 0 && opts->mom_cluster != 1 && opts->mom_cluster != 2 && opts->mom_cluster != 4 &&
            opts->mom_cluster != 8 && opts->mom_cluster != 16)
            return fail(ctx, AMCFD_E_ARG, "mom_cluster must be 0, 1, 2, 4, 8 or 16");
        ctx->mom_cluster_req = opts->mom_cluster;
        ctx->serial_launch = opts->serial_launch != 0;
        ctx->pass_launch = opts->pass_launch != 0;
        if (opts->box_ctas < 0) return fail(ctx, AMCFD_E_ARG, "box_ctas must not be negative");
        ctx->box_ctas = opts->box_ctas;
        ctx->autotune = opts->autotune != 0;
        ctx->asm_kseg = opts->asm_kseg;
        ctx->sweep_warps = opts->sweep_warps;
    }
    if (ctx->order != AMCFD_ORDER_EXACT && ctx->order != AMCFD_ORDER_REDBLACK)
        return fail(ctx, AMCFD_E_ARG, "unknown line-sweep order");
    if (ctx->precision == AMCFD_PREC_FP32_DC) {
        if (ctx->order != AMCFD_ORDER_REDBLACK)
            return fail(ctx, AMCFD_E_ARG, "defect correction runs in red-black order only");
        ctx->dc = true;
        ctx->precision = AMCFD_PREC_FP64;  // the FP64 instance carries the state
    }
    if (ctx->precision != AMCFD_PREC_FP64 && ctx->precision != AMCFD_PREC_FP32)
        return fail(ctx, AMCFD_E_ARG, "unknown precision");
    if (p.udtoolpath) {
        if (p.ntool < 2 || !p.tool_txyz || !p.tool_on || !p.tool_id)
            return fail(ctx, AMCFD_E_ARG, "toolpath needs at least 2 rows");
        ctx->tool.assign(p.tool_txyz, p.tool_txyz + 4 * p.ntool);
        ctx->tool_on.assign(p.tool_on, p.tool_on + p.ntool);
        ctx->tool_id.assign(p.tool_id, p.tool_id + p.ntool);
    }
    if (p.nheattable > 0) ctx->heattable.assign(p.heattable, p.heattable + 6 * p.nheattable);
    if (p.nvardt > 0) ctx->vardt.assign(p.vardt, p.vardt + 3 * p.nvardt);
    p.tool_txyz = nullptr; p.tool_on = nullptr; p.tool_id = nullptr;
    p.heattable = nullptr; p.vardt = nullptr;
    int sx = 0, sy = 0, sz = 0;
    for (int q = 0; q < p.nzx; q++) sx += (int)p.ncvx[q];
    for (int q = 0; q < p.nzy; q++) sy += (int)p.ncvy[q];
    for (int q = 0; q < p.nzz; q++) sz += (int)p.ncvz[q];
    ctx->ni = sx + 2; ctx->nj = sy + 2; ctx->nk = sz + 2;
    if (sx < 1 || sy < 1 || sz < 1) return fail(ctx, AMCFD_E_ARG, "empty grid");
    ctx->nk_active = ctx->nk;
    if (p.powderbed) {
        if (p.numlayers < 1 || p.ncvzlayer < 1 || !(p.layerheight > 0.0))
            return fail(ctx, AMCFD_E_ARG, "*POWDER_BED_MODE needs layers, cells per layer and a height");
        ctx->nk_active = ctx->nk - (p.numlayers - 1) * p.ncvzlayer;
        if (ctx->nk_active < 3) return fail(ctx, AMCFD_E_ARG, "powder layers exceed the z grid");
    }
    if (ctx->nj > 65535) return fail(ctx, AMCFD_E_CAPACITY, "nj above 65535");
    // 32-bit chunk indices in the pointwise kernels (32-node chunks of x-lines)
    if ((long long)ctx->nk * ctx->nj * ((sx + 2 + 31) / 32) > (1ll << 30))
        return fail(ctx, AMCFD_E_CAPACITY, "grid above 2^35 nodes");
    ctx->nip = (ctx->ni + 31) / 32 * 32;
    double cpavg = (p.acpa * p.tsolid + p.acpb + p.acpl) * 0.5;
    ctx->hlcal = p.hsmelt + cpavg * (p.tliquid - p.tsolid);
    ctx->hlatnt = p.hlfriz - ctx->hlcal;
    ctx->delt = p.nvardt > 0 ? ctx->vardt[1] : p.delt;
    ctx->outtime = p.nvardt > 0 ? ctx->vardt[2] : p.outtime;
    ctx->scanvel = p.scanvel;
    build_grid(ctx, ctx->nk);
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&ctx->st_dev, sizeof(Status)));
    CK(cudaMemset(ctx->st_dev, 0, sizeof(Status)));
    CK(cudaMallocHost(&ctx->st_host, sizeof(Status)));
    memset(ctx->st_host, 0, sizeof(Status));
    {
        // initial volumetric-source parameters and the status block defaults
        Status s;
        memset(&s, 0, sizeof(s));
        s.avolpow = p.avolpow; s.apowseta = p.apowseta; s.heatthick = p.heatthick;
        s.heatrb = p.heatrb; s.avolfact = p.avolfact;
        s.delt = ctx->delt;
        s.mp_imax = INT_MAX;
        s.mp_imin = INT_MIN;
        CK(cudaMemcpy(ctx->st_dev, &s, sizeof(s), cudaMemcpyHostToDevice));
    }
    for (int q = 0; q < 16; q++) CK(cudaEventCreate(&ctx->ev[q]));
    int rc = ctx->precision == AMCFD_PREC_FP64 ? setup_instance<double>(ctx, ctx->I64)
                                               : setup_instance<float>(ctx, ctx->I32);
    if (rc) return rc;
    ctx->diff_a = ctx->precision == AMCFD_PREC_FP64 ? (const void *)ctx->I64.g.diff_cur
                                                    : (const void *)ctx->I32.g.diff_cur;
    int cf = opts ? opts->check_finite : 0;
    ctx->I64.check_finite = cf;
    ctx->I32.check_finite = cf;
    if (ctx->autotune) {
        rc = ctx->precision == AMCFD_PREC_FP64 ? autotune<double>(ctx, ctx->I64) : autotune<float>(ctx, ctx->I32);
        if (rc) return rc;
    }
    if (p.steady) laser_coords(ctx);  // main.cpp:105-106
    return 0;
}

void amcfd_destroy(amcfd_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (void *p : ctx->allocs) cudaFree(p);
    if (ctx->st_dev) cudaFree(ctx->st_dev);
    if (ctx->st_host) cudaFreeHost(ctx->st_host);
    if (ctx->mesh_pinned) cudaFreeHost(ctx->mesh_pinned);
    if (ctx->pack) cudaFree(ctx->pack);
    for (void *q : {(void *)ctx->ws_feat, (void *)ctx->ws_y, (void *)ctx->ws_target, ctx->ws_save[0],
                    ctx->ws_save[1], ctx->ws_save[2], ctx->ws_save[3]})
        if (q) cudaFree(q);
    drop_graphs(ctx);
    for (int q = 0; q < 16; q++)
        if (ctx->ev[q]) cudaEventDestroy(ctx->ev[q]);
    if (ctx->ev_packed) cudaEventDestroy(ctx->ev_packed);
    if (ctx->ev_copied) cudaEventDestroy(ctx->ev_copied);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *amcfd_last_error(const amcfd_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int amcfd_dims(const amcfd_ctx *ctx, int *ni, int *nj, int *nk)
{
    if (!ctx || !ni || !nj || !nk) return AMCFD_E_ARG;
    *ni = ctx->ni; *nj = ctx->nj; *nk = ctx->nk;
    return 0;
}

int amcfd_step(amcfd_ctx *ctx, amcfd_step_report *report)
{
    if (!ctx) return AMCFD_E_ARG;
    CK(cudaSetDevice(ctx->device));
    int rc = begin_step(ctx);
    if (rc) return rc;
    if (ctx->ws_mode) {
        rc = ctx->precision == AMCFD_PREC_FP64 ? ws_before<double>(ctx, ctx->I64)
                                               : ws_before<float>(ctx, ctx->I32);
        if (rc) return rc;
    }
    const double alenold = ctx->st_host->alen;
    rc = ctx->precision == AMCFD_PREC_FP64 ? outer_loop<double>(ctx, ctx->I64)
                                           : outer_loop<float>(ctx, ctx->I32);
    if (rc) return rc;
    // iterativeLoopSolve :719-721: a step that used every outer iteration with an
    // unchanged melt-pool length marks the length steady (for the moving mesh)
    if (!(ctx->niter > 0 && ctx->st_host->converged) && std::fabs(ctx->st_host->alen - alenold) < 1.0e-6)
        ctx->steadylength = 1;
    // main.cpp:151-152
    if (ctx->prm.solidification && ctx->st_host->tpeak > ctx->prm.tsolid) {
        if (ctx->precision == AMCFD_PREC_FP64)
            launch_solidification<double>(ctx->I64, ctx->scanvel);
        else
            launch_solidification<float>(ctx->I32, ctx->scanvel);
        ctx->launches += 1;
    }
    if (!ctx->prm.steady) {
        if (ctx->events) cudaEventRecord(ctx->ev[12], ctx->stream);
        if (ctx->precision == AMCFD_PREC_FP64)
            run_phase_impl<double>(ctx, ctx->I64, AMCFD_PHASE_UPDATE);
        else
            run_phase_impl<float>(ctx, ctx->I32, AMCFD_PHASE_UPDATE);
        ctx->launches += phase_launches(ctx, AMCFD_PHASE_UPDATE, false);
        if (ctx->events) {
            cudaEventRecord(ctx->ev[13], ctx->stream);
            cudaEventSynchronize(ctx->ev[13]);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev[12], ctx->ev[13]);
            ctx->last_ms[7] += ms;
        }
    }
    if (ctx->ws_mode) {
        if (ctx->precision == AMCFD_PREC_FP64)
            ws_after<double>(ctx, ctx->I64);
        else
            ws_after<float>(ctx, ctx->I32);
    }
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    fill_report(ctx, report);
    return 0;
}

}  // extern "C"

// ---- internal accessors for the output writer (output.cu) -------------------------------
extern "C" {
static int field_ptr(amcfd_ctx *ctx, const char *name, void **ptr);
}
namespace amcfd {
void ctx_report(amcfd_ctx *ctx, amcfd_step_report *r) { fill_report(ctx, r); }
// The kernel set a context launches: its precision, defect correction, order and
// graph use (contexts of one kind load the same kernels).
int ctx_kind(const amcfd_ctx *ctx)
{
    return ctx->precision + 2 * (ctx->dc ? 1 : 0) + 4 * ctx->order + 8 * (ctx->use_graphs ? 1 : 0);
}
double ctx_delt(const amcfd_ctx *ctx) { return ctx->delt; }
double ctx_outtime(const amcfd_ctx *ctx) { return ctx->outtime; }
const amcfd_params &ctx_params(const amcfd_ctx *ctx) { return ctx->prm; }
void ctx_grid(const amcfd_ctx *ctx, const std::vector<double> **x, const std::vector<double> **y,
              const std::vector<double> **z)
{
    *x = &ctx->x; *y = &ctx->y; *z = &ctx->z;
}
// boundary heat fluxes of the last outer iteration: north south top bottom west east
void ctx_fluxes(const amcfd_ctx *ctx, double f[6])
{
    const Status *s = ctx->st_host;
    f[0] = s->fluxnorth; f[1] = s->fluxsouth; f[2] = s->fluxtop;
    f[3] = s->fluxbottom; f[4] = s->fluxwest; f[5] = s->fluxeast;
}
// plane k of a field, FP64 [nj][ni]
int ctx_plane(amcfd_ctx *ctx, const char *name, int k, std::vector<double> &out)
{
    void *d;
    int rc;
    if ((rc = field_ptr(ctx, name, &d))) return rc;
    if (k < 0 || k >= ctx->nk) return fail(ctx, AMCFD_E_ARG, "plane index out of range");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t ni = ctx->ni, nj = ctx->nj, nip = ctx->nip;
    out.resize(ni * nj);
    if (ctx->precision == AMCFD_PREC_FP64) {
        CK(cudaMemcpy2D(out.data(), ni * sizeof(double), (const double *)d + (size_t)k * nj * nip,
                        nip * sizeof(double), ni * sizeof(double), nj, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(ni * nj);
        CK(cudaMemcpy2D(tmp.data(), ni * sizeof(float), (const float *)d + (size_t)k * nj * nip,
                        nip * sizeof(float), ni * sizeof(float), nj, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < tmp.size(); ++q) out[q] = tmp[q];
    }
    return 0;
}
const char *ctx_error(const amcfd_ctx *ctx) { return ctx->err.c_str(); }
}  // namespace amcfd

extern "C" {

int amcfd_ws_attach(amcfd_ctx *ctx, amcfd_net *net, int mode)
{
    if (!ctx || mode < AMCFD_WS_OFF || mode > AMCFD_WS_PREDICT_H || (mode != AMCFD_WS_OFF && !net))
        return AMCFD_E_ARG;
    if (mode != AMCFD_WS_OFF && ctx->prm.nheattable > 0)
        return fail(ctx, AMCFD_E_ARG, "warm start with a volumetric heat-source table is not supported");
    if (mode != AMCFD_WS_OFF && (ctx->prm.powderbed || ctx->prm.movingmesh))
        return fail(ctx, AMCFD_E_ARG, "warm start on a growing or moving grid is not supported");
    CK(cudaSetDevice(ctx->device));
    ctx->net = net;
    ctx->ws_mode = mode;
    if (mode == AMCFD_WS_OFF || ctx->ws_feat) return 0;
    const size_t n = (size_t)ctx->ni * ctx->nj * ctx->nk;
    const size_t n3 = (size_t)ctx->nk * ctx->nj * ctx->nip;
    const size_t e = ctx->precision == AMCFD_PREC_FP64 ? sizeof(double) : sizeof(float);
    CK(cudaMalloc(&ctx->ws_feat, n * 11 * sizeof(float)));
    CK(cudaMalloc(&ctx->ws_y, n * 2 * sizeof(float)));
    CK(cudaMalloc(&ctx->ws_target, n * 2 * sizeof(float)));
    CK(cudaMemset(ctx->ws_target, 0, n * 2 * sizeof(float)));
    for (auto &q : ctx->ws_save) CK(cudaMalloc(&q, n3 * e));
    return 0;
}

int amcfd_ws_buffers(amcfd_ctx *ctx, float **feat_dev, float **target_dev)
{
    if (!ctx || !ctx->ws_feat) return AMCFD_E_ARG;
    if (feat_dev) *feat_dev = ctx->ws_feat;
    if (target_dev) *target_dev = ctx->ws_target;
    return 0;
}

int amcfd_ws_stats(const amcfd_ctx *ctx, long long *accepted, long long *rejected)
{
    if (!ctx) return AMCFD_E_ARG;
    if (accepted) *accepted = ctx->ws_accepted;
    if (rejected) *rejected = ctx->ws_rejected;
    return 0;
}

int amcfd_run_steps(amcfd_ctx *ctx, int nsteps, amcfd_step_report *report, double *device_ms)
{
    if (!ctx || nsteps < 0) return AMCFD_E_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventRecord(ctx->ev[14], ctx->stream));
    for (int s = 0; s < nsteps; ++s) {
        int rc = amcfd_step(ctx, report);
        if (rc) return rc;
    }
    CK(cudaEventRecord(ctx->ev[15], ctx->stream));
    CK(cudaEventSynchronize(ctx->ev[15]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[14], ctx->ev[15]));
    if (device_ms) *device_ms = ms;
    return 0;
}

long long amcfd_kernel_launches(const amcfd_ctx *ctx) { return ctx ? ctx->launches : -1; }

int amcfd_free_surface(amcfd_ctx *ctx, amcfd_free_surface_report *out)
{
    if (!ctx) return AMCFD_E_ARG;
    const amcfd_params &p = ctx->prm;
    if (!p.freesurface) return fail(ctx, AMCFD_E_ARG, "the deck has no *TRACK_ENERGY_BASED_FREE_SURFACE");
    CK(cudaSetDevice(ctx->device));
    // the evaporated volume to match (FreeSurfaceManager.cpp:93-124; vdp and the
    // start delay are constants there)
    const double vdp = 2e-9, startdeltn = 0.0;
    double melttime = ctx->delt * (1.0 + startdeltn), vd;
    if (ctx->st_host->tpeak <= p.tsolid) {
        vd = 0.0;
        melttime = 0.0;
    } else {
        vd = vdp * (ctx->timet - melttime - startdeltn * ctx->delt);
        if (ctx->powerindicator < 1) vd = vdp * (p.lasertime - melttime);
    }
    FsIn a;
    a.lam1 = p.fs_lam1; a.lam2 = p.fs_lam2; a.gamma = p.fs_surftens; a.c1 = p.dens * p.grav;
    a.urf = p.fs_urfree; a.tol_e = p.fs_tolenergy; a.tol_b = p.fs_tolbisect; a.vd = vd;
    a.maxit_e = (int)p.fs_maxiterenergy; a.maxit_b = (int)p.fs_maxiterbisect;
    if (ctx->precision == AMCFD_PREC_FP64)
        launch_free_surface<double>(ctx->I64, a, ctx->fs_out);
    else
        launch_free_surface<float>(ctx->I32, a, ctx->fs_out);
    ctx->launches += 2;
    FsOut h;
    CK(cudaMemcpyAsync(&h, ctx->fs_out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    if (out) {
        out->lambda = h.xmid; out->residual = h.fmid; out->fi_min = h.fimin; out->fi_max = h.fimax;
        out->volume = vd; out->iterations = h.niter; out->bracketed = h.bracketed;
    }
    return 0;
}

int amcfd_run_phase(amcfd_ctx *ctx, int phase, amcfd_step_report *report)
{
    if (!ctx) return AMCFD_E_ARG;
    if (phase == 0) return 0;
    if (!phase_ok(phase)) return fail(ctx, AMCFD_E_ARG, "unknown phase");
    CK(cudaSetDevice(ctx->device));
    int rc;
    if (phase == AMCFD_PHASE_LASER) {
        if ((rc = begin_step(ctx))) return rc;
    } else {
        if (phase == AMCFD_PHASE_ENERGY_ASSEMBLE) {
            ctx->niter++;
            ctx->itertot++;
        }
        if (ctx->precision == AMCFD_PREC_FP64)
            run_phase_impl<double>(ctx, ctx->I64, phase);
        else
            run_phase_impl<float>(ctx, ctx->I32, phase);
    }
    if ((rc = read_status(ctx))) return rc;
    fill_report(ctx, report);
    return 0;
}

const char *amcfd_phase_name(int phase)
{
    static const char *names[] = {"none", "laser", "energy_assemble", "energy_solve", "h2t",
                                  "meltpool", "momentum", "converge", "update", "species"};
    return phase_ok(phase) ? names[phase] : "unknown";
}

static int field_ptr(amcfd_ctx *ctx, const char *name, void **ptr)
{
    struct E { const char *n; size_t off; };
#define F(x) {#x, offsetof(Fields<double>, x)}
    static const E tab[] = {
        {"temp", offsetof(Fields<double>, temp)}, {"uvel", offsetof(Fields<double>, uvel)},
        {"vvel", offsetof(Fields<double>, vvel)}, {"wvel", offsetof(Fields<double>, wvel)},
        {"pressure", offsetof(Fields<double>, pressure)}, F(pp),
        {"enthalpy", offsetof(Fields<double>, h)}, F(fracl), F(fraclnot), F(hnot),
        {"diff", offsetof(Fields<double>, diff_cur)}, {"rho", offsetof(Fields<double>, rho_cur)},
        {"vis", offsetof(Fields<double>, vis_cur)}, {"diff_next", offsetof(Fields<double>, diff_nxt)},
        {"rho_next", offsetof(Fields<double>, rho_nxt)}, {"vis_next", offsetof(Fields<double>, vis_nxt)},
        F(sourceinput), F(unot), F(vnot), F(wnot), F(an), F(as), F(ae), F(aw), F(at), F(ab),
        F(ap), F(su), F(dux), F(dvy), F(dwz),
        {"avgconcentration", offsetof(Fields<double>, conc)},
        {"avgconcentrationnot", offsetof(Fields<double>, concnot)},
        {"concentration", offsetof(Fields<double>, concn)},
        {"csfrac", offsetof(Fields<double>, csfrac)}, {"solfrac", offsetof(Fields<double>, solfrac)},
        {"mpPhase", offsetof(Fields<double>, mpphase)}, {"mpLiqPhase", offsetof(Fields<double>, mpliq)},
        {"grad", offsetof(Fields<double>, grad)}, {"rate", offsetof(Fields<double>, rate)},
        {"zr", offsetof(Fields<double>, fs_zr)}, {"tempr", offsetof(Fields<double>, fs_tempr)}};
#undef F
    // Fields<float> has the same member layout of pointers
    const char *base = ctx->precision == AMCFD_PREC_FP64 ? (const char *)&ctx->I64.g
                                                         : (const char *)&ctx->I32.g;
    for (const E &e : tab)
        if (!strcmp(e.n, name)) {
            *ptr = *(void *const *)(base + e.off);
            if (!*ptr)
                return fail(ctx, AMCFD_E_ARG, std::string("field ") + name + " is not solved by this deck");
            return 0;
        }
    return fail(ctx, AMCFD_E_ARG, std::string("unknown field ") + name);
}

// Field read-out through the FP64 staging buffer; with `async` the copy to the
// host runs on the copy stream and the call returns once it is queued.
static int get_field_impl(amcfd_ctx *ctx, const char *name, double *host_out, bool async)
{
    if (!ctx || !name || !host_out) return AMCFD_E_ARG;
    void *d = nullptr;
    int rc;
    // the output writer's cell-centred velocities (PrintManager.cpp:283-285)
    const int centre = !strcmp(name, "auvel") ? 0 : !strcmp(name, "avvel") ? 1 : !strcmp(name, "awvel") ? 2 : -1;
    if (centre < 0 && (rc = field_ptr(ctx, name, &d))) return rc;
    CK(cudaSetDevice(ctx->device));
    const long long rows = (long long)ctx->nj * ctx->nk;
    const size_t bytes = (size_t)rows * ctx->ni * sizeof(double);
    if (!ctx->pack) {
        CK(cudaMalloc(&ctx->pack, bytes));
        CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device));
    }
    // the staging may still be read by an asynchronous copy
    if (ctx->copy_pending) CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_copied, 0));
    // widen and pack on the device, then one contiguous copy (full speed into pinned memory)
    if (centre >= 0) {
        if (ctx->precision == AMCFD_PREC_FP64)
            launch_centre_velocity<double>(ctx->I64, centre, ctx->pack);
        else
            launch_centre_velocity<float>(ctx->I32, centre, ctx->pack);
    } else if (ctx->precision == AMCFD_PREC_FP64)
        launch_pack_field<double>((const double *)d, ctx->pack, ctx->ni, ctx->nip, rows, ctx->sm_count,
                                  ctx->stream);
    else
        launch_pack_field<float>((const float *)d, ctx->pack, ctx->ni, ctx->nip, rows, ctx->sm_count,
                                 ctx->stream);
    CK(cudaGetLastError());
    if (async) {
        if (!ctx->copy_stream) {
            CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->ev_packed, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->ev_copied, cudaEventDisableTiming));
        }
        CK(cudaEventRecord(ctx->ev_packed, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_packed, 0));
        CK(cudaMemcpyAsync(host_out, ctx->pack, bytes, cudaMemcpyDeviceToHost, ctx->copy_stream));
        CK(cudaEventRecord(ctx->ev_copied, ctx->copy_stream));
        ctx->copy_pending = true;
        return 0;
    }
    CK(cudaMemcpyAsync(host_out, ctx->pack, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->copy_pending = false;  // the stream waited for it
    return 0;
}

int amcfd_get_field(amcfd_ctx *ctx, const char *name, double *host_out)
{
    return get_field_impl(ctx, name, host_out, false);
}

int amcfd_get_field_async(amcfd_ctx *ctx, const char *name, double *host_out)
{
    return get_field_impl(ctx, name, host_out, true);
}

int amcfd_wait_reads(amcfd_ctx *ctx)
{
    if (!ctx) return AMCFD_E_ARG;
    if (!ctx->copy_pending) return 0;
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventSynchronize(ctx->ev_copied));
    CK(cudaGetLastError());
    ctx->copy_pending = false;
    return 0;
}

int amcfd_set_field(amcfd_ctx *ctx, const char *name, const double *host_in)
{
    if (!ctx || !name || !host_in) return AMCFD_E_ARG;
    void *d;
    int rc;
    if ((rc = field_ptr(ctx, name, &d))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t rows = (size_t)ctx->nj * ctx->nk;
    if (ctx->precision == AMCFD_PREC_FP64) {
        CK(cudaMemcpy2D(d, ctx->nip * sizeof(double), host_in, ctx->ni * sizeof(double),
                        ctx->ni * sizeof(double), rows, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> tmp(host_in, host_in + (size_t)ctx->ni * rows);
        CK(cudaMemcpy2D(d, ctx->nip * sizeof(float), tmp.data(), ctx->ni * sizeof(float),
                        ctx->ni * sizeof(float), rows, cudaMemcpyHostToDevice));
    }
    return 0;
}

int amcfd_get_grid(amcfd_ctx *ctx, const char *name, double *host_out)
{
    if (!ctx || !name || !host_out) return AMCFD_E_ARG;
    const std::vector<double> *v = !strcmp(name, "x") ? &ctx->x : !strcmp(name, "y") ? &ctx->y
                                 : !strcmp(name, "z") ? &ctx->z : !strcmp(name, "xu") ? &ctx->xu
                                 : !strcmp(name, "yv") ? &ctx->yv : !strcmp(name, "zw") ? &ctx->zw
                                 : nullptr;
    if (!v) return fail(ctx, AMCFD_E_ARG, std::string("unknown grid array ") + name);
    int n = name[0] == 'x' ? ctx->ni : name[0] == 'y' ? ctx->nj : ctx->nk;
    memcpy(host_out, v->data(), n * sizeof(double));
    return 0;
}

int amcfd_last_timing(const amcfd_ctx *ctx, double *ms, int n)
{
    if (!ctx || !ms) return AMCFD_E_ARG;
    for (int q = 0; q < n && q < 16; q++) ms[q] = ctx->last_ms[q];
    return 0;
}

// Per-phase device timing: enable (1) / disable (0) and clear the accumulators.
int amcfd_profile(amcfd_ctx *ctx, int enable)
{
    if (!ctx) return AMCFD_E_ARG;
    ctx->events = enable != 0;
    for (int q = 0; q < 16; q++) ctx->last_ms[q] = 0.0;
    return 0;
}

}  // extern "C"
