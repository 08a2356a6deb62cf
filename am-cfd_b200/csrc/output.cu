// Output path of the transient run (main.cpp:92-226, PrintManager.cpp,
// vtsBinWriter.cpp): what the reference writes, in its formats.
//
//  * <directory>/<keyword_id>_<n>.vts: VTK XML StructuredGrid, one line of XML
//    headers and the appended raw binary block: a 4-byte length then the
//    Float64 data of the points (x, y, z for k < nk-1) and of every requested
//    scalar field, uvel/vvel/wvel replaced by the cell-centred auvel/avvel/awvel
//    (vtsBinWriter.cpp:49-139, 144-338; PrintManager.cpp:314-376);
//  * <keyword_id>.pvd: the collection of all outputs so far (vtsBinWriter.cpp:359-412);
//  * <keyword_id>_Residuals.txt: per output the iteration counts, residuals,
//    peak temperature, top-plane velocity maxima, melt-pool size, boundary heat
//    fluxes and cooling rates (PrintManager.cpp:381-533);
//  * the *OUTPUT_FINAL_GEOMETRY file: laser power, speed and final melt-pool
//    size (PrintManager.cpp:659-676).
// Files are opened relative to `root` (the working directory when empty).
//
// Fields come off the device one at a time (widened and packed there, the
// centre velocities interpolated there) into two pinned buffers; a second host
// thread writes each buffer to the file while the next field is copied.
//
// Deviation: where no cell of the beam row is above the solidus (or liquidus),
// the reference's cooling rates read uninitialised values
// (PrintManager.cpp:403-456); here those inputs are zero.
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "amcfd.h"

namespace amcfd {
void ctx_report(amcfd_ctx *ctx, amcfd_step_report *r);
double ctx_delt(const amcfd_ctx *ctx);
double ctx_outtime(const amcfd_ctx *ctx);
const amcfd_params &ctx_params(const amcfd_ctx *ctx);
void ctx_grid(const amcfd_ctx *ctx, const std::vector<double> **x, const std::vector<double> **y,
              const std::vector<double> **z);
void ctx_fluxes(const amcfd_ctx *ctx, double f[6]);
int ctx_plane(amcfd_ctx *ctx, const char *name, int k, std::vector<double> &out);
const char *ctx_error(const amcfd_ctx *ctx);
}  // namespace amcfd

using namespace amcfd;

struct amcfd_writer {
    amcfd_ctx *ctx = nullptr;
    std::string err, root, directory, base, geometry;
    std::vector<std::string> scalars;  // as written (uvel -> auvel, ...)
    std::vector<std::string> fetch;    // field names to read back
    double outtrack = 0.0;
    int outct = 0;
    std::vector<double> stamps;
    std::vector<std::string> files;
    double *pinned[2] = {nullptr, nullptr};
    size_t npts_all = 0;  // ni * nj * nk
};

static std::string joinp(const std::string &root, const std::string &p)
{
    if (root.empty() || (!p.empty() && p[0] == '/')) return p;
    return root + "/" + p;
}

static int werr(amcfd_writer *w, int code, const std::string &m)
{
    w->err = m;
    return code;
}

// ---- .vts ---------------------------------------------------------------------------
static int write_vts(amcfd_writer *w, const std::string &path)
{
    amcfd_ctx *ctx = w->ctx;
    int ni, nj, nk;
    amcfd_dims(ctx, &ni, &nj, &nk);
    const std::vector<double> *x, *y, *z;
    ctx_grid(ctx, &x, &y, &z);
    const int gridz = nk;
    const long long npts = (long long)ni * nj * (gridz - 1);
    std::ofstream f(joinp(w->root, path), std::ios::out | std::ios::binary);
    if (!f) return werr(w, AMCFD_E_IO, "cannot open " + path);
    // headers: offsets count the 4-byte length in front of every array
    // (a 32-bit counter, as in vtsBinWriter.h:37)
    uint32_t off = 0;
    std::ostringstream h;
    h << "<?xml version=\"1.0\"?> ";
    h << "<VTKFile type=\"StructuredGrid\" version=\"2.1\" byte_order=\"LittleEndian\"> ";
    h << "<StructuredGrid WholeExtent=\"" << 0 << " " << ni - 1 << " " << 0 << " " << nj - 1 << " " << 0 << " "
      << gridz - 2 << "\"> ";
    h << "<Piece Extent=\"" << 0 << " " << ni - 1 << " " << 0 << " " << nj - 1 << " " << 0 << " " << gridz - 2
      << "\"> ";
    h << "<Points> ";
    h << "<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"appended\" offset = \"" << (int32_t)off
      << "\" /> ";
    off += (uint32_t)(sizeof(double) * npts * 3 + sizeof(int32_t));
    h << "</Points> ";
    h << "<PointData> ";
    for (const std::string &name : w->scalars) {
        h << "<DataArray type=\"Float64\" Name=\"" << name << "\" format=\"appended\" offset=\"" << (int32_t)off
          << "\" />  ";
        off += (uint32_t)(sizeof(double) * npts + sizeof(int32_t));
    }
    // powder bed: the layers not yet built are ghost points (vtsBinWriter.cpp:76-80, 235-258)
    const bool powder = ctx_params(ctx).powderbed != 0;
    if (powder) {
        h << "<DataArray type=\"UInt8\" Name=\"vtkGhostType\" format=\"appended\" offset=\"" << (int32_t)off
          << "\" />  ";
        off += (uint32_t)(sizeof(unsigned char) * npts + sizeof(int32_t));
    }
    h << "</PointData> ";
    h << "<CellData> ";
    h << "</CellData> ";
    h << "</Piece> ";
    h << "</StructuredGrid> ";
    h << "<AppendedData encoding=\"raw\">_";
    f << h.str();
    // points; with the free surface z is the deformed height zr (vtsBinWriter.cpp:164-171)
    {
        const bool deformed = ctx_params(ctx).freesurface != 0;
        if (deformed) {
            const int rc = amcfd_get_field(ctx, "zr", w->pinned[0]);
            if (rc) return werr(w, rc, ctx_error(ctx));
        }
        const double *zr = w->pinned[0];
        int32_t bytes = (int32_t)(sizeof(double) * npts * 3);
        f.write((const char *)&bytes, sizeof(bytes));
        std::vector<double> row((size_t)ni * 3);
        for (int k = 0; k < gridz - 1; k++)
            for (int j = 0; j < nj; j++) {
                for (int i = 0; i < ni; i++) {
                    row[3 * i] = (*x)[i];
                    row[3 * i + 1] = (*y)[j];
                    row[3 * i + 2] = deformed ? zr[((size_t)k * nj + j) * ni + i] : (*z)[k];
                }
                f.write((const char *)row.data(), row.size() * sizeof(double));
            }
    }
    // fields: the device read-out of field q overlaps the file write of field
    // q-1; writes stay in order (each task first waits for the one before)
    std::shared_future<void> task[2], last;
    for (size_t q = 0; q < w->fetch.size(); ++q) {
        double *buf = w->pinned[q & 1];
        if (task[q & 1].valid()) task[q & 1].wait();  // the write of field q-2 has left this buffer
        const int rc = amcfd_get_field(ctx, w->fetch[q].c_str(), buf);
        if (rc) {
            if (last.valid()) last.wait();
            return werr(w, rc, ctx_error(ctx));
        }
        std::shared_future<void> prev = last;
        last = std::async(std::launch::async, [&f, buf, npts, prev]() {
                   if (prev.valid()) prev.wait();
                   int32_t bytes = (int32_t)(sizeof(double) * npts);
                   f.write((const char *)&bytes, sizeof(bytes));
                   f.write((const char *)buf, (size_t)npts * sizeof(double));  // k < nk-1: a prefix of [k][j][i]
               }).share();
        task[q & 1] = last;
    }
    if (last.valid()) last.wait();
    if (powder) {  // visible (0) below the active top plane, hidden (2) from it up
        amcfd_step_report r;
        ctx_report(ctx, &r);
        const int nkm1 = r.nk_active - 1;
        int32_t bytes = (int32_t)npts;
        f.write((const char *)&bytes, sizeof(bytes));
        std::vector<unsigned char> plane((size_t)ni * nj);
        for (int k = 0; k < gridz - 1; k++) {
            std::fill(plane.begin(), plane.end(), (unsigned char)(k < nkm1 ? 0 : 2));
            f.write((const char *)plane.data(), plane.size());
        }
    }
    f << "\n";
    f << "</AppendedData> </VTKFile>";
    if (!f) return werr(w, AMCFD_E_IO, "write failed: " + path);
    return 0;
}

static int write_pvd(amcfd_writer *w)
{
    std::ofstream p(joinp(w->root, w->base + ".pvd"), std::ios::out | std::ios::binary);
    if (!p) return werr(w, AMCFD_E_IO, "cannot open " + w->base + ".pvd");
    p << "<?xml version=\"1.0\"?>\n";
    p << "<VTKFile type=\"Collection\" version=\"2.1\" byte_order=\"LittleEndian\">\n";
    p << "  <Collection>\n";
    for (size_t q = 0; q < w->stamps.size(); ++q)
        p << "   <DataSet timestep=\"" << w->stamps[q] << "\" group=\"\" part=\"0\" file=\"" << w->files[q]
          << "\"/>\n";
    p << "  </Collection>\n";
    p << "</VTKFile>\n";
    return p ? 0 : werr(w, AMCFD_E_IO, "write failed: pvd");
}

// ---- _Residuals.txt -------------------------------------------------------------------
static int write_residuals(amcfd_writer *w)
{
    amcfd_ctx *ctx = w->ctx;
    amcfd_step_report r;
    ctx_report(ctx, &r);
    const amcfd_params &prm = ctx_params(ctx);
    int ni, nj, nk;
    amcfd_dims(ctx, &ni, &nj, &nk);
    const int nim1 = ni - 1, nkm2 = r.nk_active - 2;  // top interior plane of the active domain
    const std::vector<double> *x, *y, *z;
    ctx_grid(ctx, &x, &y, &z);
    const double tsolid = prm.tsolid, tliquid = prm.tliquid, scanvel = r.scanvel;
    double umax = 0.0, vmax = 0.0, wmax = 0.0;
    std::vector<double> T, U, V, W;
    int rc;
    if ((rc = ctx_plane(ctx, "temp", nkm2, T))) return werr(w, rc, ctx_error(ctx));
    if (r.tpeak > tsolid) {
        if ((rc = ctx_plane(ctx, "uvel", nkm2, U)) || (rc = ctx_plane(ctx, "vvel", nkm2, V)) ||
            (rc = ctx_plane(ctx, "wvel", nkm2, W)))
            return werr(w, rc, ctx_error(ctx));
        for (int j = r.jstat; j <= r.jend; ++j)
            for (int i = r.istat + 1; i <= r.iend - 1; ++i) {
                const size_t c = (size_t)j * ni + i;
                umax = std::max(umax, std::fabs(U[c]));
                vmax = std::max(vmax, std::fabs(V[c]));
                wmax = std::max(wmax, std::fabs(W[c]));
            }
    }
    // cooling rates along the beam row of the top interior plane
    const double *row = T.data() + (size_t)r.jstart * ni;
    double xso = 0, tso = 0, xsob = 0, tsob = 0, xliq = 0, tliq = 0;
    for (int i = 1; i < nim1; ++i)
        if (row[i] > tsolid - 290) { tsob = row[i - 1]; xsob = (*x)[i - 1]; break; }
    for (int i = 1; i < nim1; ++i)
        if (row[i] > tsolid) { tso = row[i - 1]; xso = (*x)[i - 1]; break; }
    for (int i = 1; i < nim1; ++i)
        if (row[i] > tliquid) { tliq = row[i]; xliq = (*x)[i]; break; }
    const double crs = (tso - tsob) / (xso - xsob) * scanvel;
    const double crl = (tliq - tso) / (xliq - xso) * scanvel;
    double fl[6];
    ctx_fluxes(ctx, fl);
    const double resorc = r.resorc;
    std::ofstream o(joinp(w->root, w->base + "_Residuals.txt"), std::ios::out | std::ios::app);
    if (!o) return werr(w, AMCFD_E_IO, "cannot open residual file");
    const char *bar = "====================================================================================================\n";
    o << bar;
    if (prm.steady) {
        o << "  iter    res_enth   res_mass   res_u      res_v      res_w      res_concen\n";
        o << std::setprecision(2) << std::fixed << std::setw(8) << r.niter << std::scientific << std::setw(15)
          << r.resorh << std::setw(11) << r.resorm << std::setw(11) << r.resoru << std::setw(11) << r.resorv
          << std::setw(11) << r.resorw << std::setw(11) << resorc << " \n";
    } else {
        o << "  time        iter  tot_iter    res_enth   res_mass   res_u      res_v      res_w      res_concen\n";
        o << std::setprecision(2) << std::scientific << std::setw(10) << r.timet << std::fixed << std::setw(6)
          << r.niter << std::setw(9) << r.itertot << std::scientific << std::setw(15) << r.resorh
          << std::setw(11) << r.resorm << std::setw(11) << r.resoru << std::setw(11) << r.resorv
          << std::setw(11) << r.resorw << std::setw(11) << resorc << " \n";
    }
    o << "  Tmax       umax       vmax       wmax        length      depth       width\n";
    o << std::setprecision(2) << std::fixed << std::setw(10) << r.tpeak << std::scientific << std::setw(11) << umax
      << std::setw(11) << vmax << std::setw(11) << wmax << std::setw(12) << r.alen << std::setw(12) << r.depth
      << std::setw(12) << r.width << "\n";
    o << "  north    south     top   toploss   bottom    west      east    hout    accu    hin      ratio\n";
    o << std::setprecision(1) << std::fixed << std::setw(6) << fl[0] << std::setw(9) << fl[1] << std::setw(9)
      << fl[2] << std::setw(9) << r.ahtoploss << std::setw(9) << fl[3] << std::setw(9) << fl[4] << std::setw(9)
      << fl[5] << std::setw(9) << r.heatout << std::setw(8) << r.accul << std::setw(8) << r.heatinlaser
      << std::setw(8) << r.ratio << (prm.steady ? "\n" : "\n\n");
    if (!prm.steady)
        o << std::setprecision(4) << std::scientific
          << "  Cooling rate from solidus to 290K below solidus:     " << std::setw(14) << crs << "\n"
          << "  Cooling rate from liquidus to solidus:               " << std::setw(14) << crl << "\n";
    o << bar;
    return o ? 0 : werr(w, AMCFD_E_IO, "write failed: residuals");
}

// FreeSurfaceManager::execute and its monitor line (FreeSurfaceManager.cpp:74-209)
static int free_surface(amcfd_writer *w)
{
    amcfd_free_surface_report f;
    const int rc = amcfd_free_surface(w->ctx, &f);
    if (rc) return werr(w, rc, ctx_error(w->ctx));
    amcfd_step_report r;
    ctx_report(w->ctx, &r);
    std::ofstream o(joinp(w->root, w->base + "_FreeSurfaceMonitor.txt"), std::ios::out | std::ios::app);
    if (!o) return werr(w, AMCFD_E_IO, "cannot open free-surface monitor file");
    const char *bar = "====================================================================================================\n";
    o << bar;
    o << "  time         lambda        res_bisect    min_fi         max_fi        droplet_volume   iter_bisect\n";
    o << std::setprecision(4) << std::scientific << std::setw(12) << r.timet << std::setw(14) << f.lambda
      << std::setw(14) << f.residual << std::setw(14) << f.fi_min << std::setw(14) << f.fi_max << std::setw(14)
      << f.volume << std::setw(9) << f.iterations << "\n";
    o << bar;
    return o ? 0 : werr(w, AMCFD_E_IO, "write failed: free-surface monitor");
}

static int write_output(amcfd_writer *w, bool residuals = true)
{
    if (residuals) w->outct++;
    const std::string file = w->directory + "/" + w->base + "_" + std::to_string(w->outct) + ".vts";
    int rc;
    // main.cpp:174-176, 210-212: the free surface is updated before each output but the first
    if (residuals && ctx_params(w->ctx).freesurface && (rc = free_surface(w))) return rc;
    if (residuals && (rc = write_residuals(w))) return rc;
    if ((rc = write_vts(w, file))) return rc;
    amcfd_step_report r;
    ctx_report(w->ctx, &r);
    w->stamps.push_back(r.timet);
    w->files.push_back(file);
    return write_pvd(w);
}

extern "C" {

int amcfd_writer_create(amcfd_ctx *ctx, const amcfd_deck *deck, const char *root, amcfd_writer **out)
{
    if (!ctx || !deck || !out) return AMCFD_E_ARG;
    amcfd_writer *w = new amcfd_writer();
    *out = w;
    w->ctx = ctx;
    w->root = root ? root : "";
    w->directory = amcfd_deck_string(deck, "directory");
    w->base = amcfd_deck_string(deck, "keyword_id");
    const char *g = amcfd_deck_string(deck, "geometry_file");
    w->geometry = g ? g : "";
    std::istringstream s(amcfd_deck_string(deck, "scalar_out"));
    std::string name;
    // the requested fields the registry knows (PrintManager::scanOutputData);
    // vector outputs name no registered 3-component array and are skipped, as there
    static const char *known[] = {"pp", "vis", "rho", "uvel", "vvel", "wvel", "temp", "diff", "hnot",
                                  "fracl", "fraclnot", "pressure", "enthalpy", "sourceinput", "auvel",
                                  "avvel", "awvel"};
    // with *SOLVE_SPECIES the registry also holds the two concentrations
    // (CFDSolverManager.cpp:547-551)
    const bool species = ctx_params(ctx).species != 0, powder = ctx_params(ctx).powderbed != 0;
    while (s >> name) {
        bool ok = species && (name == "avgconcentration" || name == "concentration");
        // with *POWDER_BED_MODE: CFDSolverManager.cpp:554-560
        ok |= powder && (name == "csfrac" || name == "solfrac" || name == "mpPhase" || name == "mpLiqPhase");
        // with *CALCULATE_SOLIDIFICATION_PARAMETERS: :542-546
        ok |= ctx_params(ctx).solidification && (name == "grad" || name == "rate");
        ok |= ctx_params(ctx).freesurface && (name == "zr" || name == "tempr");  // FreeSurfaceManager.cpp:67-68
        for (const char *k : known) ok |= name == k;
        if (!ok) continue;
        const std::string shown = name == "uvel" ? "auvel" : name == "vvel" ? "avvel" : name == "wvel" ? "awvel" : name;
        w->scalars.push_back(shown);
        w->fetch.push_back(shown);
    }
    mkdir(joinp(w->root, w->directory).c_str(), 0777);
    int ni, nj, nk;
    amcfd_dims(ctx, &ni, &nj, &nk);
    w->npts_all = (size_t)ni * nj * nk;
    for (auto &p : w->pinned)
        if (cudaMallocHost(&p, w->npts_all * sizeof(double)) != cudaSuccess)
            return werr(w, AMCFD_E_NOMEM, "pinned output buffer");
    // the initial-state output <keyword_id>_0.vts (main.cpp:118-119)
    return write_output(w, false);
}

// After each amcfd_step: counts simulated time and writes an output when the
// deck's output interval has passed (main.cpp:137, 165-182).  Returns 1 when
// it wrote, 0 when not, a negative AMCFD_E_* code on failure.
int amcfd_writer_step(amcfd_writer *w)
{
    if (!w) return AMCFD_E_ARG;
    if (ctx_params(w->ctx).steady) return 0;
    w->outtrack += ctx_delt(w->ctx);
    if (w->outtrack < ctx_outtime(w->ctx)) return 0;
    const int rc = write_output(w);
    w->outtrack = 0.0;
    return rc ? rc : 1;
}

// At the end of the run: the final output and, if the deck asks for it, the
// final melt-pool geometry (main.cpp:218-226, PrintManager.cpp:659-676).
int amcfd_writer_finish(amcfd_writer *w)
{
    if (!w) return AMCFD_E_ARG;
    int rc;
    if ((rc = write_output(w))) return rc;
    if (w->geometry.empty()) return 0;
    amcfd_step_report r;
    ctx_report(w->ctx, &r);
    std::ofstream g(joinp(w->root, w->geometry), std::ios::out | std::ios::app);
    if (!g) return werr(w, AMCFD_E_IO, "cannot open " + w->geometry);
    g << "\n This is the final melt pool geometry for the given process parameters\n";
    g << "===================================================================\n";
    g << "  Laser Power    Laser Speed      length      depth      width\n";
    g << std::setprecision(2) << std::fixed << std::setw(8) << ctx_params(w->ctx).alaspow << std::setw(13)
      << r.scanvel << std::scientific << std::setw(21) << r.alen << std::setw(12) << r.depth << std::setw(11)
      << r.width << "\n";
    g << "===================================================================\n";
    return g ? 0 : werr(w, AMCFD_E_IO, "write failed: " + w->geometry);
}

const char *amcfd_writer_last_error(const amcfd_writer *w) { return w ? w->err.c_str() : "null writer"; }

void amcfd_writer_destroy(amcfd_writer *w)
{
    if (!w) return;
    for (auto p : w->pinned)
        if (p) cudaFreeHost(p);
    delete w;
}

}  // extern "C"
