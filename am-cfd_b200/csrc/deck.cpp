// Keyword-deck parser: the input boundary of the solver.
//
// Reads the reference's LS-DYNA-style deck with the reference's rules
// (Mesh::getDomainInfo, src/sources/Mesh.cpp:39-435): lines starting with '$'
// are comments; a line equal to a known keyword selects it; any other line
// starting with '*' deselects; numeric rows are read left to right until the
// first token that is not a number (istream_iterator<double> semantics).  The
// mesh file (Mesh.cpp:475-550), toolpath (DomainManager.cpp:268-289),
// volumetric heat-source table (:295-312) and variable time-step table
// (Mesh.cpp:634-653) are read the same way, and the numeric rows are mapped to
// parameters as DomainManager::assignInputValues does (DomainManager.cpp:29-263).
// Blank lines are skipped (the reference would throw on them).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "amcfd.h"

namespace {

thread_local std::string g_deck_error;

std::vector<double> numbers(const std::string &line)
{
    std::vector<double> v;
    std::istringstream is(line);
    double d;
    while (is >> d) v.push_back(d);
    return v;
}

std::vector<std::string> words(const std::string &line)
{
    std::vector<std::string> v;
    std::istringstream is(line);
    std::string s;
    while (is >> s) v.push_back(s);
    return v;
}

bool read_lines(const std::string &path, std::vector<std::string> &out)
{
    std::ifstream f(path);
    if (!f.is_open()) return false;
    std::string line;
    while (std::getline(f, line)) out.push_back(line);
    return true;
}

}  // namespace

struct amcfd_deck {
    amcfd_params params;
    std::string path, keyword_id, directory = "Results", mesh_file, tool_file, heat_table_file,
                                  vardt_file, geom_out;
    std::vector<std::string> scalar_out, vector_out, cell_out;
    mutable std::string scalar_joined, vector_joined;
    std::vector<double> tool_txyz, heattable, vardt;
    std::vector<int> tool_on, tool_id;
    bool output_geometry = false, output_tec = false;
};

static int fail(int code, const std::string &msg)
{
    g_deck_error = msg;
    return code;
}

static int zones_from(const std::vector<double> &g, const char *axis, int *nz, double *len,
                      double *ncv, double *powr)
{
    if (g.empty()) return fail(AMCFD_E_PARSE, std::string("mesh file has no ") + axis + " grid");
    int n = (int)g[0];
    if (n < 1 || n > AMCFD_MAX_ZONES || (int)g.size() < 1 + 3 * n)
        return fail(AMCFD_E_PARSE, std::string("malformed ") + axis + " grid parameters");
    *nz = n;
    for (int q = 0; q < n; ++q) {
        len[q] = g[1 + q];
        ncv[q] = g[1 + n + q];
        powr[q] = g[1 + 2 * n + q];
    }
    return AMCFD_OK;
}

extern "C" int amcfd_deck_load(const char *path, amcfd_deck **out)
{
    if (!path || !out) return fail(AMCFD_E_ARG, "null argument");
    *out = nullptr;
    std::vector<std::string> lines;
    if (!read_lines(path, lines)) return fail(AMCFD_E_IO, std::string("cannot open deck ") + path);
    std::unique_ptr<amcfd_deck> d(new amcfd_deck());
    d->path = path;
    amcfd_params &p = d->params;
    memset(&p, 0, sizeof(p));
    p.alasrb = 1.0e-6;        // DomainManager.h:210
    p.scheme = AMCFD_SCHEME_UPWIND;  // Mesh.h:59
    p.navierstokes = 1;
    std::vector<double> proc, mat, relax, btemp, benergy, bmom, gauss, evap, volsrc, species,
        powder, freesurf;
    std::map<std::string, double> parameters;
    bool have_timestep = false, have_term = false, udtool = false, volsrc_on = false,
         voltable = false;
    int option = -1;
    for (const std::string &line : lines) {
        if (line.empty()) continue;
        if (line[0] == '$') continue;
        static const std::map<std::string, int> kw = {
            {"*SINGLE_TRACK_TOOL", 3}, {"*MATERIAL_PROPERTIES", 4}, {"*UNDER_RELAXATION", 5},
            {"*BOUNDARY_TEMPERATURES", 6}, {"*MESH_FILE", 7}, {"*KEYWORD_ID", 8},
            {"*PARAMETERS", 9}, {"*BOUNDARY_ENERGY_EQUATION", 10}, {"*CONTROL_TIMESTEP", 11},
            {"*CONTROL_TERMINATION", 12}, {"*GAUSS_LASER_PARAMETERS", 13},
            {"*BOUNDARY_MOMENTUM_EQUATION", 14}, {"*VECTOR_OUT", 15}, {"*SCALAR_OUT", 16},
            {"*CELL_OUT", 17}, {"*DIRECTORY", 18}, {"*OUTPUT_TEC", 19},
            {"*BOUNDARY_EVAPORATION", 20}, {"*SOLVE_SPECIES", 21}, {"*TOOLPATH_FILE", 22},
            {"*ACTIVATE_MOVING_MESH", 23}, {"*TRACK_ENERGY_BASED_FREE_SURFACE", 24},
            {"*SELECT_DISCRETIZATION", 25}, {"*POWDER_BED_MODE", 26},
            {"*VOLUMETRIC_HEAT_SOURCE", 27}, {"*OUTPUT_FINAL_GEOMETRY", 28},
            {"*OUTPUT_SECTION", 29}, {"*VOLUMETRIC_HEAT_SOURCE_TABLE", 30},
            {"*CONTROL_TIMESTEP_VARIABLE", 31}};
        if (line == "*FLUID_FLOW_OFF") { p.navierstokes = 0; continue; }
        if (line == "*CALCULATE_SOLIDIFICATION_PARAMETERS") { p.solidification = 1; continue; }
        auto it = kw.find(line);
        if (it != kw.end()) {
            option = it->second;
            switch (option) {
            case 19: d->output_tec = true; break;
            case 20: p.isevap = 1; break;
            case 21: p.species = 1; break;
            case 22: udtool = true; break;
            case 23: p.movingmesh = 1; break;
            case 24: p.freesurface = 1; break;
            case 26: p.powderbed = 1; break;
            case 27: volsrc_on = true; break;
            case 28: d->output_geometry = true; break;
            case 30: volsrc_on = true; voltable = true; break;
            default: break;
            }
            continue;
        }
        if (line[0] == '*') { option = -1; continue; }
        std::vector<double> v;
        std::vector<std::string> w;
        switch (option) {
        case 3: v = numbers(line); proc.insert(proc.end(), v.begin(), v.end()); break;
        case 4: v = numbers(line); mat.insert(mat.end(), v.begin(), v.end()); break;
        case 5: v = numbers(line); relax.insert(relax.end(), v.begin(), v.end()); break;
        case 6: v = numbers(line); btemp.insert(btemp.end(), v.begin(), v.end()); break;
        case 7: w = words(line); if (!w.empty()) d->mesh_file = w[0]; break;
        case 8: w = words(line); if (!w.empty()) d->keyword_id = w[0]; break;
        case 9:
            w = words(line);
            if (w.size() < 2) return fail(AMCFD_E_PARSE, "*PARAMETERS row needs a name and a value: " + line);
            parameters[w[0]] = strtod(w[1].c_str(), nullptr);
            break;
        case 10: v = numbers(line); benergy.insert(benergy.end(), v.begin(), v.end()); break;
        case 11:
            v = numbers(line);
            if (v.size() < 2) return fail(AMCFD_E_PARSE, "*CONTROL_TIMESTEP needs dt and output interval");
            // a later *CONTROL_TIMESTEP switches the variable table off (Mesh.cpp:288-290)
            p.delt = v[0]; p.outtime = v[1]; have_timestep = true;
            d->vardt.clear();
            break;
        case 12:
            v = numbers(line);
            if (v.size() < 3) return fail(AMCFD_E_PARSE, "*CONTROL_TERMINATION needs 3 values");
            // maxit is compared as a double with the integer count (CFDSolverManager.cpp:612)
            p.finaltime = v[0]; p.maxit = (int)ceil(v[1]); p.nonlintol = v[2]; have_term = true;
            break;
        case 13: v = numbers(line); gauss.insert(gauss.end(), v.begin(), v.end()); break;
        case 14: v = numbers(line); bmom.insert(bmom.end(), v.begin(), v.end()); break;
        case 15: w = words(line); if (!w.empty()) d->vector_out.push_back(w[0]); break;
        case 16: w = words(line); if (!w.empty()) d->scalar_out.push_back(w[0]); break;
        case 17: w = words(line); if (!w.empty()) d->cell_out.push_back(w[0]); break;
        case 18: w = words(line); if (!w.empty()) d->directory = w[0]; break;
        case 20: v = numbers(line); evap.insert(evap.end(), v.begin(), v.end()); break;
        case 21: v = numbers(line); species.insert(species.end(), v.begin(), v.end()); break;
        case 22: w = words(line); if (!w.empty()) d->tool_file = w[0]; break;
        case 24: v = numbers(line); freesurf.insert(freesurf.end(), v.begin(), v.end()); break;
        case 23:  // Mesh.cpp:364-370: 1-based zone numbers
            v = numbers(line);
            if (v.size() < 2) return fail(AMCFD_E_PARSE, "*ACTIVATE_MOVING_MESH needs x and y zone numbers");
            p.xmoveindex = (int)v[0] - 1; p.ymoveindex = (int)v[1] - 1;
            break;
        case 25:
            w = words(line);
            if (!w.empty() && w[0] == "power_law") p.scheme = AMCFD_SCHEME_POWER_LAW;
            else if (!w.empty() && w[0] == "exponential_law") p.scheme = AMCFD_SCHEME_EXPONENTIAL;
            break;
        case 26: v = numbers(line); powder.insert(powder.end(), v.begin(), v.end()); break;
        case 27: v = numbers(line); volsrc.insert(volsrc.end(), v.begin(), v.end()); break;
        case 28: w = words(line); if (!w.empty()) d->geom_out = w[0]; break;
        case 30: w = words(line); if (!w.empty()) d->heat_table_file = w[0]; break;
        case 31: {
            w = words(line);
            if (w.empty()) break;
            d->vardt_file = w[0];
            std::vector<std::string> rows;
            if (!read_lines(d->vardt_file, rows))
                return fail(AMCFD_E_IO, "cannot open variable time-step table " + d->vardt_file);
            d->vardt.clear();
            for (auto &r : rows) {
                auto n = numbers(r);
                if (n.empty()) continue;
                if (n.size() < 3) return fail(AMCFD_E_PARSE, "variable time-step row needs t dt outtime");
                d->vardt.insert(d->vardt.end(), {n[0], n[1], n[2]});
            }
            if (d->vardt.empty()) return fail(AMCFD_E_PARSE, "empty variable time-step table");
            p.delt = d->vardt[1];
            p.outtime = d->vardt[2];
            have_timestep = true;
            break;
        }
        default: break;
        }
    }
    // *PARAMETERS (Mesh.cpp:440-470)
    auto par = [&](const char *name, double *dst) {
        auto f = parameters.find(name);
        if (f != parameters.end()) *dst = f->second;
    };
    par("accelGravity", &p.grav);
    par("radBoltzmann", &p.sigm);
    par("ambientTemp", &p.tempamb);
    par("ambientPres", &p.pressamb);
    par("gasConstant", &p.gasconst);

    // mesh file (Mesh.cpp:475-550)
    if (d->mesh_file.empty())
        return fail(AMCFD_E_PARSE, "need to specify mesh file name with keyword \"*MESH_FILE\"");
    std::vector<std::string> mlines;
    if (!read_lines(d->mesh_file, mlines))
        return fail(AMCFD_E_IO, "specified mesh was not found: " + d->mesh_file);
    std::vector<double> gx, gy, gz;
    int mopt = -1;
    for (const std::string &line : mlines) {
        if (line.empty() || line[0] == '$') continue;
        if (line == "*X_GRID_PARAMETERS") { mopt = 1; continue; }
        if (line == "*Y_GRID_PARAMETERS") { mopt = 2; continue; }
        if (line == "*Z_GRID_PARAMETERS") { mopt = 3; continue; }
        if (line[0] == '*') { mopt = -1; continue; }
        auto v = numbers(line);
        std::vector<double> &dst = mopt == 1 ? gx : mopt == 2 ? gy : gz;
        if (mopt > 0) dst.insert(dst.end(), v.begin(), v.end());
    }
    int rc;
    if ((rc = zones_from(gx, "x", &p.nzx, p.xzone, p.ncvx, p.powrx))) return rc;
    if ((rc = zones_from(gy, "y", &p.nzy, p.yzone, p.ncvy, p.powry))) return rc;
    if ((rc = zones_from(gz, "z", &p.nzz, p.zzone, p.ncvz, p.powrz))) return rc;

    // DomainManager::assignInputValues (DomainManager.cpp:48-199)
    p.udtoolpath = udtool ? 1 : 0;
    if (!udtool) {
        if (proc.size() < 4) return fail(AMCFD_E_PARSE, "*SINGLE_TRACK_TOOL needs lasertime xstart ystart scanvel");
        p.lasertime = proc[0]; p.xstart = proc[1]; p.ystart = proc[2]; p.scanvel = proc[3];
    }
    if (mat.size() < 15) return fail(AMCFD_E_PARSE, "*MATERIAL_PROPERTIES needs 15 values");
    p.dens = mat[0]; p.denl = mat[1]; p.viscos = mat[2]; p.tsolid = mat[3]; p.tliquid = mat[4];
    p.hsmelt = mat[5]; p.hlfriz = mat[6]; p.acpa = mat[7]; p.acpb = mat[8]; p.acpl = mat[9];
    p.thconsa = mat[10]; p.thconsb = mat[11]; p.thconsc = mat[12]; p.thconla = mat[13];
    p.thconlb = mat[14];
    if (relax.size() < 5) return fail(AMCFD_E_PARSE, "*UNDER_RELAXATION needs 5 values");
    p.urfu = relax[0]; p.urfv = relax[1]; p.urfw = relax[2]; p.urfp = relax[3]; p.urfh = relax[4];
    if (benergy.size() < 5) return fail(AMCFD_E_PARSE, "*BOUNDARY_ENERGY_EQUATION needs 5 values");
    p.htci = benergy[0]; p.htcj = benergy[1]; p.htck1 = benergy[2]; p.htckn = benergy[3];
    p.emiss = benergy[4];
    if (btemp.size() < 5) return fail(AMCFD_E_PARSE, "*BOUNDARY_TEMPERATURES needs 5 values");
    p.tempwest = btemp[0]; p.tempeast = btemp[1]; p.tempnorth = btemp[2];
    p.tempbottom = btemp[3]; p.temppreheat = btemp[4];
    if (bmom.size() < 4) return fail(AMCFD_E_PARSE, "*BOUNDARY_MOMENTUM_EQUATION needs 4 values");
    p.beta = bmom[0]; p.dgdtp = bmom[1]; p.darcyKo = bmom[2]; p.a_oxygen = bmom[3];
    if (!gauss.empty()) {
        if (gauss.size() < 4) return fail(AMCFD_E_PARSE, "*GAUSS_LASER_PARAMETERS needs 4 values");
        p.alaspow = gauss[0]; p.alaseta = gauss[1]; p.alasrb = gauss[2]; p.alasfact = gauss[3];
    }
    if (p.isevap) {
        if (evap.size() < 4) return fail(AMCFD_E_PARSE, "*BOUNDARY_EVAPORATION needs 4 values");
        p.evaplatent = evap[0]; p.evaptemp = evap[1]; p.evapfact = evap[2]; p.molarmass = evap[3];
    }
    if (p.powderbed) {  // DomainManager.cpp:147-162: the build layers extend the last z-zone
        if (powder.size() < 8) return fail(AMCFD_E_PARSE, "*POWDER_BED_MODE needs 8 values");
        p.numlayers = (int)powder[0]; p.ncvzlayer = (int)powder[1]; p.layerheight = powder[2];
        p.powderden = powder[3]; p.powdercpa = powder[4]; p.powdercpb = powder[5];
        p.powderthcona = powder[6]; p.powderthconb = powder[7];
        if (p.nzz < 1) return fail(AMCFD_E_PARSE, "*POWDER_BED_MODE needs a z grid");
        p.zzone[p.nzz - 1] += p.numlayers * p.layerheight;
        p.ncvz[p.nzz - 1] += p.numlayers * p.ncvzlayer;
    }
    if (p.freesurface) {  // DomainManager.cpp:133-143
        if (freesurf.size() < 8) return fail(AMCFD_E_PARSE, "*TRACK_ENERGY_BASED_FREE_SURFACE needs 8 values");
        p.fs_lam1 = freesurf[0]; p.fs_lam2 = freesurf[1]; p.fs_surftens = freesurf[2];
        p.fs_maxiterenergy = freesurf[3]; p.fs_tolenergy = freesurf[4]; p.fs_maxiterbisect = freesurf[5];
        p.fs_tolbisect = freesurf[6]; p.fs_urfree = freesurf[7];
    }
    if (p.species) {  // DomainManager.cpp:123-129
        if (species.size() < 4) return fail(AMCFD_E_PARSE, "*SOLVE_SPECIES needs 4 values");
        p.initconc = species[0]; p.massdiff = species[1]; p.kp = species[2]; p.urfc = species[3];
    }
    if (volsrc_on && !voltable) {
        if (volsrc.size() < 5) return fail(AMCFD_E_PARSE, "*VOLUMETRIC_HEAT_SOURCE needs 5 values");
        p.avolpow = volsrc[0]; p.apowseta = volsrc[1]; p.heatthick = volsrc[2];
        p.heatrb = volsrc[3]; p.avolfact = volsrc[4];
    }
    if (voltable) {
        std::vector<std::string> rows;
        if (!read_lines(d->heat_table_file, rows))
            return fail(AMCFD_E_IO, "cannot open heat-source table " + d->heat_table_file);
        for (auto &r : rows) {
            auto n = numbers(r);
            if (n.empty()) continue;
            if (n.size() < 6) return fail(AMCFD_E_PARSE, "heat-source table row needs 6 values");
            d->heattable.insert(d->heattable.end(), n.begin(), n.begin() + 6);
        }
        if (d->heattable.empty()) return fail(AMCFD_E_PARSE, "empty heat-source table");
        p.avolpow = d->heattable[1]; p.apowseta = d->heattable[2]; p.heatthick = d->heattable[3];
        p.heatrb = d->heattable[4]; p.avolfact = d->heattable[5];
    }
    if (udtool) {
        std::vector<std::string> rows;
        if (!read_lines(d->tool_file, rows))
            return fail(AMCFD_E_IO, "cannot open toolpath " + d->tool_file);
        for (auto &r : rows) {
            auto n = numbers(r);
            if (n.empty()) continue;
            if (n.size() < 6) return fail(AMCFD_E_PARSE, "toolpath row needs t x y z on trackID");
            d->tool_txyz.insert(d->tool_txyz.end(), n.begin(), n.begin() + 4);
            d->tool_on.push_back((int)n[4]);
            d->tool_id.push_back((int)n[5]);
        }
        if (d->tool_on.size() < 2) return fail(AMCFD_E_PARSE, "toolpath needs at least 2 rows");
    }
    if (!have_timestep) return fail(AMCFD_E_PARSE, "missing *CONTROL_TIMESTEP");
    if (!have_term) return fail(AMCFD_E_PARSE, "missing *CONTROL_TERMINATION");
    p.steady = p.delt < 100.0 ? 0 : 1;
    *out = d.release();
    return AMCFD_OK;
}

extern "C" int amcfd_deck_params(const amcfd_deck *d, amcfd_params *out)
{
    if (!d || !out) return fail(AMCFD_E_ARG, "null argument");
    *out = d->params;
    out->ntool = (int)d->tool_on.size();
    out->tool_txyz = d->tool_txyz.empty() ? nullptr : d->tool_txyz.data();
    out->tool_on = d->tool_on.empty() ? nullptr : d->tool_on.data();
    out->tool_id = d->tool_id.empty() ? nullptr : d->tool_id.data();
    out->nheattable = (int)(d->heattable.size() / 6);
    out->heattable = d->heattable.empty() ? nullptr : d->heattable.data();
    out->nvardt = (int)(d->vardt.size() / 3);
    out->vardt = d->vardt.empty() ? nullptr : d->vardt.data();
    return AMCFD_OK;
}

extern "C" const char *amcfd_deck_error(void) { return g_deck_error.c_str(); }

extern "C" void amcfd_deck_free(amcfd_deck *d) { delete d; }

// Names the output writers need (keyword id, directory, requested fields).
extern "C" const char *amcfd_deck_string(const amcfd_deck *d, const char *what)
{
    if (!d || !what) return nullptr;
    if (!strcmp(what, "keyword_id")) return d->keyword_id.c_str();
    if (!strcmp(what, "directory")) return d->directory.c_str();
    if (!strcmp(what, "geometry_file")) return d->output_geometry ? d->geom_out.c_str() : nullptr;
    if (!strcmp(what, "mesh_file")) return d->mesh_file.c_str();
    // space-separated *SCALAR_OUT / *VECTOR_OUT names (Mesh.cpp:316-325)
    if (!strcmp(what, "scalar_out") || !strcmp(what, "vector_out")) {
        const auto &v = what[0] == 's' ? d->scalar_out : d->vector_out;
        std::string &j = what[0] == 's' ? d->scalar_joined : d->vector_joined;
        j.clear();
        for (size_t q = 0; q < v.size(); ++q) j += (q ? " " : "") + v[q];
        return j.c_str();
    }
    return nullptr;
}

extern "C" size_t amcfd_sizeof_params(void) { return sizeof(amcfd_params); }
extern "C" size_t amcfd_sizeof_report(void) { return sizeof(amcfd_step_report); }
