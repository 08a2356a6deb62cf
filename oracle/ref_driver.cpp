// Dump/timing driver around the reference AM-CFD managers (test infrastructure).
//
// It reproduces the reference time loop of src/main.cpp:52-162 (construction,
// PrintManager::initialization, updateLaser -> generateGrid (moving mesh) ->
// iterativeLoopSolve -> getSolidificationParameters -> updateSolutions per
// step) without the VTK/residual output, and writes a
// binary record of the state after each selected step so that the C
// restatement (oracle/amcfd_oracle.c) and the GPU path can be compared with
// the reference's own arithmetic.  Built by oracle/build_ref.sh against the
// reference objects; never part of the product.
//
// usage: amcfd_ref_dump <deck.k> [--out FILE] [--steps N] [--every K]
//                       [--time]          (timing only: no dumps, JSON on stdout)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <iostream>
#include <sstream>
#include <unistd.h>
#include <fcntl.h>

#include <Mesh.h>
#include <BoundCondManager.h>
#include <CFDSolverManager.h>
#include <DomainManager.h>
#include <FreeSurfaceManager.h>
#include <PrintManager.h>
#include <SolutionVariableManager.h>
#include <vtsBinWriter.h>
#include <omp.h>

static const char *kFields[] = {"temp", "uvel", "vvel", "wvel", "pressure", "enthalpy",
                                "fracl", "pp", "diff", "rho", "vis", "hnot", "fraclnot"};
static const int kNumFields = sizeof(kFields) / sizeof(kFields[0]);
// appended after kFields when the deck solves the species equation, then the
// powder-bed fields when it runs in powder-bed mode
static const char *kSpeciesFields[] = {"avgconcentration", "concentration"};
static const char *kPowderFields[] = {"csfrac", "solfrac", "mpPhase", "mpLiqPhase"};
static const char *kSolidFields[] = {"grad", "rate"};
static const char *kFreeSurfFields[] = {"zr", "tempr"};
static const char *kGeom[] = {"x", "y", "z", "xu", "yv", "dxpwinv", "dypsinv", "dzpbinv",
                              "fracx", "fracy"};
static const int kNumGeom = sizeof(kGeom) / sizeof(kGeom[0]);

static void put_i32(FILE *f, int v) { fwrite(&v, 4, 1, f); }
static void put_f64(FILE *f, double v) { fwrite(&v, 8, 1, f); }

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s deck.k [--out FILE] [--steps N] [--every K] [--time]\n", argv[0]);
        return 2;
    }
    std::string deck = argv[1];
    std::string out = "ref_dump.bin";
    long max_steps = -1;
    int every = 1;
    bool timing = false;
    for (int a = 2; a < argc; ++a) {
        if (!strcmp(argv[a], "--out") && a + 1 < argc) out = argv[++a];
        else if (!strcmp(argv[a], "--steps") && a + 1 < argc) max_steps = atol(argv[++a]);
        else if (!strcmp(argv[a], "--every") && a + 1 < argc) every = atoi(argv[++a]);
        else if (!strcmp(argv[a], "--time")) timing = true;
    }

    // The reference prints banners to stdout; keep stdout clean for --time JSON.
    int saved_stdout = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    fflush(stdout);
    dup2(devnull, 1);

    Mesh meshObj(deck);
    meshObj.getDomainInfo();
    meshObj.assignParameters();
    char *deckc = argv[1];
    meshObj.outputInputs(deckc);
    DomainManager *domainMgr = new DomainManager(&meshObj);
    SolutionVariableManager *solVarMgr = new SolutionVariableManager();
    BoundCondManager *bcMgr = new BoundCondManager(&meshObj, domainMgr, solVarMgr);
    CFDSolverManager *cfd = new CFDSolverManager(&meshObj, domainMgr, solVarMgr, bcMgr);
    FreeSurfaceManager *fs = new FreeSurfaceManager(&meshObj, domainMgr, solVarMgr, bcMgr);
    std::string dir = meshObj.directoryName_;
    std::string outFile = dir + "/" + meshObj.outFileName_ + "_0.vts";
    PrintManager *pm = new vtsBinWriter(&meshObj, domainMgr, solVarMgr, bcMgr, cfd, fs,
                                        outFile, dir, meshObj.outFileName_);
    pm->initialization();
    if (domainMgr->steady_) bcMgr->updateLaser();
    std::cout.flush();
    fflush(stdout);
    dup2(saved_stdout, 1);

    // every array holds all powder layers; PrintManager::initialization has made
    // only the first of them active (nk_)
    const int ni = domainMgr->ni_, nj = domainMgr->nj_,
              nk = domainMgr->nk_ + (meshObj.powderbed_ ? (domainMgr->numlayers_ - 1) * domainMgr->ncvzlayer_ : 0);
    const size_t n = (size_t)ni * nj * nk;
    const int nspecies = meshObj.species_ ? 2 : 0;
    const int npowder = meshObj.powderbed_ ? 4 : 0;
    const int nsolid = meshObj.solidificationparams_ ? 2 : 0;
    std::vector<const char *> names(kFields, kFields + kNumFields);
    names.insert(names.end(), kSpeciesFields, kSpeciesFields + nspecies);
    names.insert(names.end(), kPowderFields, kPowderFields + npowder);
    names.insert(names.end(), kSolidFields, kSolidFields + nsolid);
    if (meshObj.energyfreesurface_) names.insert(names.end(), kFreeSurfFields, kFreeSurfFields + 2);
    FILE *f = nullptr;
    if (!timing) {
        f = fopen(out.c_str(), "wb");
        if (!f) { perror("fopen"); return 1; }
        fwrite("AMCR", 1, 4, f);
        put_i32(f, 2);  // version 2: the field names follow the field count
        put_i32(f, ni); put_i32(f, nj); put_i32(f, nk);
        put_i32(f, (int)names.size());
        put_i32(f, kNumGeom);
        for (const char *nm : names) {
            put_i32(f, (int)strlen(nm));
            fwrite(nm, 1, strlen(nm), f);
        }
        // geometry: 1-D arrays x,y,z (+ face arrays), each written at its own length
        for (int g = 0; g < kNumGeom; ++g) {
            const char *nm = kGeom[g];
            int len = (nm[0] == 'x' || !strcmp(nm, "dxpwinv") || !strcmp(nm, "fracx")) ? ni
                    : (nm[0] == 'y' || !strcmp(nm, "dypsinv") || !strcmp(nm, "fracy")) ? nj : nk;
            put_i32(f, len);
            fwrite(solVarMgr->mapGeometryVars_[nm], 8, len, f);
        }
    }

    double simtime = meshObj.finaltime_;
    domainMgr->timet_ = 0.0;
    long step = 0;
    int vstate = 0;
    double total_s = 0.0;
    long total_iters = 0;
    std::vector<double> step_s;
    std::vector<int> step_it;
    while (domainMgr->timet_ < simtime) {
        if (max_steps >= 0 && step >= max_steps) break;
        if (meshObj.variableTimeStepFileName_.compare("FALSE")) {
            if ((domainMgr->timet_ > meshObj.variableTimeStepValues[vstate][0]) &&
                (vstate < (int)meshObj.variableTimeStepValues.size() - 1))
                vstate += 1;
            meshObj.delt_ = meshObj.variableTimeStepValues[vstate][1];
            meshObj.outtime_ = meshObj.variableTimeStepValues[vstate][2];
        }
        auto t0 = std::chrono::high_resolution_clock::now();
        domainMgr->timet_ += meshObj.delt_;
        if (!domainMgr->steady_) bcMgr->updateLaser();
        if (meshObj.movingmesh_) cfd->generateGrid();
        cfd->iterativeLoopSolve();
        if (meshObj.solidificationparams_) cfd->getSolidificationParameters();
        if (!domainMgr->steady_) cfd->updateSolutions();
        // the free surface, which main.cpp:174-176 runs at output times, after every step here
        // (it feeds nothing back into the solution)
        if (meshObj.energyfreesurface_) {
            fflush(stdout);
            dup2(devnull, 1);
            fs->execute();
            std::cout.flush();
            fflush(stdout);
            dup2(saved_stdout, 1);
        }
        auto t1 = std::chrono::high_resolution_clock::now();
        double dt_s = 1e-9 * std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
        total_s += dt_s;
        total_iters += cfd->niter_;
        step_s.push_back(dt_s);
        step_it.push_back(cfd->niter_);
        ++step;
        if (f && (step % every == 0)) {
            put_i32(f, (int)step);
            put_i32(f, cfd->niter_);
            put_i32(f, cfd->itertot_);
            double sc[] = {domainMgr->timet_, cfd->resorh_, cfd->resorm_, cfd->resoru_,
                           cfd->resorv_, cfd->resorw_, bcMgr->tpeak_, bcMgr->alen_,
                           bcMgr->depth_, bcMgr->width_, bcMgr->ratio_, bcMgr->heatinlaser_,
                           bcMgr->ahtoploss_, bcMgr->accul_, bcMgr->heatout_, bcMgr->heatvol_,
                           bcMgr->fluxwest_, bcMgr->fluxeast_, bcMgr->fluxtop_,
                           bcMgr->fluxbottom_, bcMgr->fluxnorth_, bcMgr->fluxsouth_,
                           bcMgr->beamposx_, bcMgr->beamposy_, domainMgr->scanvel_, cfd->resorc_};
            put_i32(f, (int)(sizeof(sc) / 8));
            fwrite(sc, 8, sizeof(sc) / 8, f);
            int ix[] = {bcMgr->istat_, bcMgr->iend_, bcMgr->jstat_, bcMgr->jend_, bcMgr->kstat_,
                        bcMgr->jstart_, bcMgr->powerindicator_, domainMgr->nk_, bcMgr->trackindx_,
                        (int)bcMgr->steadylength_};
            put_i32(f, (int)(sizeof(ix) / 4));
            fwrite(ix, 4, sizeof(ix) / 4, f);
            for (const char *nm : names) fwrite(solVarMgr->mapSolutionVars_[nm], 8, n, f);
            // the grid of this step (it moves with a moving mesh)
            for (const char *nm : {"x", "y"}) fwrite(solVarMgr->mapGeometryVars_[nm], 8, nm[0] == 'x' ? ni : nj, f);
        }
    }
    if (f) { put_i32(f, -1); fclose(f); }
    if (timing) {
        long ncell = (long)(ni - 2) * (nj - 2) * (nk - 2);
        printf("{\"steps\": %ld, \"outer_iters\": %ld, \"seconds\": %.6f, \"threads\": %d, "
               "\"interior_cells\": %ld, \"cell_iters_per_s\": %.6e, \"sim_ms_per_wall_s\": %.6e, "
               "\"step_seconds\": [",
               step, total_iters, total_s, omp_get_max_threads(), ncell,
               total_s > 0 ? (double)ncell * total_iters / total_s : 0.0,
               total_s > 0 ? 1e3 * domainMgr->timet_ / total_s : 0.0);
        for (size_t s = 0; s < step_s.size(); ++s) printf("%s%.6f", s ? ", " : "", step_s[s]);
        printf("], \"step_iters\": [");
        for (size_t s = 0; s < step_it.size(); ++s) printf("%s%d", s ? ", " : "", step_it[s]);
        printf("]}\n");
    }
    return 0;
}
