/*
 * amcfd_oracle.c -- CPU restatement of the AM-CFD melt-pool hot path.
 *
 * TEST INFRASTRUCTURE.  This file is the checker the GPU path is compared
 * with: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * load it (as liboracle.so).  It is never linked into the product.
 *
 * It restates, in plain sequential FP64 C, the reference functions named in
 * each comment (paths relative to the reference project), in the reference's
 * evaluation order, so that it reproduces a single-threaded run of the
 * reference bit for bit.  std::max/std::min are restated as MAXD/MIND with
 * the same NaN behaviour ((a<b)?b:a and (b<a)?b:a).  It is pinned against the
 * compiled reference (oracle/_ref/amcfd_ref_dump, built by
 * oracle/build_ref.sh) by tests/test_oracle.py (live runs of the reference)
 * and the committed golden records under tests/golden/.
 *
 * Restated beyond the SIMPLE loop itself: the species equation, powder-bed
 * properties and layer activation, the moving mesh with its remap,
 * solidification G/R and the energy-balance free surface (orc_species,
 * orc_move_mesh, orc_free_surface ...).  Not restated: the output writers
 * (their files are compared with the compiled reference's directly).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <float.h>

#include "../include/amcfd.h"

#define MAXD(a, b) (((a) < (b)) ? (b) : (a))
#define MIND(a, b) (((b) < (a)) ? (b) : (a))
#define SMALL 1.0e-6  /* CFDSolverManager.h:143 */
#define LARGE 1.0e20  /* CFDSolverManager.h:144 */

typedef struct orc {
    amcfd_params p;
    double *tool;
    int *tool_on, *tool_id;
    int ni, nj, nk, nim1, njm1, nkm1, nim2, njm2, nkm2;
    int nk_alloc;     /* planes of every 3-D array; nk is DomainManager::nk_ (powder: active) */
    int layer_overflow; /* a powder layer was requested beyond the generated grid */
    double hlcal, hlatnt, enthbottom, scanvel, timet;
    /* 1-D grid */
    double *x, *y, *z, *xu, *yv, *zw, *dxpwinv, *dypsinv, *dzpbinv, *fracx, *fracy, *fracz;
    /* 2-D face areas */
    double *areaij, *areauij, *areavij, *areaik, *areawik, *areauik, *areajk, *areavjk, *areawjk;
    /* 3-D */
    double *volume, *volume_u, *volume_v, *volume_w;
    double *vis, *diff, *uvel, *vvel, *wvel, *enthalpy, *temp, *pp, *hnot, *fracl, *fraclnot;
    double *sourceinput, *rho, *unot, *vnot, *wnot, *pressure;
    double *ap, *an, *as, *ae, *aw, *at, *ab, *apnot, *dux, *dvy, *dwz, *su, *sp;
    /* species: avgconcentration, avgconcentrationnot, concentration */
    double *conc, *concnot, *concn;
    /* powder bed: csfrac, solfrac, mpPhase, mpLiqPhase */
    double *csfrac, *solfrac, *mpphase, *mpliq;
    /* solidification parameters: G and R */
    double *grad, *rate;
    /* free surface: deflection fi and its iterate zzm ([j][i]), deformed heights zr and
     * the temperatures on them */
    double *fi, *zzm, *zr, *tempr;
    double resoru, resorv, resorw, resorm, resorh, resorc, refmom;
    int itertot, niter;
    /* BoundCondManager state */
    double *heatin;
    double ahtoploss, heatout, accul, heatvol, ratio, tpeak;
    double fluxwest, fluxeast, fluxtop, fluxbottom, fluxnorth, fluxsouth;
    double alen, depth, width;
    int steadylength;
    int istat, jstat, kstat, iend, jend, istatp1, iendm1;
    int jstart, istart, imin, imax, jmin, jmax, kmin, kmax;
    double heatinlaser, beamposx, beamposy, beamposz, oldbeamposx, oldbeamposy, oldbeamposz;
    double peakhin;
    int powerindicator, init, trackindx;
    int last_box_cells;
    int heat_iter, vardt_state;
    double *heattable, *vardt;
} orc;

#define ID(i, j, k) ((size_t)(k) * (size_t)nj * (size_t)ni + (size_t)(j) * (size_t)ni + (size_t)(i))

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ---- scheme functions: CFDSolverManager.cpp:3071-3101 ---------------------------- */
static double scheme_fn(int scheme, double pe)
{
    if (scheme == AMCFD_SCHEME_POWER_LAW) {
        double base = 1.0 - 0.1 * pe;
        double out = base;
        for (int q = 1; q < 5; q++) out *= base;
        return MAXD(0.0, out);
    }
    if (scheme == AMCFD_SCHEME_EXPONENTIAL) return pe / (exp(pe) - 1.0);
    return 1.0;
}

/* ---- grid: CFDSolverManager.cpp:126-286 ------------------------------------------ */
static void zone_faces(int nz, const double *len, const double *ncv, const double *powr,
                       double *face)
{
    face[0] = 0.0;
    face[1] = 0.0;
    int ist = 2;
    double statloc = 0.0;
    for (int zi = 0; zi < nz; zi++) {
        for (int q = 0; q < ncv[zi]; q++) {
            double term;
            if (powr[zi] >= 0.0)
                term = pow((double)(q + 1) / ncv[zi], powr[zi]);
            else
                term = 1.0 - pow(1.0 - (double)(q + 1) / ncv[zi], -powr[zi]);
            face[q + ist] = statloc + len[zi] * term;
        }
        ist += (int)ncv[zi];
        statloc += len[zi];
    }
}

static void centres(int n, const double *face, double *c)
{
    for (int q = 0; q < n - 1; q++) c[q] = (face[q + 1] + face[q]) * 0.5;
    c[n - 1] = face[n - 1];
}

static void generate_grid(orc *o)
{
    const int ni = o->ni, nj = o->nj, nk = o->nk;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1;
    zone_faces(o->p.nzx, o->p.xzone, o->p.ncvx, o->p.powrx, o->xu);
    centres(ni, o->xu, o->x);
    zone_faces(o->p.nzy, o->p.yzone, o->p.ncvy, o->p.powry, o->yv);
    centres(nj, o->yv, o->y);
    zone_faces(o->p.nzz, o->p.zzone, o->p.ncvz, o->p.powrz, o->zw);
    centres(nk, o->zw, o->z);
    for (int i = 1; i < ni; i++) o->dxpwinv[i] = 1.0 / (o->x[i] - o->x[i - 1]);
    for (int j = 1; j < nj; j++) o->dypsinv[j] = 1.0 / (o->y[j] - o->y[j - 1]);
    for (int k = 1; k < nk; k++) o->dzpbinv[k] = 1.0 / (o->z[k] - o->z[k - 1]);
    for (int i = 0; i < nim1; i++) o->fracx[i] = (o->x[i + 1] - o->xu[i + 1]) / (o->x[i + 1] - o->x[i]);
    for (int j = 0; j < njm1; j++) o->fracy[j] = (o->y[j + 1] - o->yv[j + 1]) / (o->y[j + 1] - o->y[j]);
    for (int k = 0; k < nkm1; k++) o->fracz[k] = (o->z[k + 1] - o->zw[k + 1]) / (o->z[k + 1] - o->z[k]);
    const double *x = o->x, *y = o->y, *z = o->z, *xu = o->xu, *yv = o->yv, *zw = o->zw;
    for (int k = 1; k < nkm1; k++)
        for (int j = 1; j < njm1; j++)
            for (int i = 1; i < nim1; i++) {
                size_t c = ID(i, j, k);
                o->volume[c] = (xu[i + 1] - xu[i]) * (yv[j + 1] - yv[j]) * (zw[k + 1] - zw[k]);
                o->volume_u[c] = (x[i] - x[i - 1]) * (yv[j + 1] - yv[j]) * (zw[k + 1] - zw[k]);
                o->volume_v[c] = (xu[i + 1] - xu[i]) * (y[j] - y[j - 1]) * (zw[k + 1] - zw[k]);
                o->volume_w[c] = (xu[i + 1] - xu[i]) * (yv[j + 1] - yv[j]) * (z[k] - z[k - 1]);
            }
    for (int j = 1; j < njm1; j++)
        for (int i = 1; i < nim1; i++) {
            o->areaij[j * ni + i] = (xu[i + 1] - xu[i]) * (yv[j + 1] - yv[j]);
            o->areauij[j * ni + i] = (x[i] - x[i - 1]) * (yv[j + 1] - yv[j]);
            o->areavij[j * ni + i] = (xu[i + 1] - xu[i]) * (y[j] - y[j - 1]);
        }
    for (int k = 1; k < nkm1; k++)
        for (int i = 1; i < nim1; i++) {
            o->areaik[k * ni + i] = (xu[i + 1] - xu[i]) * (zw[k + 1] - zw[k]);
            o->areawik[k * ni + i] = (xu[i + 1] - xu[i]) * (z[k] - z[k - 1]);
            o->areauik[k * ni + i] = (x[i] - x[i - 1]) * (zw[k + 1] - zw[k]);
        }
    for (int k = 1; k < nkm1; k++)
        for (int j = 1; j < njm1; j++) {
            o->areajk[k * nj + j] = (yv[j + 1] - yv[j]) * (zw[k + 1] - zw[k]);
            o->areavjk[k * nj + j] = (y[j] - y[j - 1]) * (zw[k + 1] - zw[k]);
            o->areawjk[k * nj + j] = (yv[j + 1] - yv[j]) * (z[k] - z[k - 1]);
        }
}

/* ---- initializeSolver: CFDSolverManager.cpp:402-590 ------------------------------- */
static void initialize_solver(orc *o)
{
    const amcfd_params *p = &o->p;
    const int ni = o->ni, nj = o->nj, nk = o->nk, nim1 = o->nim1, njm1 = o->njm1;
    double hpre = 0.5 * p->acpa * p->temppreheat * p->temppreheat + p->acpb * p->temppreheat;
    double hwest = 0.5 * p->acpa * p->tempwest * p->tempwest + p->acpb * p->tempwest;
    double heast = 0.5 * p->acpa * p->tempeast * p->tempeast + p->acpb * p->tempeast;
    double hnorth = 0.5 * p->acpa * p->tempnorth * p->tempnorth + p->acpb * p->tempnorth;
    double hbottom = 0.5 * p->acpa * p->tempbottom * p->tempbottom + p->acpb * p->tempbottom;
    double diff0 = (p->thconsa * p->temppreheat * p->temppreheat + p->thconsb * p->temppreheat +
                    p->thconsc) / (p->acpa * p->temppreheat + p->acpb);
    size_t n = (size_t)ni * nj * nk;
    for (size_t c = 0; c < n; c++) {
        o->vis[c] = p->viscos;
        o->rho[c] = p->dens;
        o->diff[c] = diff0;
        o->enthalpy[c] = hpre;
        o->hnot[c] = hpre;
        o->temp[c] = p->temppreheat;
        if (p->species) {  /* CFDSolverManager.cpp:474-479 */
            o->conc[c] = p->initconc;
            o->concnot[c] = p->initconc;
            o->concn[c] = p->initconc;
        }
    }
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++) {
            o->enthalpy[ID(0, j, k)] = hwest;
            o->enthalpy[ID(nim1, j, k)] = heast;
        }
    for (int j = 0; j < nj; j++)
        for (int i = 0; i < ni; i++) o->enthalpy[ID(i, j, 0)] = hbottom;
    for (int k = 0; k < nk; k++)
        for (int i = 0; i < ni; i++) o->enthalpy[ID(i, njm1, k)] = hnorth;
    o->enthbottom = hbottom;
    o->resoru = o->resorv = o->resorw = o->resorm = o->resorh = o->resorc = 0.0;
    o->itertot = 0;
}

/* ---- updateLaser / getLaserCoords: BoundCondManager.cpp:68-275 -------------------- */
static void laser_coords(orc *o)
{
    const amcfd_params *p = &o->p;
    if (!p->udtoolpath) {
        o->oldbeamposx = o->beamposx;
        if (o->timet <= p->lasertime) {
            o->beamposx = p->xstart + o->timet * o->scanvel;
            if (o->init) {
                o->oldbeamposx = o->beamposx;
                o->init = 0;
            }
        } else {
            o->beamposx = p->xstart + p->lasertime * o->scanvel;
            o->powerindicator = 0;
        }
        o->beamposy = p->ystart;
        return;
    }
    double tx = 0.0, ty = 0.0, tz = 0.0, deltaty = 0.0;
    const double small = 1.0e-8;
    o->oldbeamposx = o->beamposx;
    o->oldbeamposy = o->beamposy;
    o->oldbeamposz = o->beamposz;
    int oldpower = o->powerindicator;
    for (int ii = 1; ii < p->ntool; ii++) {
        const double *b = &o->tool[4 * ii];
        if (o->timet <= b[0] + small) {
            const double *a = &o->tool[4 * (ii - 1)];
            double ratio = (o->timet - a[0]) / (b[0] - a[0]);
            double deltatx = b[1] - a[1];
            deltaty = b[2] - a[2];
            double deltatz = b[3] - a[3];
            tx = ratio * deltatx + a[1];
            ty = ratio * deltaty + a[2];
            tz = ratio * deltatz + a[3];
            o->powerindicator = o->tool_on[ii];
            if (o->init) {
                o->oldbeamposx = a[1];
                o->oldbeamposy = a[2];
                o->oldbeamposz = a[3];
                oldpower = o->tool_on[ii - 1];
                o->init = 0;
            }
            break;
        }
    }
    o->beamposx = tx;
    o->beamposy = ty;
    o->beamposz = tz;
    double dist = sqrt((o->beamposx - o->oldbeamposx) * (o->beamposx - o->oldbeamposx) +
                       (o->beamposy - o->oldbeamposy) * (o->beamposy - o->oldbeamposy) +
                       (o->beamposz - o->oldbeamposz) * (o->beamposz - o->oldbeamposz));
    o->scanvel = dist / p->delt;
    if (oldpower - o->powerindicator > 0 && deltaty > small) o->trackindx++;
    /* powder bed: the beam switching on activates the next layer (BoundCondManager.cpp:266-272) */
    if (o->powerindicator - oldpower > 0 && p->powderbed) {
        o->trackindx++;
        if (o->nk + p->ncvzlayer > o->nk_alloc) {
            o->layer_overflow = 1;  /* the reference indexes past its generated grid here */
        } else {
            o->nk += p->ncvzlayer;
            o->nkm1 = o->nk - 1;
            o->nkm2 = o->nk - 2;
        }
    }
}

void orc_update_laser(orc *o)
{
    const amcfd_params *p = &o->p;
    const int ni = o->ni, nj = o->nj;
    if (p->steady)
        o->beamposx = p->xstart;
    else
        laser_coords(o);
    int iout = 0, jout = 0;
    double xloc = o->beamposx;
    for (int i = 1; i < o->nim1; i++) {
        if (xloc <= o->x[i]) break;
        iout = i;
    }
    if (fabs(xloc - o->x[iout + 1]) < fabs(xloc - o->x[iout])) iout++;
    o->istart = iout;
    for (int j = 1; j < o->njm1; j++) {
        if (o->beamposy <= o->y[j]) break;
        jout = j;
    }
    if (fabs(o->beamposy - o->y[jout + 1]) < fabs(o->beamposy - o->y[jout])) jout++;
    o->jstart = jout;
    o->heatinlaser = 0.0;
    double rb2 = p->alasrb * p->alasrb;
    double varlas = p->alaspow * p->alaseta;
    o->peakhin = p->alasfact * varlas / (M_PI * rb2);
    for (int j = 0; j < nj; j++) {
        double ydist = o->beamposy - o->y[j];
        for (int i = 0; i < ni; i++) {
            int c = ni * j + i;
            double xdist = o->beamposx - o->x[i];
            double dist2 = (xdist * xdist) + (ydist * ydist);
            o->heatin[c] = o->peakhin * exp(-p->alasfact * dist2 / rb2) * (double)o->powerindicator;
            if (p->alasfact < 1.0e-6 && dist2 < rb2)
                o->heatin[c] = varlas / (M_PI * rb2) * (double)o->powerindicator;
            o->heatinlaser += o->areaij[c] * o->heatin[c];
        }
    }
    o->imin = o->istart - 2;
    o->imax = o->istart + 2;
    o->jmin = o->jstart - 2;
    o->jmax = o->jstart + 2;
    o->kmin = o->nkm2 - 3;
    o->kmax = o->nkm2;
}

/* ---- getMeltPoolShape: BoundCondManager.cpp:280-447 ------------------------------- */
void orc_meltpool(orc *o)
{
    const int ni = o->ni, nj = o->nj, nk = o->nk;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2, njm2 = o->njm2,
              nkm2 = o->nkm2;
    const double ts = o->p.tsolid;
    const double *T = o->temp, *x = o->x, *y = o->y, *z = o->z;
    size_t n = (size_t)ni * nj * nk;
    double tp = T[0];
    for (size_t c = 1; c < n; c++)
        if (tp < T[c]) tp = T[c];
    o->tpeak = tp;
    if (o->tpeak <= ts) {
        o->alen = o->depth = o->width = 0.0;
        return;
    }
    const int js = o->jstart;
    int i, j, k;
    o->imax = o->istart;
    o->imin = o->istart;
    o->alen = 0.0;
    for (i = o->istart; i < nim1; i++) {
        o->imax = i;
        if (T[ID(i, js, nkm1)] <= ts) break;
    }
    double dtdxxinv = (x[o->imax] - x[o->imax + 1]) /
                      (T[ID(o->imax, js, nkm1)] - T[ID(o->imax + 1, js, nkm1)]);
    double xxmax = x[o->imax] + (ts - T[ID(o->imax, js, nkm1)]) * dtdxxinv;
    for (i = o->istart; i > 0; i--) {
        o->imin = i;
        if (T[ID(i, js, nkm1)] < ts) break;
    }
    dtdxxinv = (x[o->imin] - x[o->imin - 1]) /
               (T[ID(o->imin, js, nkm1)] - T[ID(o->imin - 1, js, nkm1)]);
    double xxmin = x[o->imin] + (ts - T[ID(o->imin, js, nkm1)]) * dtdxxinv;
    o->alen = xxmax - xxmin;

    o->kmin = nkm2;
    o->depth = 0.0;
    for (i = 1; i < nim1; i++)
        for (k = nkm2; k > 0; k--) {
            if (T[ID(i, js, k)] < ts) break;
            o->kmin = MIND(o->kmin, k);
        }
    o->kmin--;
    if (o->kmin == 0) {
        o->depth = z[nkm1] - z[0];
    } else {
        for (i = 1; i < nim1; i++) {
            if (T[ID(i, js, o->kmin + 1)] < ts) continue;
            double dtdzzinv = (z[o->kmin] - z[o->kmin - 1]) /
                              (T[ID(i, js, o->kmin)] - T[ID(i, js, o->kmin - 1)]);
            double dep = z[nkm1] - z[o->kmin] + (T[ID(i, js, o->kmin)] - ts) * dtdzzinv;
            o->depth = MAXD(dep, o->depth);
        }
    }
    o->kmax = nkm2;

    o->jmax = js;
    o->jmin = js;
    o->width = 0.0;
    for (i = 1; i < nim1; i++)
        for (j = js; j < njm1; j++) {
            if (T[ID(i, j, nkm1)] < ts) break;
            o->jmax = MAXD(o->jmax, j);
        }
    o->jmax++;
    double yymax = y[0];
    if (o->jmax != js) {
        for (i = 1; i < nim1; i++) {
            if (T[ID(i, o->jmax - 1, nkm1)] < ts) continue;
            double dtdyyinv = (y[o->jmax] - y[o->jmax + 1]) /
                              (T[ID(i, o->jmax, nkm1)] - T[ID(i, o->jmax + 1, nkm1)]);
            double wid = y[o->jmax] + (ts - T[ID(i, o->jmax, nkm1)]) * dtdyyinv;
            yymax = MAXD(wid, yymax);
        }
    }
    for (i = 1; i < nim1; i++)
        for (j = js; j > 0; j--) {
            if (T[ID(i, j, nkm1)] < ts) break;
            o->jmin = MIND(o->jmin, j);
        }
    o->jmin--;
    double yymin = y[js];
    if (o->jmin != js) {
        for (i = 1; i < nim1; i++) {
            if (T[ID(i, o->jmin + 1, nkm1)] < ts) continue;
            double dtdyyinv = (y[o->jmin] - y[o->jmin - 1]) /
                              (T[ID(i, o->jmin, nkm1)] - T[ID(i, o->jmin - 1, nkm1)]);
            double wid = y[o->jmin] + (ts - T[ID(i, o->jmin, nkm1)]) * dtdyyinv;
            yymin = MIND(wid, yymin);
        }
    }
    o->width = yymax - yymin;
    o->istat = MAXD(o->imin - 3, 1);
    o->iend = MIND(o->imax + 3, nim2);
    o->jstat = MAXD(o->jmin - 3, 1);
    o->jend = MIND(o->jmax + 2, njm2);
    o->kstat = MAXD(o->kmin - 2, 2);
    o->istatp1 = o->istat + 1;
    o->iendm1 = o->iend - 1;
}

/* ---- getSurfaceTensionGradient: BoundCondManager.cpp:706-741 ---------------------- */
static double surface_tension_gradient(const orc *o, double t, double a0)
{
    const double A = 4.3e-4, R = 8314, gamma0 = 1.943, Ts = 2.03e-8, k1 = 1.38e-2, H0 = -1.46e8;
    (void)gamma0;
    double K = k1 * exp(-H0 / R / t);
    double g = (-A - R * Ts * log(1 + K * a0) - (K * a0 / (1 + K * a0)) * (Ts * H0 / t)) * 1;
    if (t >= 2500) g = 0;
    if (a0 < 0) g = o->p.dgdtp;
    return g;
}

/* ---- applyBCs: BoundCondManager.cpp:452-701 --------------------------------------- */
void orc_apply_bcs(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2, njm2 = o->njm2,
              nkm2 = o->nkm2;
    const amcfd_params *p = &o->p;
    int i, j, k;
    switch (ivar) {
    case 1:
        for (j = o->jstat; j <= o->jend; j++)
            for (i = o->istatp1; i <= o->iendm1; i++) {
                double dtdx = (o->temp[ID(i, j, nkm1)] - o->temp[ID(i - 1, j, nkm1)]) * o->dxpwinv[i];
                double fraclu = o->fracl[ID(i, j, nkm1)] * (1.0 - o->fracx[i - 1]) +
                                o->fracl[ID(i - 1, j, nkm1)] * o->fracx[i - 1];
                double visu1 = o->vis[ID(i, j, nkm2)] * o->vis[ID(i - 1, j, nkm2)] /
                               (o->vis[ID(i, j, nkm2)] * (1.0 - o->fracx[i - 1]) +
                                o->vis[ID(i - 1, j, nkm2)] * o->fracx[i - 1]);
                double term1 = fraclu * surface_tension_gradient(o, o->temp[ID(i, j, nkm1)], p->a_oxygen) *
                               dtdx / (visu1 * o->dzpbinv[nkm1]);
                o->uvel[ID(i, j, nkm1)] = o->uvel[ID(i, j, nkm2)] + term1;
            }
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++) {
                o->uvel[ID(o->istat, j, k)] = 0.0;
                o->uvel[ID(o->iend, j, k)] = 0.0;
            }
        break;
    case 2:
        for (j = o->jstat; j <= o->jend; j++)
            for (i = o->istatp1; i <= o->iendm1; i++) {
                double dtdy = (o->temp[ID(i, j, nkm1)] - o->temp[ID(i, j - 1, nkm1)]) * o->dypsinv[j];
                double fraclv = o->fracl[ID(i, j, nkm1)] * (1.0 - o->fracy[j - 1]) +
                                o->fracl[ID(i, j - 1, nkm1)] * o->fracy[j - 1];
                double visv1 = o->vis[ID(i, j, nkm2)] * o->vis[ID(i, j - 1, nkm2)] /
                               (o->vis[ID(i, j, nkm2)] * (1.0 - o->fracy[j - 1]) +
                                o->vis[ID(i, j - 1, nkm2)] * o->fracy[j - 1]);
                double term1 = fraclv * surface_tension_gradient(o, o->temp[ID(i, j, nkm1)], p->a_oxygen) *
                               dtdy / (visv1 * o->dzpbinv[nkm1]);
                o->vvel[ID(i, j, nkm1)] = o->vvel[ID(i, j, nkm2)] + term1;
            }
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++) {
                o->vvel[ID(o->istat, j, k)] = 0.0;
                o->vvel[ID(o->iend, j, k)] = 0.0;
            }
        break;
    case 3:
    case 4: {
        double *phi = ivar == 3 ? o->wvel : o->pp;
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++) {
                phi[ID(o->istat, j, k)] = 0.0;
                phi[ID(o->iend, j, k)] = 0.0;
            }
        break;
    }
    case 5: {
        double hlossevap = 0.0;
        o->ahtoploss = 0.0;
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                double t = o->temp[ID(i, j, nkm1)];
                if (p->isevap) {
                    double psat = p->pressamb * exp(-p->evaplatent * p->molarmass / p->gasconst *
                                                    (1.0 / t - 1.0 / p->evaptemp));
                    double mdot = p->evapfact * psat * sqrt(p->molarmass / (2.0 * M_PI * p->gasconst * t));
                    hlossevap = mdot * p->evaplatent;
                }
                double t4 = t;
                for (int q = 1; q < 4; q++) t4 *= t;
                double a4 = p->tempamb;
                for (int q = 1; q < 4; q++) a4 *= p->tempamb;
                double hlossradia = p->emiss * p->sigm * (t4 - a4);
                double ctmp1 = o->diff[ID(i, j, nkm2)] * o->dzpbinv[nkm1];
                o->enthalpy[ID(i, j, nkm1)] = o->enthalpy[ID(i, j, nkm2)] +
                    (o->heatin[j * ni + i] - hlossradia - hlossradia - hlossevap) / ctmp1;
                o->ahtoploss += (hlossradia + hlossradia + hlossevap) * o->areaij[j * ni + i];
            }
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++) {
                double hc = p->htci * (o->temp[ID(0, j, k)] - p->tempamb);
                double ctmp1 = o->diff[ID(1, j, k)] * o->dxpwinv[1];
                o->enthalpy[ID(0, j, k)] = o->enthalpy[ID(1, j, k)] - hc / ctmp1;
                hc = p->htci * (o->temp[ID(nim1, j, k)] - p->tempamb);
                ctmp1 = o->diff[ID(nim2, j, k)] * o->dxpwinv[nim2];
                o->enthalpy[ID(nim1, j, k)] = o->enthalpy[ID(nim2, j, k)] - hc / ctmp1;
            }
        for (k = 1; k < nkm1; k++)
            for (i = 1; i < nim1; i++) {
                double hc = p->htcj * (o->temp[ID(i, 0, k)] - p->tempamb);
                double ctmp1 = o->diff[ID(i, 1, k)] * o->dypsinv[1];
                o->enthalpy[ID(i, 0, k)] = o->enthalpy[ID(i, 1, k)] - hc / ctmp1;
                hc = p->htcj * (o->temp[ID(i, njm1, k)] - p->tempamb);
                ctmp1 = o->diff[ID(i, njm2, k)] * o->dypsinv[njm2];
                o->enthalpy[ID(i, njm1, k)] = o->enthalpy[ID(i, njm2, k)] - hc / ctmp1;
            }
        break;
    }
    case 6: {
        /* BoundCondManager.cpp:655-699: top (flux towards the surface value 13 where
         * the top node is above the liquidus) and bottom planes, then the south/north
         * rows over every (k, i), then the west/east columns over every (k, j) */
        const double initval = p->initconc, dsl = p->dens * p->massdiff;
        double *cn = o->conc;
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                if (o->temp[ID(i, j, nkm1)] > p->tliquid)
                    cn[ID(i, j, nkm1)] = 2.0 * (13.0 - cn[ID(i, j, nkm2)]) / o->dzpbinv[nkm1] / dsl +
                                         cn[ID(i, j, nkm2)];
                else
                    cn[ID(i, j, nkm1)] = cn[ID(i, j, nkm2)];
                cn[ID(i, j, 0)] = initval;
            }
        for (k = 0; k < o->nk; k++)
            for (i = 0; i < ni; i++) {
                cn[ID(i, 0, k)] = cn[ID(i, 1, k)];
                cn[ID(i, njm1, k)] = cn[ID(i, njm1 - 1, k)];
            }
        for (k = 0; k < o->nk; k++)
            for (j = 0; j < nj; j++) {
                cn[ID(0, j, k)] = cn[ID(1, j, k)];
                cn[ID(nim1, j, k)] = cn[ID(nim1 - 1, j, k)];
            }
        break;
    }
    }
}

/* ---- discretizeEquations: CFDSolverManager.cpp:727-1264 --------------------------- */
#define HARM(a, b, f) ((a) * (b) / ((f) * (b) + (1.0 - (f)) * (a)))
static void coef_pair(int scheme, double d, double f, double *aplus, double *aminus)
{
    /* aplus: d*A(|f|/d) + max(0,-f) ; aminus: d*A(|f|/d) + max(0,f) */
    double a = d * scheme_fn(scheme, fabs(f) / d);
    *aplus = a + MAXD(0.0, -f);
    *aminus = a + MAXD(0.0, f);
}

void orc_discretize(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2, njm2 = o->njm2,
              nkm2 = o->nkm2;
    const int sch = o->p.scheme;
    const double delt = o->p.delt;
    const double *fx = o->fracx, *fy = o->fracy, *fz = o->fracz;
    const double *u = o->uvel, *v = o->vvel, *w = o->wvel, *rho = o->rho, *vis = o->vis;
    const double *xu = o->xu, *yv = o->yv, *zw = o->zw;
    int i, j, k;
    double tmp;
    switch (ivar) {
    case 1:
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    double vn = v[ID(i, j + 1, k)] * (1.0 - fx[i - 1]) + v[ID(i - 1, j + 1, k)] * fx[i - 1];
                    double vs = v[c] * (1.0 - fx[i - 1]) + v[ID(i - 1, j, k)] * fx[i - 1];
                    double ue = (u[ID(i + 1, j, k)] + u[c]) * 0.5;
                    double uw = (u[ID(i - 1, j, k)] + u[c]) * 0.5;
                    double wt = w[ID(i, j, k + 1)] * (1.0 - fx[i - 1]) + w[ID(i - 1, j, k + 1)] * fx[i - 1];
                    double wb = w[c] * (1.0 - fx[i - 1]) + w[ID(i - 1, j, k)] * fx[i - 1];
                    double fn = vn * rho[c] * o->areauik[k * ni + i];
                    double fs = vs * rho[c] * o->areauik[k * ni + i];
                    double fe = ue * rho[c] * o->areajk[k * nj + j];
                    double fw = uw * rho[c] * o->areajk[k * nj + j];
                    double ft = wt * rho[c] * o->areauij[j * ni + i];
                    double fb = wb * rho[c] * o->areauij[j * ni + i];
                    double visu = vis[c] * vis[ID(i - 1, j, k)] /
                                  (fx[i - 1] * vis[ID(i - 1, j, k)] + (1.0 - fx[i - 1]) * vis[c]);
                    double visun = vis[ID(i, j + 1, k)] * vis[ID(i - 1, j + 1, k)] /
                                   (fx[i - 1] * vis[ID(i - 1, j + 1, k)] + (1.0 - fx[i - 1]) * vis[ID(i, j + 1, k)]);
                    double visus = vis[ID(i, j - 1, k)] * vis[ID(i - 1, j - 1, k)] /
                                   (fx[i - 1] * vis[ID(i - 1, j - 1, k)] + (1.0 - fx[i - 1]) * vis[ID(i, j - 1, k)]);
                    double visn = (j == njm2) ? visu : visu * visun / ((1.0 - fy[j]) * visun + fy[j] * visu);
                    double viss = (j == 1) ? visu : visu * visus / (fy[j - 1] * visus + (1.0 - fy[j - 1]) * visu);
                    double vise = vis[c];
                    double visw = vis[ID(i - 1, j, k)];
                    double visut = vis[ID(i, j, k + 1)] * vis[ID(i - 1, j, k + 1)] /
                                   (fx[i - 1] * vis[ID(i - 1, j, k + 1)] + (1.0 - fx[i - 1]) * vis[ID(i, j, k + 1)]);
                    double visub = vis[ID(i, j, k - 1)] * vis[ID(i - 1, j, k - 1)] /
                                   (fx[i - 1] * vis[ID(i - 1, j, k - 1)] + (1.0 - fx[i - 1]) * vis[ID(i, j, k - 1)]);
                    double vist = (k == nkm2) ? visu : visut * visu / (fz[k] * visu + (1.0 - fz[k]) * visut);
                    double visb = (k == 1) ? visu : visub * visu / ((1.0 - fz[k - 1]) * visu + fz[k - 1] * visub);
                    double dn = visn * o->areauik[k * ni + i] * o->dypsinv[j + 1];
                    double ds = viss * o->areauik[k * ni + i] * o->dypsinv[j];
                    double de = vise * o->areajk[k * nj + j] / (xu[i + 1] - xu[i]);
                    double dw = visw * o->areajk[k * nj + j] / (xu[i] - xu[i - 1]);
                    double dt = vist * o->areauij[j * ni + i] * o->dzpbinv[k + 1];
                    double db = visb * o->areauij[j * ni + i] * o->dzpbinv[k];
                    coef_pair(sch, dn, fn, &o->an[c], &tmp);
                    coef_pair(sch, ds, fs, &tmp, &o->as[c]);
                    coef_pair(sch, de, fe, &o->ae[c], &tmp);
                    coef_pair(sch, dw, fw, &tmp, &o->aw[c]);
                    coef_pair(sch, dt, ft, &o->at[c], &tmp);
                    coef_pair(sch, db, fb, &tmp, &o->ab[c]);
                    o->apnot[c] = rho[c] * o->volume_u[c] / delt;
                    double delf = fn - fs + fe - fw + ft - fb;
                    double cp0 = MAXD(0.0, delf), cp1 = MIND(0.0, delf);
                    o->su[c] = -cp1 * u[c];
                    o->su[c] += o->areajk[k * nj + j] * (o->pressure[ID(i - 1, j, k)] - o->pressure[c]);
                    o->sp[c] = -cp0;
                    o->su[c] += o->apnot[c] * o->unot[c];
                    double dudxp = (u[ID(i + 1, j, k)] - u[c]) / (xu[i + 1] - xu[i]);
                    double dudxm = (u[c] - u[ID(i - 1, j, k)]) / (xu[i] - xu[i - 1]);
                    o->su[c] += (vise * dudxp - visw * dudxm) * o->areajk[k * nj + j];
                    double dvdxp = (v[ID(i, j + 1, k)] - v[ID(i - 1, j + 1, k)]) * o->dxpwinv[i];
                    double dvdxm = (v[c] - v[ID(i - 1, j, k)]) * o->dxpwinv[i];
                    o->su[c] += (visn * dvdxp - viss * dvdxm) * o->areauik[k * ni + i];
                    double dwdxp = (w[ID(i, j, k + 1)] - w[ID(i - 1, j, k + 1)]) * o->dxpwinv[i];
                    double dwdxm = (w[c] - w[ID(i - 1, j, k)]) * o->dxpwinv[i];
                    o->su[c] += (vist * dwdxp - visb * dwdxm) * o->areauij[j * ni + i];
                }
        break;
    case 2:
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    double vn = (v[c] + v[ID(i, j + 1, k)]) * 0.5;
                    double vs = (v[c] + v[ID(i, j - 1, k)]) * 0.5;
                    double ue = u[ID(i + 1, j, k)] * (1.0 - fy[j - 1]) + u[ID(i + 1, j - 1, k)] * fy[j - 1];
                    double uw = u[c] * (1.0 - fy[j - 1]) + u[ID(i, j - 1, k)] * fy[j - 1];
                    double wt = w[ID(i, j, k + 1)] * (1.0 - fy[j - 1]) + w[ID(i, j - 1, k + 1)] * fy[j - 1];
                    double wb = w[c] * (1.0 - fy[j - 1]) + w[ID(i, j - 1, k)] * fy[j - 1];
                    double fn = vn * rho[c] * o->areaik[k * ni + i];
                    double fs = vs * rho[c] * o->areaik[k * ni + i];
                    double fe = ue * rho[c] * o->areavjk[k * nj + j];
                    double fw = uw * rho[c] * o->areavjk[k * nj + j];
                    double ft = wt * rho[c] * o->areavij[j * ni + i];
                    double fb = wb * rho[c] * o->areavij[j * ni + i];
                    double visn = vis[c];
                    double viss = vis[ID(i, j - 1, k)];
                    double visv = vis[c] * vis[ID(i, j - 1, k)] /
                                  (fy[j - 1] * vis[ID(i, j - 1, k)] + (1.0 - fy[j - 1]) * vis[c]);
                    double visve = vis[ID(i + 1, j, k)] * vis[ID(i + 1, j - 1, k)] /
                                   (fy[j - 1] * vis[ID(i + 1, j - 1, k)] + (1.0 - fy[j - 1]) * vis[ID(i + 1, j, k)]);
                    double visvw = vis[ID(i - 1, j, k)] * vis[ID(i - 1, j - 1, k)] /
                                   (fy[j - 1] * vis[ID(i - 1, j - 1, k)] + (1.0 - fy[j - 1]) * vis[ID(i - 1, j, k)]);
                    double vise = (i == nim2) ? visv : visv * visve / ((1.0 - fx[i]) * visve + fx[i] * visv);
                    double visw = (i == 1) ? visv : visv * visvw / (fx[i - 1] * visvw + (1.0 - fx[i - 1]) * visv);
                    double visvt = vis[ID(i, j, k + 1)] * vis[ID(i, j - 1, k + 1)] /
                                   (fy[j - 1] * vis[ID(i, j - 1, k + 1)] + (1.0 - fy[j - 1]) * vis[ID(i, j, k + 1)]);
                    double visvb = vis[ID(i, j, k - 1)] * vis[ID(i, j - 1, k - 1)] /
                                   (fy[j - 1] * vis[ID(i, j - 1, k - 1)] + (1.0 - fy[j - 1]) * vis[ID(i, j, k - 1)]);
                    double vist = (k == nkm2) ? visv : visv * visvt / ((1.0 - fz[k]) * visvt + fz[k] * visv);
                    double visb = (k == 1) ? visv : visv * visvb / (fz[k - 1] * visvb + (1.0 - fz[k - 1]) * visv);
                    double dn = visn * o->areaik[k * ni + i] / (yv[j + 1] - yv[j]);
                    double ds = viss * o->areaik[k * ni + i] / (yv[j] - yv[j - 1]);
                    double de = vise * o->areavjk[k * nj + j] * o->dxpwinv[i + 1];
                    double dw = visw * o->areavjk[k * nj + j] * o->dxpwinv[i];
                    double dt = vist * o->areavij[j * ni + i] * o->dzpbinv[k + 1];
                    double db = visb * o->areavij[j * ni + i] * o->dzpbinv[k];
                    coef_pair(sch, dn, fn, &o->an[c], &tmp);
                    coef_pair(sch, ds, fs, &tmp, &o->as[c]);
                    coef_pair(sch, de, fe, &o->ae[c], &tmp);
                    coef_pair(sch, dw, fw, &tmp, &o->aw[c]);
                    coef_pair(sch, dt, ft, &o->at[c], &tmp);
                    coef_pair(sch, db, fb, &tmp, &o->ab[c]);
                    o->apnot[c] = rho[c] * o->volume_v[c] / delt;
                    double delf = fn - fs + fe - fw + ft - fb;
                    double cp0 = MAXD(0.0, delf), cp1 = MIND(0.0, delf);
                    o->su[c] = -cp1 * v[c];
                    o->su[c] += o->areaik[k * ni + i] * (o->pressure[ID(i, j - 1, k)] - o->pressure[c]);
                    o->sp[c] = -cp0;
                    o->su[c] += o->apnot[c] * o->vnot[c];
                    double dudyp = (u[ID(i + 1, j, k)] - u[ID(i + 1, j - 1, k)]) * o->dypsinv[j];
                    double dudym = (u[c] - u[ID(i, j - 1, k)]) * o->dypsinv[j];
                    o->su[c] += (vise * dudyp - visw * dudym) * o->areavjk[k * nj + j];
                    double dvdyp = (v[ID(i, j + 1, k)] - v[c]) / (yv[j + 1] - yv[j]);
                    double dvdym = (v[c] - v[ID(i, j - 1, k)]) / (yv[j] - yv[j - 1]);
                    o->su[c] += (visn * dvdyp - viss * dvdym) * o->areaik[k * ni + i];
                    double dwdyp = (w[ID(i, j, k + 1)] - w[ID(i, j - 1, k + 1)]) * o->dypsinv[j];
                    double dwdym = (w[c] - w[ID(i, j - 1, k)]) * o->dypsinv[j];
                    o->su[c] += (vist * dwdyp - visb * dwdym) * o->areavij[j * ni + i];
                }
        break;
    case 3:
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    double vn = v[ID(i, j + 1, k)] * (1.0 - fz[k - 1]) + v[ID(i, j + 1, k - 1)] * fz[k - 1];
                    double vs = v[c] * (1.0 - fz[k - 1]) + v[ID(i, j, k - 1)] * fz[k - 1];
                    double ue = u[ID(i + 1, j, k)] * (1.0 - fz[k - 1]) + u[ID(i + 1, j, k - 1)] * fz[k - 1];
                    double uw = u[c] * (1.0 - fz[k - 1]) + u[ID(i, j, k - 1)] * fz[k - 1];
                    double wt = (w[c] + w[ID(i, j, k + 1)]) * 0.5;
                    double wb = (w[c] + w[ID(i, j, k - 1)]) * 0.5;
                    double fn = vn * rho[c] * o->areawik[k * ni + i];
                    double fs = vs * rho[c] * o->areawik[k * ni + i];
                    double fe = ue * rho[c] * o->areawjk[k * nj + j];
                    double fw = uw * rho[c] * o->areawjk[k * nj + j];
                    double ft = wt * rho[c] * o->areaij[j * ni + i];
                    double fb = wb * rho[c] * o->areaij[j * ni + i];
                    double vis_w = vis[c] * vis[ID(i, j, k - 1)] /
                                   (fz[k - 1] * vis[ID(i, j, k - 1)] + (1.0 - fz[k - 1]) * vis[c]);
                    double viswn = vis[ID(i, j + 1, k)] * vis[ID(i, j + 1, k - 1)] /
                                   (fz[k - 1] * vis[ID(i, j + 1, k - 1)] + (1.0 - fz[k - 1]) * vis[ID(i, j + 1, k)]);
                    double visws = vis[ID(i, j - 1, k)] * vis[ID(i, j - 1, k - 1)] /
                                   (fz[k - 1] * vis[ID(i, j - 1, k - 1)] + (1.0 - fz[k - 1]) * vis[ID(i, j - 1, k)]);
                    double visn = (j == njm2) ? vis_w : vis_w * viswn / ((1.0 - fy[j]) * viswn + fy[j] * vis_w);
                    double viss = (j == 1) ? vis_w : vis_w * visws / (fy[j - 1] * visws + (1.0 - fy[j - 1]) * vis_w);
                    double viswe = vis[ID(i + 1, j, k)] * vis[ID(i + 1, j, k - 1)] /
                                   (fz[k - 1] * vis[ID(i + 1, j, k - 1)] + (1.0 - fz[k - 1]) * vis[ID(i + 1, j, k)]);
                    double visww = vis[ID(i - 1, j, k)] * vis[ID(i - 1, j, k - 1)] /
                                   (fz[k - 1] * vis[ID(i - 1, j, k - 1)] + (1.0 - fz[k - 1]) * vis[ID(i - 1, j, k)]);
                    double vise = (i == nim2) ? vis_w : vis_w * viswe / ((1.0 - fx[i]) * viswe + fx[i] * vis_w);
                    double visw = (i == 1) ? vis_w : vis_w * visww / (fx[i - 1] * visww + (1.0 - fx[i - 1]) * vis_w);
                    double vist = vis[c];
                    double visb = vis[ID(i, j, k - 1)];
                    double dn = visn * o->areawik[k * ni + i] * o->dypsinv[j + 1];
                    double ds = viss * o->areawik[k * ni + i] * o->dypsinv[j];
                    double de = vise * o->areawjk[k * nj + j] * o->dxpwinv[i + 1];
                    double dw = visw * o->areawjk[k * nj + j] * o->dxpwinv[i];
                    double dt = vist * o->areaij[j * ni + i] / (zw[k + 1] - zw[k]);
                    double db = visb * o->areaij[j * ni + i] / (zw[k] - zw[k - 1]);
                    coef_pair(sch, dn, fn, &o->an[c], &tmp);
                    coef_pair(sch, ds, fs, &tmp, &o->as[c]);
                    coef_pair(sch, de, fe, &o->ae[c], &tmp);
                    coef_pair(sch, dw, fw, &tmp, &o->aw[c]);
                    coef_pair(sch, dt, ft, &o->at[c], &tmp);
                    coef_pair(sch, db, fb, &tmp, &o->ab[c]);
                    o->apnot[c] = rho[c] * o->volume_w[c] / delt;
                    double delf = fn - fs + fe - fw + ft - fb;
                    double cp0 = MAXD(0.0, delf), cp1 = MIND(0.0, delf);
                    o->su[c] = -cp1 * w[c];
                    o->su[c] += o->areaij[j * ni + i] * (o->pressure[ID(i, j, k - 1)] - o->pressure[c]);
                    o->sp[c] = -cp0;
                    o->su[c] += o->apnot[c] * o->wnot[c];
                    double dudzp = (u[ID(i + 1, j, k)] - u[ID(i + 1, j, k - 1)]) * o->dzpbinv[k];
                    double dudzm = (u[c] - u[ID(i, j, k - 1)]) * o->dzpbinv[k];
                    o->su[c] += (vise * dudzp - visw * dudzm) * o->areawjk[k * nj + j];
                    double dvdzp = (v[ID(i, j + 1, k)] - v[ID(i, j + 1, k - 1)]) * o->dzpbinv[k];
                    double dvdzm = (v[c] - v[ID(i, j, k - 1)]) * o->dzpbinv[k];
                    o->su[c] += (visn * dvdzp - viss * dvdzm) * o->areawik[k * ni + i];
                    double dwdzp = (w[ID(i, j, k + 1)] - w[c]) / (zw[k + 1] - zw[k]);
                    double dwdzm = (w[c] - w[ID(i, j, k - 1)]) / (zw[k] - zw[k - 1]);
                    o->su[c] += (vist * dwdzp - visb * dwdzm) * o->areaij[j * ni + i];
                }
        break;
    case 4:
        o->resorm = 0.0;
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    o->an[c] = o->areaik[k * ni + i] * o->dvy[ID(i, j + 1, k)] * rho[c];
                    o->as[c] = o->areaik[k * ni + i] * o->dvy[c] * rho[c];
                    o->ae[c] = o->areajk[k * nj + j] * o->dux[ID(i + 1, j, k)] * rho[c];
                    o->aw[c] = o->areajk[k * nj + j] * o->dux[c] * rho[c];
                    o->at[c] = o->areaij[j * ni + i] * o->dwz[ID(i, j, k + 1)] * rho[c];
                    o->ab[c] = o->areaij[j * ni + i] * o->dwz[c] * rho[c];
                    double fn = v[ID(i, j + 1, k)] * o->areaik[k * ni + i] * rho[c];
                    double fs = v[c] * o->areaik[k * ni + i] * rho[c];
                    double fe = u[ID(i + 1, j, k)] * o->areajk[k * nj + j] * rho[c];
                    double fw = u[c] * o->areajk[k * nj + j] * rho[c];
                    double ft = w[ID(i, j, k + 1)] * o->areaij[j * ni + i] * rho[c];
                    double fb = w[c] * o->areaij[j * ni + i] * rho[c];
                    double delf = fn - fs + fe - fw + ft - fb;
                    o->sp[c] = 0.0;
                    o->su[c] = -delf;
                    o->resorm += fabs(delf);
                }
        break;
    case 5: {
        const double *df = o->diff;
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++)
                for (i = 1; i < nim1; i++) {
                    size_t c = ID(i, j, k);
                    double vn = v[ID(i, j + 1, k)];
                    double ue = u[ID(i + 1, j, k)];
                    double wt = w[ID(i, j, k + 1)];
                    double densbydt = rho[c] / delt;
                    double fn = rho[ID(i, j + 1, k)] * vn * o->areaik[k * ni + i];
                    double fe = rho[ID(i + 1, j, k)] * ue * o->areajk[k * nj + j];
                    double ft = rho[ID(i, j, k + 1)] * wt * o->areaij[j * ni + i];
                    double difn = df[c] * df[ID(i, j + 1, k)] /
                                  ((1.0 - fy[j]) * df[ID(i, j + 1, k)] + fy[j] * df[c]);
                    double dife = df[c] * df[ID(i + 1, j, k)] /
                                  ((1.0 - fx[i]) * df[ID(i + 1, j, k)] + fx[i] * df[c]);
                    double dift = df[c] * df[ID(i, j, k + 1)] /
                                  ((1.0 - fz[k]) * df[ID(i, j, k + 1)] + fz[k] * df[c]);
                    double dn = difn * o->areaik[k * ni + i] * o->dypsinv[j + 1];
                    double de = dife * o->areajk[k * nj + j] * o->dxpwinv[i + 1];
                    double dt = dift * o->areaij[j * ni + i] * o->dzpbinv[k + 1];
                    coef_pair(sch, dn, fn, &o->an[c], &o->as[ID(i, j + 1, k)]);
                    coef_pair(sch, de, fe, &o->ae[c], &o->aw[ID(i + 1, j, k)]);
                    coef_pair(sch, dt, ft, &o->at[c], &o->ab[ID(i, j, k + 1)]);
                    o->apnot[c] = densbydt * o->volume[c];
                    o->sp[c] = 0.0;
                    o->su[c] = o->apnot[c] * o->hnot[c];
                }
        for (k = 1; k < nkm1; k++)
            for (i = 1; i < nim1; i++) {
                double vs = v[ID(i, 1, k)];
                double fs = rho[ID(i, 1, k)] * vs * o->areaik[k * ni + i];
                double ds = df[ID(i, 1, k)] * o->areaik[k * ni + i] * o->dypsinv[1];
                coef_pair(sch, ds, fs, &tmp, &o->as[ID(i, 1, k)]);
                double vn = v[ID(i, njm1, k)];
                double fn = rho[ID(i, njm1, k)] * vn * o->areaik[k * ni + i];
                double dn = df[ID(i, njm2, k)] * o->areaik[k * ni + i] * o->dypsinv[njm1];
                coef_pair(sch, dn, fn, &o->an[ID(i, njm2, k)], &tmp);
            }
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++) {
                double uw = u[ID(1, j, k)];
                double fw = rho[ID(1, j, k)] * uw * o->areajk[k * nj + j];
                double dw = df[ID(1, j, k)] * o->areajk[k * nj + j] * o->dxpwinv[1];
                coef_pair(sch, dw, fw, &tmp, &o->aw[ID(1, j, k)]);
                double ue = u[ID(nim1, j, k)];
                double fe = rho[ID(nim1, j, k)] * ue * o->areajk[k * nj + j];
                double de = df[ID(nim2, j, k)] * o->areajk[k * nj + j] * o->dxpwinv[nim1];
                coef_pair(sch, de, fe, &o->ae[ID(nim2, j, k)], &tmp);
            }
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                double wb = w[ID(i, j, 1)];
                double fb = rho[ID(i, j, 1)] * wb * o->areaij[j * ni + i];
                double db = df[ID(i, j, 1)] * o->areaij[j * ni + i] * o->dzpbinv[1];
                coef_pair(sch, db, fb, &tmp, &o->ab[ID(i, j, 1)]);
                double wt = w[ID(i, j, nkm1)];
                double ft = rho[ID(i, j, nkm1)] * wt * o->areaij[j * ni + i];
                double dt = df[ID(i, j, nkm2)] * o->areaij[j * ni + i] * o->dzpbinv[nkm1];
                coef_pair(sch, dt, ft, &o->at[ID(i, j, nkm2)], &tmp);
            }
        break;
    }
    case 6: {
        /* discretizeEquations(6), :1265-1362.  Cell diffusivity 1e-11 at or below the
         * solidus, massdiff * rho above; face velocities doubled in the mass fluxes;
         * each face conductance uses the diffusivity of the cell on its low side. */
        const size_t n = (size_t)ni * nj * o->nk;
        double *ds = dalloc(n);
        for (size_t c = 0; c < n; c++) ds[c] = o->temp[c] <= o->p.tsolid ? 1e-11 : o->p.massdiff * rho[c];
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++)
                for (i = 1; i < nim1; i++) {
                    size_t c = ID(i, j, k);
                    double vn = v[ID(i, j + 1, k)] * 2.0;
                    double ue = u[ID(i + 1, j, k)] * 2.0;
                    double wt = w[ID(i, j, k + 1)] * 2.0;
                    double fn = rho[ID(i, j + 1, k)] * vn * o->areaik[k * ni + i];
                    double fe = rho[ID(i + 1, j, k)] * ue * o->areajk[k * nj + j];
                    double ft = rho[ID(i, j, k + 1)] * wt * o->areaij[j * ni + i];
                    double dn = ds[c] * o->areaik[k * ni + i] * o->dypsinv[j + 1];
                    double de = ds[c] * o->areajk[k * nj + j] * o->dxpwinv[i + 1];
                    double dt = ds[c] * o->areaij[j * ni + i] * o->dzpbinv[k + 1];
                    double densbydt = rho[c] / delt;
                    coef_pair(sch, dn, fn, &o->an[c], &o->as[ID(i, j + 1, k)]);
                    coef_pair(sch, de, fe, &o->ae[c], &o->aw[ID(i + 1, j, k)]);
                    coef_pair(sch, dt, ft, &o->at[c], &o->ab[ID(i, j, k + 1)]);
                    o->apnot[c] = densbydt * o->volume[c];
                    o->sp[c] = 0.0;
                    o->su[c] = o->apnot[c] * o->concnot[c];
                }
        for (k = 1; k < nkm1; k++)
            for (i = 1; i < nim1; i++) {
                double vs = v[ID(i, 1, k)] * 2;
                double fs = rho[ID(i, 1, k)] * vs * o->areaik[k * ni + i];
                double dss = ds[ID(i, 1, k)] * o->areaik[k * ni + i] * o->dypsinv[1];
                coef_pair(sch, dss, fs, &tmp, &o->as[ID(i, 1, k)]);
            }
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++) {
                double uw = u[ID(1, j, k)] * 2;
                double fw = rho[ID(1, j, k)] * uw * o->areajk[k * nj + j];
                double dw = ds[ID(1, j, k)] * o->areajk[k * nj + j] * o->dxpwinv[1];
                coef_pair(sch, dw, fw, &tmp, &o->aw[ID(1, j, k)]);
            }
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                double wb = w[ID(i, j, 1)] * 2;
                double fb = rho[ID(i, j, 1)] * wb * o->areaij[j * ni + i];
                double db = ds[ID(i, j, 1)] * o->areaij[j * ni + i] * o->dzpbinv[1];
                coef_pair(sch, db, fb, &tmp, &o->ab[ID(i, j, 1)]);
            }
        free(ds);
        break;
    }
    }
}

/* ---- calculateSource: CFDSolverManager.cpp:1376-1843 ------------------------------ */
static void momentum_source(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj;
    const int nkm1 = o->nkm1, nkm2 = o->nkm2;
    const amcfd_params *p = &o->p;
    double *phi = ivar == 1 ? o->uvel : ivar == 2 ? o->vvel : o->wvel;
    double *dcoef = ivar == 1 ? o->dux : ivar == 2 ? o->dvy : o->dwz;
    const double *vol = ivar == 1 ? o->volume_u : ivar == 2 ? o->volume_v : o->volume_w;
    double urf = ivar == 1 ? p->urfu : ivar == 2 ? p->urfv : p->urfw;
    int i, j, k;
    for (k = o->kstat; k < nkm1; k++)
        for (j = o->jstat; j <= o->jend; j++)
            for (i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, k);
                double fl;
                size_t cn;  /* upstream neighbour of the staggered face */
                if (ivar == 1) {
                    cn = ID(i - 1, j, k);
                    fl = o->fracl[c] * (1.0 - o->fracx[i - 1]) + o->fracl[cn] * o->fracx[i - 1];
                } else if (ivar == 2) {
                    cn = ID(i, j - 1, k);
                    fl = o->fracl[c] * (1.0 - o->fracy[j - 1]) + o->fracl[cn] * o->fracy[j - 1];
                } else {
                    cn = ID(i, j, k - 1);
                    fl = o->fracl[c] * (1.0 - o->fracz[k - 1]) + o->fracl[cn] * o->fracz[k - 1];
                }
                double rhoscan = o->rho[c] * o->scanvel;
                double boufac = o->rho[c] * p->grav * p->beta;
                if (fl > 0) {
                    double term = p->darcyKo * ((1.0 - fl) * (1.0 - fl)) / ((fl * fl * fl) + SMALL);
                    o->sp[c] -= term * vol[c];
                    if (p->steady) {
                        double area = ivar == 1 ? o->areajk[k * nj + j]
                                    : ivar == 2 ? o->areavjk[k * nj + j] : o->areawjk[k * nj + j];
                        double term1 = rhoscan * area * (phi[ID(i - 1, j, k)] - phi[c]);
                        o->su[c] += term1;
                    }
                    if (ivar == 3) {
                        double tw = o->temp[c] * (1.0 - o->fracz[k - 1]) + o->temp[cn] * o->fracz[k - 1];
                        o->su[c] += boufac * vol[c] * (tw - p->tsolid);
                    }
                }
            }
    if (ivar != 3) {
        for (j = o->jstat; j <= o->jend; j++)
            for (i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, nkm2);
                o->su[c] += o->at[c] * phi[ID(i, j, nkm1)];
                o->sp[c] -= o->at[c];
                o->at[c] = 0.0;
            }
    }
    for (k = o->kstat; k < nkm1; k++)
        for (j = o->jstat; j <= o->jend; j++)
            for (i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, k);
                o->ap[c] = o->an[c] + o->as[c] + o->ae[c] + o->aw[c] + o->at[c] + o->ab[c] +
                           o->apnot[c] - o->sp[c];
                double area = ivar == 1 ? o->areajk[k * nj + j]
                            : ivar == 2 ? o->areaik[k * ni + i] : o->areaij[j * ni + i];
                dcoef[c] = area / o->ap[c];
                o->ap[c] /= urf;
                o->su[c] += (1.0 - urf) * o->ap[c] * phi[c];
                dcoef[c] *= urf;
                size_t cn = ivar == 1 ? ID(i - 1, j, k) : ivar == 2 ? ID(i, j - 1, k) : ID(i, j, k - 1);
                double tlc = MIND(o->temp[c], o->temp[cn]);
                if (tlc <= p->tsolid) {
                    o->su[c] = 0.0;
                    o->an[c] = o->as[c] = o->ae[c] = o->aw[c] = o->at[c] = o->ab[c] = 0.0;
                    o->ap[c] = LARGE;
                }
            }
}

/* Boundary folds and under-relaxation shared by calculateSource(5) and (6)
 * (CFDSolverManager.cpp:1779-1839, 1853-1920): the k, then j, then i boundary
 * coefficients move into su/sp against the boundary values of phi, then
 * ap = sum(a_nb) + apnot - sp, ap /= urf, su += (1 - urf) ap phi. */
static void fold_and_relax(orc *o, const double *h, double urf)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2, njm2 = o->njm2,
              nkm2 = o->nkm2;
    int i, j, k;
    for (j = 1; j < njm1; j++)
        for (i = 1; i < nim1; i++) {
            size_t c = ID(i, j, 1);
            o->su[c] += o->ab[c] * h[ID(i, j, 0)];
            o->sp[c] -= o->ab[c];
            o->ab[c] = 0.0;
            c = ID(i, j, nkm2);
            o->su[c] += o->at[c] * h[ID(i, j, nkm1)];
            o->sp[c] -= o->at[c];
            o->at[c] = 0.0;
        }
    for (k = 1; k < nkm1; k++)
        for (i = 1; i < nim1; i++) {
            size_t c = ID(i, 1, k);
            o->su[c] += o->as[c] * h[ID(i, 0, k)];
            o->sp[c] -= o->as[c];
            o->as[c] = 0.0;
            c = ID(i, njm2, k);
            o->su[c] += o->an[c] * h[ID(i, njm1, k)];
            o->sp[c] -= o->an[c];
            o->an[c] = 0.0;
        }
    for (k = 1; k < nkm1; k++)
        for (j = 1; j < njm1; j++) {
            size_t c = ID(1, j, k);
            o->su[c] += o->aw[c] * h[ID(0, j, k)];
            o->sp[c] -= o->aw[c];
            o->aw[c] = 0.0;
            c = ID(nim2, j, k);
            o->su[c] += o->ae[c] * h[ID(nim1, j, k)];
            o->sp[c] -= o->ae[c];
            o->ae[c] = 0.0;
        }
    for (k = 1; k < nkm1; k++)
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                size_t c = ID(i, j, k);
                o->ap[c] = o->an[c] + o->as[c] + o->ae[c] + o->aw[c] + o->at[c] + o->ab[c] +
                           o->apnot[c] - o->sp[c];
                o->ap[c] /= urf;
                o->su[c] += (1.0 - urf) * o->ap[c] * h[c];
            }
}

void orc_source(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1;
    const amcfd_params *p = &o->p;
    int i, j, k;
    if (ivar >= 1 && ivar <= 3) {
        momentum_source(o, ivar);
        return;
    }
    if (ivar == 4) {
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    o->ap[c] = o->an[c] + o->as[c] + o->ae[c] + o->aw[c] + o->at[c] + o->ab[c] - o->sp[c];
                    if (o->temp[c] <= p->tsolid) {
                        o->su[c] = 0.0;
                        o->an[c] = o->as[c] = o->ae[c] = o->aw[c] = o->at[c] = o->ab[c] = 0.0;
                        o->ap[c] = LARGE;
                    }
                }
        return;
    }
    if (ivar == 6) {  /* calculateSource(6), :1844-1920 */
        fold_and_relax(o, o->conc, p->urfc);
        return;
    }
    if (ivar != 5) return;
    /* volumetric source: scalar form (patched branch of :1698-1705) or the
     * time table, advanced at most one row per call (:1707-1717) */
    double avolfact = p->avolfact, avolpow = p->avolpow, apowseta = p->apowseta,
           heatthick = p->heatthick, heatrb = p->heatrb;
    if (p->nheattable > 0) {
        if (o->timet > o->heattable[6 * o->heat_iter] && o->heat_iter < p->nheattable - 1)
            o->heat_iter += 1;
        const double *row = &o->heattable[6 * o->heat_iter];
        avolpow = row[1];
        apowseta = row[2];
        heatthick = row[3];
        heatrb = row[4];
        avolfact = row[5];
    }
    for (k = 1; k < nkm1; k++)
        for (j = 1; j < njm1; j++)
            for (i = 1; i < nim1; i++) {
                size_t c = ID(i, j, k);
                if (o->z[nkm1] - o->z[k] <= heatthick) {
                    o->sourceinput[c] = avolpow * avolfact / M_PI / (heatrb * heatrb) / heatthick * apowseta *
                        exp(-avolfact / (heatrb * heatrb) *
                            (((o->beamposx - o->x[i]) * (o->beamposx - o->x[i])) +
                             ((o->beamposy - o->y[j]) * (o->beamposy - o->y[j])))) *
                        (double)o->powerindicator;
                    o->su[c] += o->volume[c] * o->sourceinput[c];
                } else {
                    o->sourceinput[c] = 0.0;
                }
                double variable1 = o->hlatnt * o->rho[c] / p->delt;
                double volht = o->volume[c] * variable1;
                o->su[c] -= volht * (o->fracl[c] - o->fraclnot[c]);
                const double *fl = o->fracl, *u = o->uvel, *v = o->vvel, *w = o->wvel;
                double flew = o->areajk[k * nj + j] *
                    (MAXD(u[c], 0.0) * fl[ID(i - 1, j, k)] - MAXD(-u[c], 0.0) * fl[c] +
                     MAXD(-u[ID(i + 1, j, k)], 0.0) * fl[ID(i + 1, j, k)] - MAXD(u[ID(i + 1, j, k)], 0.0) * fl[c]);
                double flns = o->areaik[k * ni + i] *
                    (MAXD(v[c], 0.0) * fl[ID(i, j - 1, k)] - MAXD(-v[c], 0.0) * fl[c] +
                     MAXD(-v[ID(i, j + 1, k)], 0.0) * fl[ID(i, j + 1, k)] - MAXD(v[ID(i, j + 1, k)], 0.0) * fl[c]);
                double fltb = o->areaij[j * ni + i] *
                    (MAXD(w[c], 0.0) * fl[ID(i, j, k - 1)] - MAXD(-w[c], 0.0) * fl[c] +
                     MAXD(-w[ID(i, j, k + 1)], 0.0) * fl[ID(i, j, k + 1)] - MAXD(w[ID(i, j, k + 1)], 0.0) * fl[c]);
                o->su[c] += o->rho[c] * o->hlatnt * (flew + flns + fltb);
            }
    fold_and_relax(o, o->enthalpy, p->urfh);
}

/* ---- calculateResiduals: CFDSolverManager.cpp:1933-2132 --------------------------- */
void orc_residual(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1;
    int i, j, k;
    if (ivar >= 1 && ivar <= 3) {
        const double *phi = ivar == 1 ? o->uvel : ivar == 2 ? o->vvel : o->wvel;
        double sumd = 0.0;
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    double r = o->an[c] * phi[ID(i, j + 1, k)] + o->as[c] * phi[ID(i, j - 1, k)] +
                               o->ae[c] * phi[ID(i + 1, j, k)] + o->aw[c] * phi[ID(i - 1, j, k)] +
                               o->at[c] * phi[ID(i, j, k + 1)] + o->ab[c] * phi[ID(i, j, k - 1)] +
                               o->su[c] - o->ap[c] * phi[c];
                    sumd += fabs(r);
                }
        if (ivar == 1) {
            double umaxt = 0.0;
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++)
                    umaxt = MAXD(umaxt, fabs(o->uvel[ID(i, j, nkm1)]));
            o->refmom = 0.25 * M_PI * (o->width * o->width) * o->p.dens * (umaxt * umaxt);
            o->resoru = sumd / o->refmom;
        } else if (ivar == 2) {
            o->resorv = sumd / o->refmom;
        } else {
            o->resorw = sumd / o->refmom;
        }
        return;
    }
    if (ivar == 4) {
        double denom = 0.0;
        for (k = o->kstat; k < nkm1; k++)
            for (j = o->jstat; j <= o->jend; j++)
                for (i = o->istatp1; i <= o->iendm1; i++) {
                    size_t c = ID(i, j, k);
                    double dtpvar = (fabs(o->uvel[c]) + fabs(o->uvel[ID(i + 1, j, k)])) * o->areajk[k * nj + j] +
                                    (fabs(o->vvel[c]) + fabs(o->vvel[ID(i, j + 1, k)])) * o->areaik[k * ni + i] +
                                    (fabs(o->wvel[c]) + fabs(o->wvel[ID(i, j, k + 1)])) * o->areaij[j * ni + i];
                    denom += 0.5 * fabs(dtpvar);
                }
        denom *= o->p.dens;
        o->resorm /= (denom + SMALL);
        return;
    }
    if (ivar == 5) {
        const double *h = o->enthalpy;
        double sumh = 0.0, sumd = 0.0;
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++)
                for (i = 1; i < nim1; i++) {
                    size_t c = ID(i, j, k);
                    double r = (o->an[c] * h[ID(i, j + 1, k)] + o->as[c] * h[ID(i, j - 1, k)] +
                                o->ae[c] * h[ID(i + 1, j, k)] + o->aw[c] * h[ID(i - 1, j, k)] +
                                o->at[c] * h[ID(i, j, k + 1)] + o->ab[c] * h[ID(i, j, k - 1)] + o->su[c]) /
                                   o->ap[c] - h[c];
                    sumd += fabs(r);
                    sumh += fabs(h[c]);
                }
        o->resorh = sumd / (sumh + SMALL);
    }
    if (ivar == 6) {  /* :2102-2128 */
        const double *cn = o->conc;
        double sumc = 0.0, sumd = 0.0;
        for (k = 1; k < nkm1; k++)
            for (j = 1; j < njm1; j++)
                for (i = 1; i < nim1; i++) {
                    size_t c = ID(i, j, k);
                    double r = (o->an[c] * cn[ID(i, j + 1, k)] + o->as[c] * cn[ID(i, j - 1, k)] +
                                o->ae[c] * cn[ID(i + 1, j, k)] + o->aw[c] * cn[ID(i - 1, j, k)] +
                                o->at[c] * cn[ID(i, j, k + 1)] + o->ab[c] * cn[ID(i, j, k - 1)] + o->su[c]) /
                                   o->ap[c] - cn[c];
                    sumd += fabs(r);
                    sumc += fabs(cn[c]);
                }
        o->resorc = sumd / (sumc + SMALL);
    }
}

/* ---- bareplateMaterialProps: CFDSolverManager.cpp:2137-2189 ----------------------- */
void orc_props(orc *o)
{
    const amcfd_params *p = &o->p;
    size_t n = (size_t)o->ni * o->nj * o->nk;
    for (size_t c = 0; c < n; c++) {
        double t = o->temp[c];
        double diffl = (p->thconla * t + p->thconlb) / p->acpl;
        o->diff[c] = diffl;
        o->rho[c] = p->denl;
        o->vis[c] = p->viscos;
        if (t >= p->tliquid) continue;
        double diffs, rhos = p->dens;
        if (!p->powderbed) {
            diffs = (p->thconsa * (t * t) + p->thconsb * t + p->thconsc) / (p->acpa * t + p->acpb);
        } else {  /* powderMaterialProps, CFDSolverManager.cpp:2236-2252 */
            double cps = p->acpa * t + p->acpb;
            double conds = p->thconsa * (t * t) + p->thconsb * t + p->thconsc;
            double diffp = (p->powderthcona * t + p->powderthconb) / (p->powdercpa * t + p->powdercpb);
            diffs = (1.0 - o->csfrac[c]) * diffp + o->csfrac[c] * conds / cps;
            rhos = (1.0 - o->csfrac[c]) * p->powderden + o->csfrac[c] * p->dens;
        }
        o->diff[c] = diffs;
        o->rho[c] = rhos;
        o->vis[c] = 1e10;
        if (t <= p->tsolid) continue;
        o->diff[c] = o->fracl[c] * diffl + (1.0 - o->fracl[c]) * diffs;
        o->rho[c] = o->fracl[c] * p->denl + (1.0 - o->fracl[c]) * rhos;
        o->vis[c] = p->viscos;
    }
}

/* ---- enhanceConvergenceSpeed(5): CFDSolverManager.cpp:2270-2362 ------------------- */
static void block_correct_phi(orc *o, double *phi)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2;
    double *bl = dalloc(ni), *blp = dalloc(ni), *blm = dalloc(ni), *blc = dalloc(ni);
    double *delphi = dalloc(ni), *pib = dalloc(ni), *qib = dalloc(ni);
    for (int k = 1; k < nkm1; k++)
        for (int j = 1; j < njm1; j++)
            for (int i = 1; i < nim1; i++) {
                size_t c = ID(i, j, k);
                bl[i] += o->ap[c] - o->an[c] - o->as[c] - o->at[c] - o->ab[c];
                blp[i] += o->ae[c];
                blm[i] += o->aw[c];
                blc[i] += o->ae[c] * phi[ID(i + 1, j, k)] + o->aw[c] * phi[ID(i - 1, j, k)] +
                          o->an[c] * phi[ID(i, j + 1, k)] + o->as[c] * phi[ID(i, j - 1, k)] +
                          o->at[c] * phi[ID(i, j, k + 1)] + o->ab[c] * phi[ID(i, j, k - 1)] + o->su[c] -
                          o->ap[c] * phi[c];
            }
    pib[1] = blp[1] / bl[1];
    qib[1] = blc[1] / bl[1];
    for (int i = 2; i < nim1; i++) {
        double denom = bl[i] - blm[i] * pib[i - 1];
        pib[i] = blp[i] / denom;
        qib[i] = (blc[i] + blm[i] * qib[i - 1]) / denom;
    }
    delphi[nim2] = qib[nim2];
    for (int i = nim2 - 1; i > 0; i--) delphi[i] = pib[i] * delphi[i + 1] + qib[i];
    for (int k = 1; k < nkm1; k++)
        for (int j = 1; j < njm1; j++)
            for (int i = 1; i < nim1; i++) phi[ID(i, j, k)] += delphi[i];
    free(bl); free(blp); free(blm); free(blc); free(delphi); free(pib); free(qib);
}
void orc_block_correct(orc *o) { block_correct_phi(o, o->enthalpy); }

/* ---- solveEntireDomain(5): CFDSolverManager.cpp:2459-2526 ------------------------- */
static void solve_entire_phi(orc *o, double *phi)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nim2 = o->nim2, nkm2 = o->nkm2;
    double *pr = dalloc(ni), *qr = dalloc(ni);
    for (int ks = 0; ks < 2; ks++)
        for (int k = nkm2; k > 0; k--)
            for (int js = 0; js < 2; js++)
                for (int j = 1; j < njm1; j++) {
                    pr[0] = 0.0;
                    qr[0] = phi[ID(0, j, k)];
                    for (int i = 1; i < nim1; i++) {
                        size_t c = ID(i, j, k);
                        double d = o->at[c] * phi[ID(i, j, k + 1)] + o->ab[c] * phi[ID(i, j, k - 1)] +
                                   o->an[c] * phi[ID(i, j + 1, k)] + o->as[c] * phi[ID(i, j - 1, k)] + o->su[c];
                        double denom = o->ap[c] - o->aw[c] * pr[i - 1];
                        pr[i] = o->ae[c] / denom;
                        qr[i] = (d + o->aw[c] * qr[i - 1]) / denom;
                    }
                    for (int i = nim2; i > 0; i--) phi[ID(i, j, k)] = pr[i] * phi[ID(i + 1, j, k)] + qr[i];
                }
    free(pr); free(qr);
}
void orc_solve_entire(orc *o) { solve_entire_phi(o, o->enthalpy); }

/* ---- solveLiquidDomain(1..4): CFDSolverManager.cpp:2367-2454 ---------------------- */
void orc_solve_liquid(orc *o, int ivar)
{
    const int ni = o->ni, nj = o->nj, nkm2 = o->nkm2;
    double *phi = ivar == 1 ? o->uvel : ivar == 2 ? o->vvel : ivar == 3 ? o->wvel : o->pp;
    double *pr = dalloc(ni), *qr = dalloc(ni);
    for (int ks = 0; ks < 2; ks++)
        for (int k = nkm2; k >= o->kstat; k--)
            for (int js = 0; js < 2; js++)
                for (int j = o->jstat; j <= o->jend; j++) {
                    pr[o->istat] = 0.0;
                    qr[o->istat] = phi[ID(o->istat, j, k)];
                    for (int i = o->istatp1; i <= o->iendm1; i++) {
                        size_t c = ID(i, j, k);
                        double d = o->at[c] * phi[ID(i, j, k + 1)] + o->ab[c] * phi[ID(i, j, k - 1)] +
                                   o->an[c] * phi[ID(i, j + 1, k)] + o->as[c] * phi[ID(i, j - 1, k)] + o->su[c];
                        double denom = o->ap[c] - o->aw[c] * pr[i - 1];
                        if (fabs(denom) <= 1e-12) denom += SMALL;
                        pr[i] = o->ae[c] / denom;
                        qr[i] = (d + o->aw[c] * qr[i - 1]) / denom;
                    }
                    for (int i = o->iendm1; i >= o->istatp1; i--)
                        phi[ID(i, j, k)] = pr[i] * phi[ID(i + 1, j, k)] + qr[i];
                }
    free(pr); free(qr);
}

/* ---- convertEnthalpyToTemp: CFDSolverManager.cpp:2531-2571 ------------------------ */
void orc_h2t(orc *o)
{
    const amcfd_params *p = &o->p;
    double deltemp = p->tliquid - p->tsolid;
    size_t n = (size_t)o->ni * o->nj * o->nk;
    for (size_t c = 0; c < n; c++) {
        double h = o->enthalpy[c];
        if (h >= o->hlcal) {
            o->fracl[c] = 1.0;
            o->temp[c] = (h - o->hlcal) / p->acpl + p->tliquid;
        } else if (h <= p->hsmelt) {
            o->fracl[c] = 0.0;
            o->temp[c] = (sqrt(p->acpb * p->acpb + 2 * p->acpa * h) - p->acpb) / p->acpa;
        } else {
            o->fracl[c] = (h - p->hsmelt) / (o->hlcal - p->hsmelt);
            o->temp[c] = deltemp * o->fracl[c] + p->tsolid;
        }
    }
}

/* ---- cleanVelocities: CFDSolverManager.cpp:2577-2620 ------------------------------ */
void orc_clean_velocities(orc *o)
{
    const int ni = o->ni, nj = o->nj, nkm1 = o->nkm1;
    const double ts = o->p.tsolid;
    for (int k = o->kstat; k < nkm1; k++)
        for (int j = o->jstat; j <= o->jend; j++)
            for (int i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, k);
                double tulc = MIND(o->temp[c], o->temp[ID(i + 1, j, k)]);
                double tvlc = MIND(o->temp[c], o->temp[ID(i, j + 1, k)]);
                double twlc = MIND(o->temp[c], o->temp[ID(i, j, k + 1)]);
                if (tulc <= ts) o->uvel[ID(i + 1, j, k)] = 0.0;
                if (tvlc <= ts) o->vvel[ID(i, j + 1, k)] = 0.0;
                if (twlc <= ts) o->wvel[ID(i, j, k + 1)] = 0.0;
            }
}

/* ---- correctPressure: CFDSolverManager.cpp:2692-2758 ------------------------------ */
void orc_correct_pressure(orc *o)
{
    const int ni = o->ni, nj = o->nj, nkm1 = o->nkm1;
    const double ts = o->p.tsolid;
    for (int k = o->kstat; k < nkm1; k++)
        for (int j = o->jstat; j <= o->jend; j++)
            for (int i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, k);
                if (MIND(o->temp[c], o->temp[ID(i - 1, j, k)]) > ts)
                    o->uvel[c] += o->dux[c] * (o->pp[ID(i - 1, j, k)] - o->pp[c]);
                if (MIND(o->temp[c], o->temp[ID(i, j - 1, k)]) > ts)
                    o->vvel[c] += o->dvy[c] * (o->pp[ID(i, j - 1, k)] - o->pp[c]);
                if (MIND(o->temp[c], o->temp[ID(i, j, k - 1)]) > ts)
                    o->wvel[c] += o->dwz[c] * (o->pp[ID(i, j, k - 1)] - o->pp[c]);
            }
    for (int k = o->kstat; k < nkm1; k++)
        for (int j = o->jstat; j <= o->jend; j++)
            for (int i = o->istatp1; i <= o->iendm1; i++) {
                size_t c = ID(i, j, k);
                if (o->temp[c] > ts) {
                    o->pressure[c] += o->p.urfp * o->pp[c];
                    o->pp[c] = 0.0;
                }
            }
}

/* ---- calculateFluxes: BoundCondManager.cpp:746-858 -------------------------------- */
void orc_fluxes(orc *o)
{
    const int ni = o->ni, nj = o->nj;
    const int nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1, nim2 = o->nim2, njm2 = o->njm2,
              nkm2 = o->nkm2;
    const double *h = o->enthalpy, *df = o->diff;
    o->fluxwest = o->fluxeast = o->fluxbottom = o->fluxtop = o->fluxnorth = o->fluxsouth = 0.0;
    o->accul = o->heatvol = 0.0;
    for (int k = 1; k < nkm1; k++)
        for (int j = 1; j < njm1; j++) {
            double fi = df[ID(1, j, k)] * (h[ID(0, j, k)] - h[ID(1, j, k)]) * o->dxpwinv[1];
            double fl = df[ID(nim2, j, k)] * (h[ID(nim1, j, k)] - h[ID(nim2, j, k)]) * o->dxpwinv[nim1];
            o->fluxwest += o->areajk[k * nj + j] * fi;
            o->fluxeast += o->areajk[k * nj + j] * fl;
        }
    for (int j = 1; j < njm1; j++)
        for (int i = 1; i < nim1; i++) {
            double fk = df[ID(i, j, 1)] * (h[ID(i, j, 0)] - h[ID(i, j, 1)]) * o->dzpbinv[1];
            double fn = df[ID(i, j, nkm2)] * (h[ID(i, j, nkm1)] - h[ID(i, j, nkm2)]) * o->dzpbinv[nkm1];
            o->fluxbottom += o->areaij[j * ni + i] * fk;
            o->fluxtop += o->areaij[j * ni + i] * fn;
        }
    for (int k = 1; k < nkm1; k++)
        for (int i = 1; i < nim1; i++) {
            double fj = df[ID(i, 1, k)] * (h[ID(i, 0, k)] - h[ID(i, 1, k)]) * o->dypsinv[1];
            double fm = df[ID(i, njm2, k)] * (h[ID(i, njm1, k)] - h[ID(i, njm2, k)]) * o->dypsinv[njm1];
            o->fluxsouth += o->areaik[k * ni + i] * fj;
            o->fluxnorth += o->areaik[k * ni + i] * fm;
        }
    if (!o->p.steady) {
        for (int k = 1; k < nkm1; k++)
            for (int j = 1; j < njm1; j++)
                for (int i = 1; i < nim1; i++) {
                    size_t c = ID(i, j, k);
                    double dh1 = h[c] - o->hnot[c] + (o->fracl[c] - o->fraclnot[c]) * o->hlatnt;
                    o->accul += o->volume[c] * o->rho[c] * dh1 / o->p.delt;
                    o->heatvol += o->sourceinput[c] * o->volume[c];
                }
    }
    o->heatout = (o->fluxnorth + o->fluxbottom + o->fluxwest + o->fluxeast + o->fluxsouth) - o->ahtoploss;
    if (o->p.steady)
        o->ratio = -o->heatout / o->heatinlaser;
    else
        o->ratio = (o->heatvol + o->heatinlaser) / (o->accul - o->heatout);
}

/* ---- updateSolutions: CFDSolverManager.cpp:2625-2687 ------------------------------ */
void orc_update_solutions(orc *o)
{
    size_t n = (size_t)o->ni * o->nj * o->nk;
    /* :2637-2645: track id of the first toolpath row not earlier than the time
     * (undefined in the reference without one; 0 here) */
    const double trackindx = (double)o->trackindx;
    int trackid = 0;
    for (int i = o->p.ntool; i > 0; i--)
        if (o->p.udtoolpath && o->timet <= o->tool[4 * (i - 1)]) trackid = o->tool_id[i - 1];
    for (size_t c = 0; c < n; c++) {
        if (o->temp[c] <= o->p.tsolid) {
            o->uvel[c] = 0.0;
            o->vvel[c] = 0.0;
            o->wvel[c] = 0.0;
        }
        o->unot[c] = o->uvel[c];
        o->vnot[c] = o->vvel[c];
        o->wnot[c] = o->wvel[c];
        o->hnot[c] = o->enthalpy[c];
        o->fraclnot[c] = o->fracl[c];
        if (o->p.powderbed) {  /* :2666-2678 */
            o->csfrac[c] = MAXD(o->csfrac[c], o->fracl[c]);
            o->solfrac[c] = MAXD(o->solfrac[c], o->fracl[c] * trackindx);
            if (o->temp[c] > o->p.tsolid) o->mpphase[c] = trackid;
            if (o->temp[c] > o->p.tliquid) o->mpliq[c] = trackid;
        }
        if (o->p.species) {  /* :2680-2685 */
            o->concnot[c] = o->conc[c];
            o->concn[c] = o->conc[c] / (o->fracl[c] + o->p.kp * (1.0 - o->fracl[c]));
        }
    }
}

/* ---- phase groups used by the tests --------------------------------------------- */
void orc_energy_assemble(orc *o)
{
    orc_apply_bcs(o, 5);
    orc_discretize(o, 5);
    orc_source(o, 5);
}

int orc_momentum(orc *o)
{
    /* iterativeLoopSolve :660-675 */
    if (!(o->tpeak > o->p.tsolid && o->p.navierstokes)) return 0;
    orc_clean_velocities(o);
    for (int ivar = 1; ivar < 5; ivar++) {
        orc_apply_bcs(o, ivar);
        orc_discretize(o, ivar);
        orc_source(o, ivar);
        orc_residual(o, ivar);
        orc_solve_liquid(o, ivar);
        if (ivar == 4) orc_correct_pressure(o);
    }
    o->last_box_cells = (o->iendm1 - o->istatp1 + 1) * (o->jend - o->jstat + 1) * (o->nkm1 - o->kstat);
    return 1;
}

/* ---- moving mesh: generateGrid with !init_ (CFDSolverManager.cpp:72-124, 345-346) and
 * remapSolutions (:2810-3051) ------------------------------------------------------- */
static double interp_ref(double x0, double x1, double y0, double y1, double x)
{
    double yd = y1 - y0, xd = x1 - x0;
    return y0 + (x - x0) * (yd / xd);
}

void orc_move_mesh(orc *o)
{
    amcfd_params *p = &o->p;
    const int ni = o->ni, nj = o->nj, nk = o->nk;
    const double dx = o->beamposx - o->oldbeamposx, dy = o->beamposy - o->oldbeamposy;
    const int dirx = dx < 0 ? -1 : 1, diry = dy < 0 ? -1 : 1;
    const int indx = p->xmoveindex, indy = p->ymoveindex;
    p->xzone[indx - 1] += dx;
    p->xzone[indx + 1] -= dx;
    if (o->steadylength) {
        p->yzone[indy - 1] += dy;
        p->yzone[indy + 1] -= dy;
    } else { /* the reference uses the x zone index here (:111-112) */
        p->yzone[indx - 1] += dy;
        p->yzone[indx + 1] -= dy;
    }
    double *oldx = dalloc(ni), *oldy = dalloc(nj);
    memcpy(oldx, o->x, sizeof(double) * ni);
    memcpy(oldy, o->y, sizeof(double) * nj);
    generate_grid(o);
    double *f[14] = {o->enthalpy, o->hnot, o->temp, o->fracl, o->uvel, o->vvel, o->wvel, o->unot,
                     o->vnot, o->wnot, o->pressure, o->pp, o->conc, o->concnot};
    const int nf = p->species ? 14 : 12;
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj - 1; j++)
            for (int i = 1; i < ni - 1; i++) {
                size_t loc = ID(i, j, k);
                if (fabs(oldx[i] - o->x[i]) > 1e-6)
                    for (int q = 0; q < nf; q++)
                        f[q][loc] = interp_ref(oldx[i], oldx[i + dirx], f[q][loc], f[q][loc + dirx], o->x[i]);
            }
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj - 1; j++)
            for (int i = 1; i < ni - 1; i++) {
                size_t loc = ID(i, j, k);
                if (fabs(oldy[j] - o->y[j]) > 1e-6 && j + diry >= 0)
                    for (int q = 0; q < nf; q++)
                        f[q][loc] = interp_ref(oldy[j], oldy[j + diry], f[q][loc],
                                               f[q][(size_t)((long long)loc + (long long)diry * ni)], o->y[j]);
            }
    free(oldx);
    free(oldy);
}

/* ---- getSolidificationParameters: CFDSolverManager.cpp:2764-2804 ------------------
 * Rows whose front lies at i < 2, on the j = 0 / nj-1 rows or the k = 0 plane are
 * skipped: the reference reads outside its arrays there. */
void orc_solidification(orc *o)
{
    if (o->tpeak <= o->p.tsolid) return;
    const int ni = o->ni, nj = o->nj;
    const double *t = o->temp;
    for (int k = 0; k < o->nkm1; k++)
        for (int j = 0; j < nj; j++)
            for (int i = 0; i < ni; i++) {
                if (t[ID(i, j, k)] >= o->p.tsolid) {
                    if (i >= 2 && j >= 1 && j <= nj - 2 && k >= 1) {
                        double gx = (t[ID(i, j, k)] - t[ID(i - 2, j, k)]) / (o->x[i] - o->x[i - 1]) / 2;
                        double gy = (t[ID(i - 1, j + 1, k)] - t[ID(i - 1, j - 1, k)]) / (o->y[j] - o->y[j - 1]) / 2;
                        double gz = (t[ID(i - 1, j, k + 1)] - t[ID(i - 1, j, k - 1)]) / (o->z[k] - o->z[k - 1]) / 2;
                        size_t c = ID(i - 1, j, k);
                        o->grad[c] = sqrt(gx * gx + gy * gy + gz * gz);
                        o->rate[c] = o->scanvel * gx / o->grad[c];
                    }
                    break;
                }
            }
}

/* ---- energy-balance free surface: FreeSurfaceManager.cpp:74-341 -------------------- */
static void fs_ebal(orc *o, double alambda)
{
    const int ni = o->ni, nj = o->nj, nim1 = o->nim1, njm1 = o->njm1, nkm1 = o->nkm1;
    const amcfd_params *p = &o->p;
    const int nitermax = (int)p->fs_maxiterenergy;
    const double c1 = p->dens * p->grav, gamma = p->fs_surftens, urfree = p->fs_urfree, tol = p->fs_tolenergy;
    const double *x = o->x, *y = o->y, *xu = o->xu, *yv = o->yv;
    double *zzm = o->zzm, *fi = o->fi;
    int niter = 0;
    double difmax = 0.0;  /* not reset per sweep (:262, 298-300) */
    for (int loc = 0; loc < ni * nj; loc++) zzm[loc] = 0.0;
    while (niter < nitermax) {
        niter++;
        /* one thread of the reference's max reduction: a private maximum starting at the
         * lowest double, folded into the shared one after the sweep */
        double priv = -DBL_MAX;
        for (int j = 1; j < njm1; j++)
            for (int i = 1; i < nim1; i++) {
                if (o->temp[ID(i, j, nkm1)] < p->tsolid) continue;
                double dely = yv[j + 1] - yv[j - 1], dely1 = y[j + 1] - y[j - 1];
                double delyp = y[j + 1] - y[j], delym = y[j] - y[j - 1];
                double delx = xu[i + 1] - xu[i - 1], delx1 = x[i + 1] - x[i - 1];
                double delxp = x[i + 1] - x[i], delxm = x[i] - x[i - 1];
                double c2 = 0.0 + alambda; /* apdis = 0 */
                double dzdx = (zzm[j * ni + i + 1] - zzm[j * ni + i - 1]) / delx1;
                double dzdy = (zzm[(j + 1) * ni + i] - zzm[(j - 1) * ni + i]) / dely1;
                double dzdyp1 = (zzm[(j + 1) * ni + i + 1] - zzm[(j - 1) * ni + i + 1]) / dely1;
                double dzdym1 = (zzm[(j + 1) * ni + i - 1] - zzm[(j - 1) * ni + i - 1]) / dely1;
                double d2zdxdy = (dzdyp1 - dzdym1) / delx1;
                double c3 = pow(1.0 + dzdx * dzdx + dzdy * dzdy, 1.5);
                double c4 = 1.0 + dzdy * dzdy, c5 = 1.0 + dzdx * dzdx;
                double c6 = 2.0 * dzdx * dzdy * d2zdxdy;
                double c7 = zzm[j * ni + i + 1] / (delxp * delx) + zzm[j * ni + i - 1] / (delxm * delx);
                double c8 = zzm[(j + 1) * ni + i] / (delyp * dely) + zzm[(j - 1) * ni + i] / (delym * dely);
                double c9 = 1.0 / (delxp * delx) + 1.0 / (delxm * delx);
                double c10 = 1.0 / (delyp * dely) + 1.0 / (delym * dely);
                double c11 = gamma / c3;
                double term1 = c2 + c11 * (c4 * c7 + c5 * c8 - c6);
                double term2 = c1 + c11 * (c4 * c9 + c5 * c10);
                fi[j * ni + i] = urfree * term1 / term2 + (1.0 - urfree) * zzm[j * ni + i];
                double diff1 = fabs((fi[j * ni + i] - zzm[j * ni + i]) / zzm[j * ni + i]);
                priv = (diff1 < priv) ? priv : diff1;  /* std::max(diff1, difmax) */
            }
        difmax = (priv > difmax) ? priv : difmax;
        if (difmax < tol) break;
        for (int loc = 0; loc < ni * nj; loc++) zzm[loc] = fi[loc];
    }
}

static double fs_delta_vol(orc *o, double alambda)
{
    const int ni = o->ni;
    fs_ebal(o, alambda);
    double delv = 0.0;
    for (int j = 1; j < o->njm1; j++)
        for (int i = 1; i < o->nim1; i++) delv += o->areaij[j * ni + i] * o->fi[j * ni + i];
    return delv;
}

void orc_free_surface(orc *o, double *rep /* lambda, residual, fi_min, fi_max, volume, iterations, bracketed */)
{
    const amcfd_params *p = &o->p;
    const int ni = o->ni, nj = o->nj, nk = o->nk, nkm1 = o->nkm1;
    const int nitermax = (int)p->fs_maxiterbisect;
    const double alam1 = p->fs_lam1, alam2 = p->fs_lam2, tol = p->fs_tolbisect, delt = p->delt;
    const double startdeltn = 0.0, vdp = 2e-9;
    double melttime = delt * (1.0 + startdeltn), vd;
    if (o->tpeak <= p->tsolid) {
        vd = 0.0;
        melttime = 0.0;
    } else {
        vd = vdp * (o->timet - melttime - startdeltn * delt);
        if (o->powerindicator < 1) vd = vdp * (p->lasertime - melttime);
    }
    double f = fs_delta_vol(o, alam1) + vd;
    double fmid = fs_delta_vol(o, alam2) + vd;
    int bracketed = !(f * fmid >= 0.0 && f != vd);
    double alamopt, dx, xmid = 0.0;
    if (f < 0.0) { alamopt = alam1; dx = alam2 - alam1; }
    else { alamopt = alam2; dx = alam1 - alam2; }
    int niter;
    for (niter = 0; niter < nitermax; niter++) {
        dx *= 0.5;
        xmid = alamopt + dx;
        fmid = fs_delta_vol(o, xmid) + vd;
        if (fmid < 0.0) alamopt = xmid;
        if (fabs(dx) < 1.0e-5 || (fabs(fmid) < tol && niter != 0)) break;
    }
    for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++)
            for (int i = 0; i < ni; i++) {
                size_t c = ID(i, j, k);
                double factor = o->fi[j * ni + i] / o->z[nkm1];
                o->zr[c] = o->z[k] * (1.0 - factor);
                if (o->zr[c] > o->z[nkm1]) continue;
                if (o->zr[c] == o->z[nkm1]) o->tempr[c] = o->temp[ID(i, j, nkm1)];
                for (int l = nkm1 - 1; l >= 0; l--)
                    if (o->z[l] <= o->zr[c]) {
                        o->tempr[c] = (o->zr[c] - o->z[l]) / (o->z[l + 1] - o->z[l]) *
                                          (o->temp[ID(i, j, l + 1)] - o->temp[ID(i, j, l)]) + o->temp[ID(i, j, l)];
                        break;
                    }
            }
    double mn = o->fi[0], mx = o->fi[0];
    for (int q = 1; q < ni * nj; q++) {
        if (o->fi[q] < mn) mn = o->fi[q];
        if (mx < o->fi[q]) mx = o->fi[q];
    }
    rep[0] = xmid; rep[1] = fmid; rep[2] = mn; rep[3] = mx; rep[4] = vd;
    rep[5] = niter; rep[6] = bracketed;
}

/* Species equation (iterativeLoopSolve :677-687). */
void orc_species(orc *o)
{
    if (!o->p.species) return;
    orc_apply_bcs(o, 6);
    orc_discretize(o, 6);
    orc_source(o, 6);
    orc_residual(o, 6);
    block_correct_phi(o, o->conc);
    solve_entire_phi(o, o->conc);
}

/* One outer iteration (iterativeLoopSolve :612-716); returns 1 when converged. */
int orc_outer_iteration(orc *o)
{
    o->niter++;
    o->itertot++;
    orc_energy_assemble(o);
    orc_residual(o, 5);
    orc_props(o);
    orc_block_correct(o);
    orc_solve_entire(o);
    orc_h2t(o);
    orc_meltpool(o);
    orc_momentum(o);
    orc_species(o);
    double list[5] = {o->resorm, o->resoru, o->resorv, o->resorw, o->resorc};
    double amaxres = list[0];
    for (int q = 1; q < 5; q++)
        if (amaxres < list[q]) amaxres = list[q];
    orc_fluxes(o);
    double ratio = o->ratio, tol = o->p.nonlintol;
    if (o->p.steady) return (ratio <= 1.001 && ratio >= 0.999 && amaxres < tol);
    if (o->powerindicator == 1) return (ratio <= 1.01 && ratio >= 0.99 && amaxres < tol);
    return (o->resorh < 1e-6 && amaxres < tol);
}

void orc_outer_loop(orc *o)
{
    double alenold = o->alen;
    while (o->niter < o->p.maxit)
        if (orc_outer_iteration(o)) return;
    if (fabs(o->alen - alenold) < 1.0e-6) o->steadylength = 1;
}

void orc_report(const orc *o, amcfd_step_report *r)
{
    memset(r, 0, sizeof(*r));
    r->timet = o->timet;
    r->niter = o->niter;
    r->itertot = o->itertot;
    r->resorh = o->resorh; r->resorm = o->resorm; r->resoru = o->resoru;
    r->resorv = o->resorv; r->resorw = o->resorw;
    r->tpeak = o->tpeak; r->alen = o->alen; r->depth = o->depth; r->width = o->width;
    r->ratio = o->ratio; r->heatinlaser = o->heatinlaser; r->ahtoploss = o->ahtoploss;
    r->accul = o->accul; r->heatout = o->heatout; r->heatvol = o->heatvol;
    r->beamposx = o->beamposx; r->beamposy = o->beamposy; r->scanvel = o->scanvel;
    r->istat = o->istat; r->iend = o->iend; r->jstat = o->jstat; r->jend = o->jend;
    r->kstat = o->kstat; r->jstart = o->jstart; r->powerindicator = o->powerindicator;
    r->momentum_cells = o->last_box_cells;
    r->resorc = o->resorc;
    r->nk_active = o->nk;
    r->trackindx = o->trackindx;
    r->steadylength = o->steadylength;
}

/* Start of a time step, main.cpp:125-141: variable time step, timet += delt,
 * updateLaser; resets the outer-iteration counter. */
void orc_begin_step(orc *o)
{
    if (o->p.nvardt > 0) {
        if (o->timet > o->vardt[3 * o->vardt_state] && o->vardt_state < o->p.nvardt - 1)
            o->vardt_state += 1;
        o->p.delt = o->vardt[3 * o->vardt_state + 1];
        o->p.outtime = o->vardt[3 * o->vardt_state + 2];
    }
    o->timet += o->p.delt;
    if (!o->p.steady) orc_update_laser(o);
    o->niter = 0;
}

/* One time step, main.cpp:125-162. */
void orc_step(orc *o, amcfd_step_report *r)
{
    orc_begin_step(o);
    if (o->p.movingmesh) orc_move_mesh(o);    /* main.cpp:144-145 */
    orc_outer_loop(o);
    if (o->p.solidification) orc_solidification(o);  /* :151-152 */
    if (!o->p.steady) orc_update_solutions(o);
    if (r) orc_report(o, r);
}

/* ---- construction --------------------------------------------------------------- */
static int zone_total(int nz, const double *ncv)
{
    int s = 0;
    for (int q = 0; q < nz; q++) s += (int)ncv[q];
    return s;
}

orc *orc_create(const amcfd_params *params)
{
    orc *o = (orc *)calloc(1, sizeof(orc));
    o->p = *params;
    const amcfd_params *p = &o->p;
    if (p->udtoolpath && p->ntool > 0) {
        o->tool = dalloc(4 * (size_t)p->ntool);
        o->tool_on = (int *)calloc(p->ntool, sizeof(int));
        o->tool_id = (int *)calloc(p->ntool, sizeof(int));
        memcpy(o->tool, p->tool_txyz, sizeof(double) * 4 * p->ntool);
        memcpy(o->tool_on, p->tool_on, sizeof(int) * p->ntool);
        memcpy(o->tool_id, p->tool_id, sizeof(int) * p->ntool);
    }
    o->p.tool_txyz = o->tool;
    o->p.tool_on = o->tool_on;
    o->p.tool_id = o->tool_id;
    if (p->nheattable > 0) {
        o->heattable = dalloc(6 * (size_t)p->nheattable);
        memcpy(o->heattable, p->heattable, sizeof(double) * 6 * p->nheattable);
    }
    if (p->nvardt > 0) {
        o->vardt = dalloc(3 * (size_t)p->nvardt);
        memcpy(o->vardt, p->vardt, sizeof(double) * 3 * p->nvardt);
        o->p.delt = o->vardt[1];
        o->p.outtime = o->vardt[2];
    }
    o->p.heattable = o->heattable;
    o->p.vardt = o->vardt;
    o->ni = zone_total(p->nzx, p->ncvx) + 2;
    o->nj = zone_total(p->nzy, p->ncvy) + 2;
    o->nk = zone_total(p->nzz, p->ncvz) + 2;
    o->nim1 = o->ni - 1; o->njm1 = o->nj - 1; o->nkm1 = o->nk - 1;
    o->nim2 = o->ni - 2; o->njm2 = o->nj - 2; o->nkm2 = o->nk - 2;
    double cpavg = (p->acpa * p->tsolid + p->acpb + p->acpl) * 0.5;
    o->hlcal = p->hsmelt + cpavg * (p->tliquid - p->tsolid);
    o->hlatnt = p->hlfriz - o->hlcal;
    o->scanvel = p->scanvel;
    const size_t ni = o->ni, nj = o->nj, nk = o->nk, n = ni * nj * nk;
    o->x = dalloc(ni); o->xu = dalloc(ni); o->dxpwinv = dalloc(ni); o->fracx = dalloc(ni);
    o->y = dalloc(nj); o->yv = dalloc(nj); o->dypsinv = dalloc(nj); o->fracy = dalloc(nj);
    o->z = dalloc(nk); o->zw = dalloc(nk); o->dzpbinv = dalloc(nk); o->fracz = dalloc(nk);
    o->areaij = dalloc(nj * ni); o->areauij = dalloc(nj * ni); o->areavij = dalloc(nj * ni);
    o->areaik = dalloc(nk * ni); o->areawik = dalloc(nk * ni); o->areauik = dalloc(nk * ni);
    o->areajk = dalloc(nk * nj); o->areavjk = dalloc(nk * nj); o->areawjk = dalloc(nk * nj);
    o->heatin = dalloc(nj * ni);
    double **f3[] = {&o->volume, &o->volume_u, &o->volume_v, &o->volume_w, &o->vis, &o->diff,
                     &o->uvel, &o->vvel, &o->wvel, &o->enthalpy, &o->temp, &o->pp, &o->hnot,
                     &o->fracl, &o->fraclnot, &o->sourceinput, &o->rho, &o->unot, &o->vnot,
                     &o->wnot, &o->pressure, &o->ap, &o->an, &o->as, &o->ae, &o->aw, &o->at,
                     &o->ab, &o->apnot, &o->dux, &o->dvy, &o->dwz, &o->su, &o->sp, &o->conc,
                     &o->concnot, &o->concn, &o->csfrac, &o->solfrac, &o->mpphase, &o->mpliq,
                     &o->grad, &o->rate, &o->zr, &o->tempr};
    for (size_t q = 0; q < sizeof(f3) / sizeof(f3[0]); q++) *f3[q] = dalloc(n);
    o->powerindicator = 1;
    o->init = 1;
    o->trackindx = 1;
    o->nk_alloc = o->nk;
    o->fi = dalloc(ni * nj);
    o->zzm = dalloc(ni * nj);
    generate_grid(o);
    initialize_solver(o);
    if (p->freesurface)  /* FreeSurfaceManager::initializeFreeSurface (:34-69) */
        for (size_t c = 0; c < n; c++) {
            o->zr[c] = o->z[c / (ni * nj)];
            o->tempr[c] = o->temp[c];
        }
    if (p->powderbed) {
        /* CFDSolverManager.cpp:482-492 then PrintManager.cpp:67-73: build layers are
         * powder, and only the first of them starts active */
        const double top = o->z[o->nk - 1] - ((double)p->numlayers * p->layerheight);
        for (int k = 0; k < o->nk; k++)
            for (size_t c = (size_t)k * ni * nj; c < (size_t)(k + 1) * ni * nj; c++)
                o->csfrac[c] = o->z[k] < top ? 1.0 : 0.0;
        o->nk -= (p->numlayers - 1) * p->ncvzlayer;
        o->nkm1 = o->nk - 1;
        o->nkm2 = o->nk - 2;
    }
    if (p->steady) orc_update_laser(o);
    return o;
}

void orc_free(orc *o)
{
    if (!o) return;
    double *f[] = {o->tool, o->x, o->xu, o->dxpwinv, o->fracx, o->y, o->yv, o->dypsinv, o->fracy,
                   o->z, o->zw, o->dzpbinv, o->fracz, o->areaij, o->areauij, o->areavij,
                   o->areaik, o->areawik, o->areauik, o->areajk, o->areavjk, o->areawjk,
                   o->heatin, o->volume, o->volume_u, o->volume_v, o->volume_w, o->vis, o->diff,
                   o->uvel, o->vvel, o->wvel, o->enthalpy, o->temp, o->pp, o->hnot, o->fracl,
                   o->fraclnot, o->sourceinput, o->rho, o->unot, o->vnot, o->wnot, o->pressure,
                   o->ap, o->an, o->as, o->ae, o->aw, o->at, o->ab, o->apnot, o->dux, o->dvy,
                   o->dwz, o->su, o->sp, o->conc, o->concnot, o->concn, o->csfrac, o->solfrac,
                   o->mpphase, o->mpliq, o->grad, o->rate, o->zr, o->tempr, o->fi, o->zzm};
    for (size_t q = 0; q < sizeof(f) / sizeof(f[0]); q++) free(f[q]);
    free(o->tool_on);
    free(o->tool_id);
    free(o->heattable);
    free(o->vardt);
    free(o);
}

void orc_dims(const orc *o, int *ni, int *nj, int *nk)
{
    *ni = o->ni; *nj = o->nj; *nk = o->nk_alloc;
}

/* Pointer to a named array inside the oracle state (for the test harness). */
double *orc_field(orc *o, const char *name)
{
    struct { const char *n; double *p; } t[] = {
        {"temp", o->temp}, {"uvel", o->uvel}, {"vvel", o->vvel}, {"wvel", o->wvel},
        {"pressure", o->pressure}, {"pp", o->pp}, {"enthalpy", o->enthalpy}, {"fracl", o->fracl},
        {"fraclnot", o->fraclnot}, {"hnot", o->hnot}, {"diff", o->diff}, {"rho", o->rho},
        {"vis", o->vis}, {"sourceinput", o->sourceinput}, {"unot", o->unot}, {"vnot", o->vnot},
        {"wnot", o->wnot}, {"ap", o->ap}, {"an", o->an}, {"as", o->as}, {"ae", o->ae},
        {"aw", o->aw}, {"at", o->at}, {"ab", o->ab}, {"apnot", o->apnot}, {"su", o->su},
        {"sp", o->sp}, {"dux", o->dux}, {"dvy", o->dvy}, {"dwz", o->dwz},
        {"volume", o->volume}, {"volume_u", o->volume_u}, {"volume_v", o->volume_v},
        {"volume_w", o->volume_w},
        {"x", o->x}, {"y", o->y}, {"z", o->z}, {"xu", o->xu}, {"yv", o->yv}, {"zw", o->zw},
        {"dxpwinv", o->dxpwinv}, {"dypsinv", o->dypsinv}, {"dzpbinv", o->dzpbinv},
        {"fracx", o->fracx}, {"fracy", o->fracy}, {"fracz", o->fracz}, {"heatin", o->heatin},
        {"areaij", o->areaij}, {"areajk", o->areajk}, {"areaik", o->areaik},
        {"avgconcentration", o->conc}, {"avgconcentrationnot", o->concnot},
        {"concentration", o->concn}, {"csfrac", o->csfrac}, {"solfrac", o->solfrac},
        {"mpPhase", o->mpphase}, {"mpLiqPhase", o->mpliq}, {"grad", o->grad}, {"rate", o->rate},
        {"zr", o->zr}, {"tempr", o->tempr}, {"fi", o->fi}};
    for (size_t q = 0; q < sizeof(t) / sizeof(t[0]); q++)
        if (!strcmp(t[q].n, name)) return t[q].p;
    return NULL;
}

/* Scalar state access for the harness (box indices, time, laser). */
void orc_get_state(const orc *o, double *timet, int *box /* istat,iend,jstat,jend,kstat,jstart,istart */)
{
    *timet = o->timet;
    box[0] = o->istat; box[1] = o->iend; box[2] = o->jstat; box[3] = o->jend;
    box[4] = o->kstat; box[5] = o->jstart; box[6] = o->istart;
}
