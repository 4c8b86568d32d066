/* Passive mode 4 of pfwi (lstric): the time-reversal modelling operator and
 * the least-squares source inversion by conjugate gradients.  Test
 * infrastructure only -- see pw_oracle.c.  Instantiated for REAL=float
 * (PW_F32=1: the reference's float evaluation order, operation by
 * operation, no contraction) and REAL=double (the FP64 oracle).
 *
 * Restates:
 *   timerev_init / timerev_lop   pywave/src/wave_triutil.c:48-180
 *     padded grid nzpad = nz + 2 nb, nxpad = nx + 2 nb, z fastest;
 *     vvpad = (v v) dt^2, the interior replicated onto every face;
 *     three fields rotated by pointer; on [4, pad - 4) of both axes
 *       u2 = Lap(u1) + 2 u1 - u0, Lap = ((Sx) / dx^2 + (Sz) / dz^2) vvpad
 *       (modelling) or LapT, where every neighbour carries its own vvpad
 *       (adjoint), S the 8th-order sum c4 (a+4 + a-4) + c3 (..) + c2 (..)
 *       + c1 (..) + c0 a in that order (wave_triutil.h:7-32);
 *     modelling: record row rz+nb of u1, step, rotate, add mod[it] vvpad on
 *       the interior, sponge u0 then u1;
 *     adjoint: sponge u1 then u0, image mod[it] += u1 vvpad, step, rotate,
 *       add dat[:, it] on row rz+nb;
 *   pfwiabc_apply / pfwiabc_cal  wave_triutil.c:264-316
 *     z faces then x faces (corners twice), decay[ib] = exp(-c^2 (nb-1-ib)^2)
 *     with the exponent formed in float and exp taken in double;
 *   lstri / lstri_op             wave_fwi.c:121-175, wave_fwigradient.c:454-520
 *   np_solver (mwt = 1, no x0)   wave_bigsolver.c:1170-1430
 *   np_cgstep                    wave_cgstep.c:16-67; its step vectors S, Ss
 *     are reset only at the first call, so later shots of one call start
 *     from the previous shot's S and Ss (the reference keeps them in statics
 *     for the whole process; here they live for one call);
 *   cblas_dsdot / snrm2 / sscal / saxpy  wave_blas.c:3-88 (snrm2 is the
 *     float sum of squares, without a square root).
 * Arrays: vel [nx][nz]; mod / src [nt][nx][nz] per shot; dat [nx][nt]. */

typedef struct SFX(trg) {
    int nz, nx, nt, nb, nzpad, nxpad, depth;
    REAL sx, sz;
    REAL *vvpad, *decay, *u0, *u1, *u2;
} SFX(trg);

#if PW_F32
#define TR_C0 (-205.0f / 72.0f)
#define TR_C1 (+8.0f / 5.0f)
#define TR_C2 (-1.0f / 5.0f)
#define TR_C3 (+8.0f / 315.0f)
#define TR_C4 (-1.0f / 560.0f)
#else
#define TR_C0 (-205.0 / 72.0)
#define TR_C1 (+8.0 / 5.0)
#define TR_C2 (-1.0 / 5.0)
#define TR_C3 (+8.0 / 315.0)
#define TR_C4 (-1.0 / 560.0)
#endif

static void SFX(tr_setup)(SFX(trg) *g, int nz, int nx, int nt, int nb, int rz, float dt, float dx,
                          float dz, float coef, const float *vel)
{
    g->nz = nz; g->nx = nx; g->nt = nt; g->nb = nb;
    g->nzpad = nz + 2 * nb; g->nxpad = nx + 2 * nb; g->depth = rz + nb;
#if PW_F32
    const float dt2 = dt * dt;
    g->sx = 1.0f / (dx * dx);
    g->sz = 1.0f / (dz * dz);
#else
    const double dt2 = (double)dt * dt;
    g->sx = 1.0 / ((double)dx * dx);
    g->sz = 1.0 / ((double)dz * dz);
#endif
    const size_t np = (size_t)g->nzpad * g->nxpad;
    g->vvpad = (REAL *)calloc(np, sizeof(REAL));
    g->u0 = (REAL *)calloc(np, sizeof(REAL));
    g->u1 = (REAL *)calloc(np, sizeof(REAL));
    g->u2 = (REAL *)calloc(np, sizeof(REAL));
    g->decay = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    for (int ix = 0; ix < g->nxpad; ix++) {
        int jx = ix - nb;
        jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
        for (int iz = 0; iz < g->nzpad; iz++) {
            int jz = iz - nb;
            jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
            const REAL v = vel[(size_t)jx * nz + jz];
            g->vvpad[(size_t)ix * g->nzpad + iz] = v * v * dt2;
        }
    }
    for (int ib = 0; ib < nb; ib++) {
#if PW_F32
        const float e = -coef * coef * (float)(nb - 1 - ib) * (float)(nb - 1 - ib);
        g->decay[ib] = (float)exp((double)e);
#else
        const double e = -(double)coef * coef * (double)(nb - 1 - ib) * (double)(nb - 1 - ib);
        g->decay[ib] = exp(e);
#endif
    }
}

static void SFX(tr_free)(SFX(trg) *g)
{
    free(g->vvpad); free(g->u0); free(g->u1); free(g->u2); free(g->decay);
}

static void SFX(tr_sponge)(const SFX(trg) *g, REAL *a)
{
    const int nzp = g->nzpad, nxp = g->nxpad, nb = g->nb;
    for (int iz = 0; iz < nb; iz++)
        for (int ix = 0; ix < nxp; ix++) {
            a[(size_t)nzp * ix + iz] *= g->decay[iz];
            a[(size_t)nzp * ix + nzp - 1 - iz] *= g->decay[iz];
        }
    for (int iz = 0; iz < nzp; iz++)
        for (int ix = 0; ix < nb; ix++) {
            a[(size_t)nzp * ix + iz] *= g->decay[ix];
            a[(size_t)nzp * (nxp - 1 - ix) + iz] *= g->decay[ix];
        }
}

/* one side of the 8th-order sum along stride st, optionally weighting every
 * sample by vvpad (LapT) */
static inline REAL SFX(tr_sum)(const REAL *a, const REAL *v, ptrdiff_t c, ptrdiff_t st, int wt)
{
#define TRA(k) (wt ? a[c + (k) * st] * v[c + (k) * st] : a[c + (k) * st])
    REAL s = TR_C4 * (TRA(4) + TRA(-4));
    s = s + TR_C3 * (TRA(3) + TRA(-3));
    s = s + TR_C2 * (TRA(2) + TRA(-2));
    s = s + TR_C1 * (TRA(1) + TRA(-1));
    s = s + TR_C0 * (TRA(0));
#undef TRA
    return s;
}

static void SFX(tr_step)(SFX(trg) *g, int adj)
{
    const int nzp = g->nzpad, nxp = g->nxpad;
    const REAL *u0 = g->u0, *u1 = g->u1, *v = g->vvpad;
    REAL *u2 = g->u2;
    for (int ix = 4; ix < nxp - 4; ix++)
        for (int iz = 4; iz < nzp - 4; iz++) {
            const ptrdiff_t c = (ptrdiff_t)ix * nzp + iz;
            REAL lap;
            if (adj)
                lap = SFX(tr_sum)(u1, v, c, nzp, 1) * g->sx + SFX(tr_sum)(u1, v, c, 1, 1) * g->sz;
            else
                lap = (SFX(tr_sum)(u1, v, c, nzp, 0) * g->sx + SFX(tr_sum)(u1, v, c, 1, 0) * g->sz)
                      * v[c];
            u2[c] = lap + (REAL)2 * u1[c] - u0[c];
        }
    REAL *t = g->u0;
    g->u0 = g->u1; g->u1 = g->u2; g->u2 = t;
}

/* timerev_lop with add = false: adj = 0 fills dat [nx][nt] from mod
 * [nt][nx][nz]; adj = 1 fills mod from dat. */
static void SFX(tr_lop)(SFX(trg) *g, int adj, REAL *mod, REAL *dat)
{
    const int nz = g->nz, nx = g->nx, nt = g->nt, nb = g->nb, nzp = g->nzpad;
    const size_t np = (size_t)nzp * g->nxpad;
    if (adj) memset(mod, 0, (size_t)nz * nx * nt * sizeof(REAL));
    else memset(dat, 0, (size_t)nx * nt * sizeof(REAL));
    memset(g->u0, 0, np * sizeof(REAL));
    memset(g->u1, 0, np * sizeof(REAL));
    memset(g->u2, 0, np * sizeof(REAL));
    if (adj) {
        for (int it = nt - 1; it >= 0; it--) {
            SFX(tr_sponge)(g, g->u1);
            SFX(tr_sponge)(g, g->u0);
            for (int ix = 0; ix < nx; ix++)
                for (int iz = 0; iz < nz; iz++) {
                    const size_t c = (size_t)(ix + nb) * nzp + iz + nb;
                    mod[((size_t)it * nx + ix) * nz + iz] += g->u1[c] * g->vvpad[c];
                }
            SFX(tr_step)(g, 1);
            for (int ix = nb; ix < nb + nx; ix++)
                g->u1[(size_t)ix * nzp + g->depth] += dat[(size_t)(ix - nb) * nt + it];
        }
    } else {
        for (int it = 0; it < nt; it++) {
            for (int ix = nb; ix < nb + nx; ix++)
                dat[(size_t)(ix - nb) * nt + it] += g->u1[(size_t)ix * nzp + g->depth];
            SFX(tr_step)(g, 0);
            for (int ix = 0; ix < nx; ix++)
                for (int iz = 0; iz < nz; iz++) {
                    const size_t c = (size_t)(ix + nb) * nzp + iz + nb;
                    g->u1[c] += mod[((size_t)it * nx + ix) * nz + iz] * g->vvpad[c];
                }
            SFX(tr_sponge)(g, g->u0);
            SFX(tr_sponge)(g, g->u1);
        }
    }
}

/* cblas_dsdot / cblas_snrm2 of wave_blas.c: sequential sums */
static double SFX(tr_dsdot)(size_t n, const REAL *x, const REAL *y)
{
    double d = 0.;
    for (size_t i = 0; i < n; i++) d += (double)x[i] * y[i];
    return d;
}
static REAL SFX(tr_snrm2)(size_t n, const REAL *x)
{
    REAL s = 0;
    for (size_t i = 0; i < n; i++) s += x[i] * x[i];
    return s;
}

typedef struct SFX(trcg) {
    int allocated;
    REAL *S, *Ss;
} SFX(trcg);

static void SFX(tr_cgstep)(SFX(trcg) *cg, int forget, size_t nm, size_t nd, REAL *x, const REAL *g,
                           REAL *rr, const REAL *gg)
{
    const double EPS = (double)1.e-12f;
    double sds, gdg, gds, determ, gdr, sdr, alfa, beta;
    if (!cg->allocated) {
        cg->allocated = forget = 1;
        cg->S = (REAL *)calloc(nm, sizeof(REAL));
        cg->Ss = (REAL *)calloc(nd, sizeof(REAL));
    }
    REAL *S = cg->S, *Ss = cg->Ss;
    if (forget) {
        for (size_t i = 0; i < nm; i++) S[i] = 0;
        for (size_t i = 0; i < nd; i++) Ss[i] = 0;
        beta = 0.0;
        alfa = SFX(tr_dsdot)(nd, gg, gg);
        if (alfa <= 0.) return;
        alfa = -SFX(tr_dsdot)(nd, gg, rr) / alfa;
    } else {
        gdg = SFX(tr_dsdot)(nd, gg, gg);
        sds = SFX(tr_dsdot)(nd, Ss, Ss);
        gds = SFX(tr_dsdot)(nd, gg, Ss);
        if (gdg == 0. || sds == 0.) return;
        determ = 1.0 - (gds / gdg) * (gds / sds);
        if (determ > EPS) determ *= gdg * sds;
        else determ = gdg * sds * EPS;
        gdr = -SFX(tr_dsdot)(nd, gg, rr);
        sdr = -SFX(tr_dsdot)(nd, Ss, rr);
        alfa = (sds * gdr - gds * sdr) / determ;
        beta = (-gds * gdr + gdg * sdr) / determ;
    }
    const REAL b = (REAL)beta, a = (REAL)alfa;
    for (size_t i = 0; i < nm; i++) S[i] *= b;
    for (size_t i = 0; i < nm; i++) S[i] += a * g[i];
    for (size_t i = 0; i < nd; i++) Ss[i] *= b;
    for (size_t i = 0; i < nd; i++) Ss[i] += a * gg[i];
    for (size_t i = 0; i < nm; i++) x[i] += S[i];
    for (size_t i = 0; i < nd; i++) rr[i] += Ss[i];
}

/* np_solver(timerev_lop, np_cgstep, ..., "mwt", ones): x [nt][nx][nz] from
 * dat [nx][nt]; returns the number of iterations run */
static int SFX(tr_solve)(SFX(trg) *g, SFX(trcg) *cg, REAL *x, const REAL *dat, int niter)
{
    const float TOL = 1.e-12f;
    const size_t nm = (size_t)g->nz * g->nx * g->nt, nd = (size_t)g->nx * g->nt;
    REAL *gv = (REAL *)calloc(nm, sizeof(REAL));
    REAL *rr = (REAL *)calloc(nd, sizeof(REAL));
    REAL *gg = (REAL *)calloc(nd, sizeof(REAL));
    for (size_t i = 0; i < nd; i++) rr[i] = -dat[i];
    for (size_t i = 0; i < nm; i++) x[i] = 0;
    REAL dpr0 = SFX(tr_snrm2)(nd, rr), dpg0 = 1, dpr, dpg;
    int iter;
    for (iter = 0; iter < niter; iter++) {
        SFX(tr_lop)(g, 1, gv, rr);
        SFX(tr_lop)(g, 0, gv, gg);
        if (iter == 0) {
            dpg0 = SFX(tr_snrm2)(nm, gv);
            dpr = 1;
            dpg = 1;
        } else {
            dpr = SFX(tr_snrm2)(nd, rr) / dpr0;
            dpg = SFX(tr_snrm2)(nm, gv) / dpg0;
        }
        if (dpr < TOL || dpg < TOL) break;
        SFX(tr_cgstep)(cg, 0, nm, nd, x, gv, rr, gg);
    }
    free(gv); free(rr); free(gg);
    return iter;
}

/* lstri (wave_fwi.c:121): inv = 0 fills data [ns][nx][nt] from src
 * [ns][nt][nx][nz]; inv = 1 fills src from data, niter CG iterations per
 * shot.  iters (optional, inv = 1) receives each shot's iteration count. */
void SFX(or_lstri)(int inv, int nz, int nx, int nt, int ns, int nb, int rz, float dt, float dx,
                   float dz, float coef, int niter, const float *vel, REAL *src, REAL *data,
                   int *iters)
{
    SFX(trg) g;
    SFX(tr_setup)(&g, nz, nx, nt, nb, rz, dt, dx, dz, coef, vel);
    SFX(trcg) cg = {0, NULL, NULL};
    const size_t nm = (size_t)nz * nx * nt, nd = (size_t)nx * nt;
    for (int is = 0; is < ns; is++) {
        if (inv) {
            const int n = SFX(tr_solve)(&g, &cg, src + is * nm, data + is * nd, niter);
            if (iters) iters[is] = n;
        } else {
            SFX(tr_lop)(&g, 0, src + is * nm, data + is * nd);
        }
    }
    free(cg.S); free(cg.Ss);
    SFX(tr_free)(&g);
}

/* one application of timerev_lop (add = false) for the operator tests */
void SFX(or_timerev)(int adj, int nz, int nx, int nt, int nb, int rz, float dt, float dx, float dz,
                     float coef, const float *vel, REAL *mod, REAL *dat)
{
    SFX(trg) g;
    SFX(tr_setup)(&g, nz, nx, nt, nb, rz, dt, dx, dz, coef, vel);
    SFX(tr_lop)(&g, adj, mod, dat);
    SFX(tr_free)(&g);
}

#undef TR_C0
#undef TR_C1
#undef TR_C2
#undef TR_C3
#undef TR_C4
