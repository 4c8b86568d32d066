/* Body of the CPU oracle, instantiated for REAL=float (PW_F32=1, the
 * reference's own float evaluation order) and REAL=double (PW_F32=0, the FP64
 * oracle).  Test infrastructure only -- see pw_oracle.c. */

/* ------------------------------------------------------------------------ */
/* afd: fdm2d / fdm (pywave/src/wave_fdm.c:28-381, 397-686) driven the way    */
/* afd2dc / afd3dc set them up (pywave/src/afd.c:23-314, 316-578).            */
/* ------------------------------------------------------------------------ */

/* dim: 2 or 3.  nz1,nx1,ny1: interior sizes (ny1=1 for 2-D).
 * rick: [ns][nt] source wavelets (forward), dat_in: [ny1][nx1][nt] (TRI).
 * dat_out: [ny1][nx1][nt] receiver traces at interior depth gz (forward).
 * wfd: [ntsnap][ny1][nx1][nz1] snapshots every jsnap steps (or NULL).
 * Returns 0, or -1 on an allocation failure. */
int SFX(or_afd)(int dim, int nz1, int nx1, int ny1, int nbt, float ct, float dt,
                float dz, float dx, float dy, int nt,
                int ns, const int *spz, const int *spx, const int *spy, const REAL *rick,
                int tri, const REAL *dat_in, int jsnap, int gz,
                const REAL *vel, REAL *dat_out, REAL *wfd)
{
    const int three = (dim == 3);
    const int nz = nz1 + 2 * nbt, nx = nx1 + 2 * nbt, ny = three ? ny1 + 2 * nbt : 1;
    const int nz2 = or_pad_first(nz), nx2 = or_next_fast(nx), ny2 = three ? or_next_fast(ny) : 1;
    const size_t n = (size_t)nz * nx * ny, n2 = (size_t)nz2 * nx2 * ny2;
    const size_t sxy = (size_t)nz2 * nx2;
    REAL *vv = (REAL *)calloc(n, sizeof(REAL));
    REAL *curr = (REAL *)calloc(n2, sizeof(REAL));
    REAL *prev = (REAL *)calloc(n2, sizeof(REAL));
    REAL *wave = (REAL *)calloc(n2, sizeof(REAL));
    REAL *w = (REAL *)calloc(nbt > 0 ? nbt : 1, sizeof(REAL));
    if (!vv || !curr || !prev || !wave || !w) return -1;
#if PW_F32
    const float c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;
    const float idz = 1 / (dz * dz), idx = 1 / (dx * dx), idy = 1 / (dy * dy);
#else
    const double c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;
    const double idz = 1 / ((double)dz * dz), idx = 1 / ((double)dx * dx), idy = 1 / ((double)dy * dy);
#endif
    const int gpz = nbt + gz, gpx = nbt, gpy = three ? nbt : 0;

    /* vel_expand (wave_abc.c:14-125): edge replication into the taper */
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++)
            for (int iz = 0; iz < nz; iz++) {
                int jz = iz - nbt, jx = ix - nbt, jy = three ? iy - nbt : 0;
                jz = jz < 0 ? 0 : (jz >= nz1 ? nz1 - 1 : jz);
                jx = jx < 0 ? 0 : (jx >= nx1 ? nx1 - 1 : jx);
                jy = jy < 0 ? 0 : (jy >= ny1 ? ny1 - 1 : jy);
                REAL v = vel[jz + (size_t)nz1 * (jx + (size_t)nx1 * jy)];
                vv[iz + (size_t)nz * (ix + (size_t)nx * iy)] = v * v * (REAL)dt * (REAL)dt;
            }
    /* abc_cal (wave_abc.c:127-145); afd.c forces the same nb and c on all faces */
    for (int ib = 0; ib < nbt; ib++) {
#if PW_F32
        w[ib] = (float)exp(-ct * ct * (nbt - 1 - ib) * (nbt - 1 - ib));
#else
        w[ib] = exp(-(double)ct * ct * (nbt - 1 - ib) * (nbt - 1 - ib));
#endif
    }

    const int it1 = tri ? nt - 1 : 0, it2 = tri ? -1 : nt, its = tri ? -1 : 1;
    for (int it = it1; it != it2; it += its) {
        /* 4th-order Laplacian on [2,n2-2) of the padded grid; border stays 0 */
        for (int iy = (three ? 2 : 0); iy < (three ? ny2 - 2 : 1); iy++)
            for (int ix = 2; ix < nx2 - 2; ix++)
                for (int iz = 2; iz < nz2 - 2; iz++) {
                    size_t j = iz + (size_t)ix * nz2 + iy * sxy;
                    if (three) {
                        wave[j] = c0 * curr[j] * (idy + idx + idz) +
                                  c1 * (curr[j - sxy] + curr[j + sxy]) * idy +
                                  c2 * (curr[j - 2 * sxy] + curr[j + 2 * sxy]) * idy +
                                  c1 * (curr[j - nz2] + curr[j + nz2]) * idx +
                                  c2 * (curr[j - 2 * nz2] + curr[j + 2 * nz2]) * idx +
                                  c1 * (curr[j - 1] + curr[j + 1]) * idz +
                                  c2 * (curr[j - 2] + curr[j + 2]) * idz;
                    } else {
                        wave[j] = c0 * curr[j] * (idx + idz) +
                                  c1 * (curr[j - nz2] + curr[j + nz2]) * idx +
                                  c2 * (curr[j - 2 * nz2] + curr[j + 2 * nz2]) * idx +
                                  c1 * (curr[j - 1] + curr[j + 1]) * idz +
                                  c2 * (curr[j - 2] + curr[j + 2]) * idz;
                    }
                }
        /* leapfrog on the expanded (unpadded) extent */
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++)
                for (int iz = 0; iz < nz; iz++) {
                    size_t i = iz + (size_t)ix * nz + (size_t)iy * nz * nx;
                    size_t j = iz + (size_t)ix * nz2 + iy * sxy;
                    REAL old, c;
                    old = c = curr[j];
                    c += c - prev[j];
                    prev[j] = old;
                    c += wave[j] * vv[i];
                    curr[j] = c;
                }
        if (tri) {
            for (int iy = 0; iy < ny1; iy++)
                for (int ix = 0; ix < nx1; ix++)
                    curr[gpz + (size_t)(ix + gpx) * nz2 + (size_t)(iy + gpy) * sxy] +=
                        vv[gpz + (size_t)(ix + gpx) * nz + (size_t)(iy + gpy) * nz * nx] *
                        dat_in[((size_t)iy * nx1 + ix) * nt + it];
        } else {
            for (int i = 0; i < ns; i++)
                for (int ky = (three ? -1 : 0); ky <= (three ? 1 : 0); ky++)
                    for (int kx = -1; kx <= 1; kx++)
                        for (int kz = -1; kz <= 1; kz++) {
                            int pz = spz[i] + nbt + kz, px = spx[i] + nbt + kx;
                            int py = three ? spy[i] + nbt + ky : 0;
                            size_t ik = pz + (size_t)nz * px + (size_t)nz * nx * py;
                            size_t j = pz + (size_t)nz2 * px + sxy * py;
                            curr[j] += vv[ik] * rick[(size_t)i * nt + it] /
                                       (abs(kx) + abs(ky) + abs(kz) + 1);
                        }
        }
        /* abc_apply (wave_abc.c:203-294) on curr and prev, faces in order
         * top, bottom (from the PADDED end), left x, right x (padded end),
         * left y, right y */
        for (int pass = 0; pass < 2; pass++) {
            REAL *a = pass == 0 ? curr : prev;
            for (int iy = 0; iy < ny2; iy++)
                for (int ix = 0; ix < nx2; ix++)
                    for (int iz = 0; iz < nbt; iz++) a[iz + (size_t)ix * nz2 + iy * sxy] *= w[iz];
            for (int iy = 0; iy < ny2; iy++)
                for (int ix = 0; ix < nx2; ix++)
                    for (int iz = 0; iz < nbt; iz++)
                        a[(nz2 - 1 - iz) + (size_t)ix * nz2 + iy * sxy] *= w[iz];
            for (int iy = 0; iy < ny2; iy++)
                for (int ix = 0; ix < nbt; ix++)
                    for (int iz = 0; iz < nz2; iz++) a[iz + (size_t)ix * nz2 + iy * sxy] *= w[ix];
            for (int iy = 0; iy < ny2; iy++)
                for (int ix = 0; ix < nbt; ix++)
                    for (int iz = 0; iz < nz2; iz++)
                        a[iz + (size_t)(nx2 - 1 - ix) * nz2 + iy * sxy] *= w[ix];
            if (three) {
                for (int iy = 0; iy < nbt; iy++)
                    for (int ix = 0; ix < nx2; ix++)
                        for (int iz = 0; iz < nz2; iz++) a[iz + (size_t)ix * nz2 + iy * sxy] *= w[iy];
                for (int iy = 0; iy < nbt; iy++)
                    for (int ix = 0; ix < nx2; ix++)
                        for (int iz = 0; iz < nz2; iz++)
                            a[iz + (size_t)ix * nz2 + (ny2 - 1 - iy) * sxy] *= w[iy];
            }
        }
        if (!tri && dat_out) {
            for (int iy = 0; iy < ny1; iy++)
                for (int ix = 0; ix < nx1; ix++)
                    dat_out[((size_t)iy * nx1 + ix) * nt + it] =
                        curr[gpz + (size_t)(ix + gpx) * nz2 + (size_t)(iy + gpy) * sxy];
        }
        if (wfd && jsnap > 0 && it % jsnap == 0) {
            REAL *snap = wfd + (size_t)(it / jsnap) * nz1 * nx1 * ny1;
            for (int iy = 0; iy < ny1; iy++)
                for (int ix = 0; ix < nx1; ix++)
                    for (int iz = 0; iz < nz1; iz++)
                        snap[iz + (size_t)nz1 * ix + (size_t)nz1 * nx1 * iy] =
                            curr[iz + nbt + (size_t)(ix + nbt) * nz2 + (size_t)(iy + gpy) * sxy];
        }
    }
    free(vv); free(curr); free(prev); free(wave); free(w);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* pfwi acoustic path (pywave/src/wave_fwiutil.c, wave_fwimodeling.c,         */
/* wave_fwigradient.c).  Padded arrays are [padnx][padnz] (z fastest).        */
/* ------------------------------------------------------------------------ */

/* sponge table of preparation (wave_fwiutil.c:31-36) */
static void SFX(pf_sponge_table)(int nb, float coef, REAL *bc)
{
    for (int i = 0; i < nb; i++) {
#if PW_F32
        float tmp = coef * (nb - i);
        bc[i] = expf(-tmp * tmp);
#else
        double tmp = (double)coef * (nb - i);
        bc[i] = exp(-tmp * tmp);
#endif
    }
}

/* pad2d (wave_fwiutil.c:123-147): edge replication by nb on all sides */
static void SFX(pf_pad)(const REAL *v, REAL *vp, int nz, int nx, int nb)
{
    int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    for (int ix = 0; ix < pnx; ix++)
        for (int iz = 0; iz < pnz; iz++) {
            int jz = iz - nb, jx = ix - nb;
            jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
            jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
            vp[(size_t)ix * pnz + iz] = v[(size_t)jx * nz + jz];
        }
}

/* laplace, 8th order (wave_fwiutil.c:179-199), written on [4,pad-4) only */
static void SFX(pf_laplace)(const REAL *p, REAL *term, int pnx, int pnz, REAL dx2, REAL dz2)
{
#if PW_F32
    const float c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
#else
    const double c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
#endif
    for (int ix = 4; ix < pnx - 4; ix++)
        for (int iz = 4; iz < pnz - 4; iz++) {
            size_t j = (size_t)ix * pnz + iz;
            size_t s = pnz;
            term[j] = (c0 * p[j] + c1 * (p[j + s] + p[j - s]) + c2 * (p[j + 2 * s] + p[j - 2 * s]) +
                       c3 * (p[j + 3 * s] + p[j - 3 * s]) + c4 * (p[j + 4 * s] + p[j - 4 * s])) / dx2 +
                      (c0 * p[j] + c1 * (p[j + 1] + p[j - 1]) + c2 * (p[j + 2] + p[j - 2]) +
                       c3 * (p[j + 3] + p[j - 3]) + c4 * (p[j + 4] + p[j - 4])) / dz2;
        }
}

/* np_butter_apply (wave_butter.c:64-102): in place over one trace, the
 * first-order section first (odd nn), then each second-order section */
static void SFX(pf_butter_apply)(const or_butter_t *bw, int nx, REAL *x)
{
    const REAL d1 = bw->mid;
    const int nn = bw->nn;
    REAL d0, d2, x0 = 0, x1 = 0, x2, y0, y1 = 0, y2 = 0;
    if (nn % 2) {
        d0 = bw->den[nn / 2][0];
        d2 = bw->den[nn / 2][1];
        x0 = y1 = 0;
        for (int ix = 0; ix < nx; ix++) {
            x1 = x0; x0 = x[ix];
            y0 = bw->low ? (x0 + x1 - d2 * y1) * d0 : (x0 - x1 - d2 * y1) * d0;
            x[ix] = y1 = y0;
        }
    }
    for (int j = 0; j < nn / 2; j++) {
        d0 = bw->den[j][0];
        d2 = bw->den[j][1];
        x1 = x0 = y1 = y2 = 0;
        for (int ix = 0; ix < nx; ix++) {
            x2 = x1; x1 = x0; x0 = x[ix];
            y0 = bw->low ? (x0 + 2 * x1 + x2 - d1 * y1 - d2 * y2) * d0
                         : (x0 - 2 * x1 + x2 - d1 * y1 - d2 * y2) * d0;
            y2 = y1; x[ix] = y1 = y0;
        }
    }
}

/* apply, reverse, apply, reverse (wave_fwigradient.c:769-780): zero phase */
static void SFX(pf_butter_zero_phase)(const or_butter_t *bw, int nt, REAL *x)
{
    for (int pass = 0; pass < 2; pass++) {
        SFX(pf_butter_apply)(bw, nt, x);
        for (int i = 0; i < nt / 2; i++) {
            REAL t = x[i]; x[i] = x[nt - 1 - i]; x[nt - 1 - i] = t;
        }
    }
}

void SFX(or_butter_apply)(int low, float cutoff, int nn, int nx, REAL *x)
{
    or_butter_t bw;
    or_butter_init(&bw, low, cutoff, nn);
    SFX(pf_butter_apply)(&bw, nx, x);
}

/* apply_sponge (wave_fwiutil.c:201-223): top, bottom per column, then left,
 * right per row */
static void SFX(pf_apply_sponge)(REAL *p, const REAL *bc, int pnx, int pnz, int nb)
{
    for (int ix = 0; ix < pnx; ix++) {
        for (int iz = 0; iz < nb; iz++) p[(size_t)ix * pnz + iz] = bc[iz] * p[(size_t)ix * pnz + iz];
        for (int iz = pnz - nb; iz < pnz; iz++)
            p[(size_t)ix * pnz + iz] = bc[pnz - iz - 1] * p[(size_t)ix * pnz + iz];
    }
    for (int iz = 0; iz < pnz; iz++) {
        for (int ix = 0; ix < nb; ix++) p[(size_t)ix * pnz + iz] = bc[ix] * p[(size_t)ix * pnz + iz];
        for (int ix = pnx - nb; ix < pnx; ix++)
            p[(size_t)ix * pnz + iz] = bc[pnx - ix - 1] * p[(size_t)ix * pnz + iz];
    }
}

/* source_map (wave_fwiutil.c:149-177) with rect 2x2 as pfwi.c:822-823 sets */
static void SFX(pf_source_map)(int sx, int sz, int pnx, int pnz, REAL *rr)
{
    float *f = (float *)calloc((size_t)pnx * pnz, sizeof(float));
    f[(size_t)sx * pnz + sz] = 1.f;
    or_smooth2d(2, 2, pnz, pnx, f);
    for (size_t i = 0; i < (size_t)pnx * pnz; i++) rr[i] = f[i];
    free(f);
}

/* One leapfrog step of the pfwi scheme: p2 = 2 p1 - p0 + v^2 dt^2 term
 * (wave_fwimodeling.c:92-96), then rotate and sponge p0 and p1
 * (:99-103).  Arrays rotate through the three pointers. */
static void SFX(pf_update_in)(REAL **p0, REAL **p1, REAL **p2, const REAL *vp, const REAL *term,
                              REAL dt2, const REAL *bc, int pnx, int pnz, int nb, int inner)
{
    size_t np = (size_t)pnx * pnz;
    if (inner) {  /* gradient_pas_av (wave_fwigradient.c:740-745): [4, pad-4) only */
        for (int ix = 4; ix < pnx - 4; ix++)
            for (int iz = 4; iz < pnz - 4; iz++) {
                size_t j = (size_t)ix * pnz + iz;
                (*p2)[j] = 2 * (*p1)[j] - (*p0)[j] + vp[j] * vp[j] * dt2 * term[j];
            }
    } else {
        for (size_t j = 0; j < np; j++)
            (*p2)[j] = 2 * (*p1)[j] - (*p0)[j] + vp[j] * vp[j] * dt2 * term[j];
    }
    REAL *t = *p0; *p0 = *p1; *p1 = *p2; *p2 = t;
    SFX(pf_apply_sponge)(*p0, bc, pnx, pnz, nb);
    SFX(pf_apply_sponge)(*p1, bc, pnx, pnz, nb);
}

static void SFX(pf_update)(REAL **p0, REAL **p1, REAL **p2, const REAL *vp, const REAL *term,
                           REAL dt2, const REAL *bc, int pnx, int pnz, int nb)
{
    SFX(pf_update_in)(p0, p1, p2, vp, term, dt2, bc, pnx, pnz, nb, 0);
}

/* forward_modeling_a (wave_fwimodeling.c:21-114).
 * vel: [nx][nz]; wav: [nt]; data: [ns][nr][nt].
 * Geometry (preparation, wave_fwiutil.c:44-71) is passed in resolved:
 * sx[is] (padded index), sz, rz (padded), receivers rx = r0v[is]+ir*drv for
 * ir < nr2[is], written to trace r02[is]+ir. */
void SFX(or_pfwi_forward)(int nz, int nx, int nb, float dz, float dx, int nt, float dt, float coef,
                          int ns, const int *sx, int sz, int nr, const int *r0v, const int *r02,
                          const int *nr2, int drv, int rz,
                          const REAL *vel, const REAL *wav, REAL *data)
{
    const int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    const size_t np = (size_t)pnz * pnx;
    REAL *vp = (REAL *)calloc(np, sizeof(REAL)), *rr = (REAL *)calloc(np, sizeof(REAL));
    REAL *a = (REAL *)calloc(np, sizeof(REAL)), *b = (REAL *)calloc(np, sizeof(REAL));
    REAL *c = (REAL *)calloc(np, sizeof(REAL)), *term = (REAL *)calloc(np, sizeof(REAL));
    REAL *bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    const REAL dx2 = (REAL)dx * dx, dz2 = (REAL)dz * dz, dt2 = (REAL)dt * dt;
    SFX(pf_sponge_table)(nb, coef, bc);
    SFX(pf_pad)(vel, vp, nz, nx, nb);
    for (int is = 0; is < ns; is++) {
        REAL *p0 = a, *p1 = b, *p2 = c;
        memset(p0, 0, np * sizeof(REAL)); memset(p1, 0, np * sizeof(REAL)); memset(p2, 0, np * sizeof(REAL));
        REAL *dd = data + (size_t)is * nr * nt;
        memset(dd, 0, (size_t)nr * nt * sizeof(REAL));
        SFX(pf_source_map)(sx[is], sz, pnx, pnz, rr);
        for (int it = 0; it < nt; it++) {
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                dd[(size_t)(r02[is] + ir) * nt + it] = p1[(size_t)rx * pnz + rz];
            }
            SFX(pf_laplace)(p1, term, pnx, pnz, dx2, dz2);
            for (size_t j = 0; j < np; j++) term[j] += rr[j] * wav[it];
            SFX(pf_update)(&p0, &p1, &p2, vp, term, dt2, bc, pnx, pnz, nb);
        }
        a = p0; b = p1; c = p2;
    }
    free(vp); free(rr); free(a); free(b); free(c); free(term); free(bc);
}

/* gradient_av (wave_fwigradient.c:93-242), raw: before the first-call
 * scaling and gradient_smooth2 (:244-255).  weight: [nr][nt] residual
 * weights (residual_weighting).  grad: [nx][nz] (zeroed here).  Returns the
 * misfit 0.5*sum((dobs-d)^2), accumulated as the reference does. */
static REAL SFX(pf_gradient_core)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                                  float coef, int interval,
                                  int ns, const int *sx, int sz, int nr, const int *r0v,
                                  const int *r02, const int *nr2, int drv, int rz,
                                  const REAL *vel, const REAL *wav, const REAL *dsrc,
                                  const REAL *dobs, const REAL *weight, REAL *grad,
                                  const or_butter_t *blo, const or_butter_t *bhi)
{
    const int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    const size_t np = (size_t)pnz * pnx, nzx = (size_t)nz * nx;
    const int wnt = (nt - 1) / interval + 1;
    REAL *vp = (REAL *)calloc(np, sizeof(REAL)), *rr = (REAL *)calloc(np, sizeof(REAL));
    REAL *a = (REAL *)calloc(np, sizeof(REAL)), *b = (REAL *)calloc(np, sizeof(REAL));
    REAL *c = (REAL *)calloc(np, sizeof(REAL)), *term = (REAL *)calloc(np, sizeof(REAL));
    REAL *bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    REAL *wave = (REAL *)calloc(nzx * wnt, sizeof(REAL));
    REAL *pp = (REAL *)calloc((size_t)nr * nt, sizeof(REAL));
    const REAL dx2 = (REAL)dx * dx, dz2 = (REAL)dz * dz, dt2 = (REAL)dt * dt;
#if PW_F32
    float wdt = dt * interval, wdt2 = wdt * wdt;
    float fcost = 0.;
#else
    double wdt = (double)dt * interval, wdt2 = wdt * wdt;
    double fcost = 0.;
#endif
    SFX(pf_sponge_table)(nb, coef, bc);
    SFX(pf_pad)(vel, vp, nz, nx, nb);
    memset(grad, 0, nzx * sizeof(REAL));
    for (int is = 0; is < ns; is++) {
        REAL *p0 = a, *p1 = b, *p2 = c;
        memset(p0, 0, np * sizeof(REAL)); memset(p1, 0, np * sizeof(REAL)); memset(p2, 0, np * sizeof(REAL));
        memset(pp, 0, (size_t)nr * nt * sizeof(REAL));
        if (!dsrc) SFX(pf_source_map)(sx[is], sz, pnx, pnz, rr);
        int wit = 0;
        for (int it = 0; it < nt; it++) {
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                pp[(size_t)(r02[is] + ir) * nt + it] = p1[(size_t)rx * pnz + rz];
            }
            if (it % interval == 0) {
                for (int ix = 0; ix < nx; ix++)
                    for (int iz = 0; iz < nz; iz++)
                        wave[(size_t)wit * nzx + (size_t)ix * nz + iz] = p1[(size_t)(ix + nb) * pnz + iz + nb];
                wit++;
            }
            SFX(pf_laplace)(p1, term, pnx, pnz, dx2, dz2);
            if (dsrc) {  /* gradient_pas_av (wave_fwigradient.c:732-737) */
                const REAL *w3 = dsrc + ((size_t)is * nt + it) * nzx;
                for (int ix = 0; ix < nx; ix++)
                    for (int iz = 0; iz < nz; iz++)
                        term[(size_t)(ix + nb) * pnz + iz + nb] += w3[(size_t)ix * nz + iz];
            } else {
                for (size_t j = 0; j < np; j++) term[j] += rr[j] * wav[it];
            }
            SFX(pf_update_in)(&p0, &p1, &p2, vp, term, dt2, bc, pnx, pnz, nb, dsrc != NULL);
        }
        wit--;
        const REAL *dd = dobs + (size_t)is * nr * nt;
        for (int ir = 0; ir < nr; ir++)
            for (int it = 0; it < nt; it++) {
                size_t k = (size_t)ir * nt + it;
                pp[k] = dd[k] - pp[k];
                fcost += 0.5 * pp[k] * pp[k];
            }
        for (int ir = 0; ir < nr; ir++) {  /* multiscale (wave_fwigradient.c:767-780) */
            if (blo) SFX(pf_butter_zero_phase)(blo, nt, pp + (size_t)ir * nt);
            if (bhi) SFX(pf_butter_zero_phase)(bhi, nt, pp + (size_t)ir * nt);
        }
        for (size_t k = 0; k < (size_t)nr * nt; k++) pp[k] *= weight[k];
        memset(p0, 0, np * sizeof(REAL)); memset(p1, 0, np * sizeof(REAL)); memset(p2, 0, np * sizeof(REAL));
        memset(term, 0, np * sizeof(REAL));
        for (int it = nt - 1; it >= 0; it--) {
            SFX(pf_laplace)(p1, term, pnx, pnz, dx2, dz2);
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                term[(size_t)rx * pnz + rz] += pp[(size_t)(r02[is] + ir) * nt + it];
            }
            if (dsrc) {  /* gradient_pas_av (:812-817): [4, pad-4) only */
                for (int ix = 4; ix < pnx - 4; ix++)
                    for (int iz = 4; iz < pnz - 4; iz++) {
                        size_t j = (size_t)ix * pnz + iz;
                        p2[j] = 2 * p1[j] - p0[j] + vp[j] * vp[j] * dt2 * term[j];
                    }
            } else {
                size_t npp = np;
                for (size_t j = 0; j < npp; j++)
                    p2[j] = 2 * p1[j] - p0[j] + vp[j] * vp[j] * dt2 * term[j];
            }
            if (it % interval == 0) {
                if (wit != wnt - 1 && wit != 0) {
                    for (int ix = 0; ix < nx; ix++)
                        for (int iz = 0; iz < nz; iz++) {
                            size_t k = (size_t)ix * nz + iz;
                            REAL temp = vp[(size_t)(ix + nb) * pnz + iz + nb];
                            temp = temp * temp * temp;
                            temp = -2. / temp;
                            grad[k] += (wave[(size_t)(wit + 1) * nzx + k] - 2. * wave[(size_t)wit * nzx + k] +
                                        wave[(size_t)(wit - 1) * nzx + k]) / wdt2 *
                                       p1[(size_t)(ix + nb) * pnz + iz + nb] * temp;
                        }
                }
                wit--;
            }
            REAL *t = p0; p0 = p1; p1 = p2; p2 = t;
            SFX(pf_apply_sponge)(p0, bc, pnx, pnz, nb);
            SFX(pf_apply_sponge)(p1, bc, pnx, pnz, nb);
        }
        a = p0; b = p1; c = p2;
    }
    free(vp); free(rr); free(a); free(b); free(c); free(term); free(bc); free(wave); free(pp);
    return fcost;
}

REAL SFX(or_pfwi_gradient_ref)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                               float coef, int interval,
                               int ns, const int *sx, int sz, int nr, const int *r0v,
                               const int *r02, const int *nr2, int drv, int rz,
                               const REAL *vel, const REAL *wav, const REAL *dobs,
                               const REAL *weight, REAL *grad)
{
    return SFX(pf_gradient_core)(nz, nx, nb, dz, dx, nt, dt, coef, interval, ns, sx, sz, nr, r0v,
                                 r02, nr2, drv, rz, vel, wav, NULL, dobs, weight, grad, NULL,
                                 NULL);
}

/* gradient_pas_av (wave_fwigradient.c:667-852) as pfwic sets it up
 * (gradient_pas_init :528-663 with onlyvel: source weight gwt = 1, no
 * multiscale filter): gradient_av with the source field dsrc
 * [ns][nt][nx][nz] added to the interior's term and the update restricted to
 * [4, pad-4).  Raw, before the scaling and gradient_smooth2b (waterz =
 * waterzb = 0, the same smoothing as gradient_smooth2 with waterz 0).
 * flo, fhi: the multiscale cutoffs in Hz (soupar, scaled by dt in
 * preparation); the residual is filtered by a 3-pole zero-phase high-pass
 * when flo*dt > 0.0001 and low-pass when fhi*dt < 0.4999
 * (gradient_pas_init :657-658).  pfwic passes flo 0, fhi 0.5/dt: no filter. */
REAL SFX(or_pfwi_gradient_pas)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                               float coef, int interval, int ns, int nr, const int *r0v,
                               const int *r02, const int *nr2, int drv, int rz,
                               const REAL *vel, const REAL *dsrc, const REAL *dobs,
                               const REAL *weight, REAL *grad, float flo, float fhi)
{
    or_butter_t lo, hi;
    const float flo_dt = flo * dt, fhi_dt = fhi * dt;
    const int use_lo = flo_dt > 0.0001, use_hi = fhi_dt < 0.5 - 0.0001;
    if (use_lo) or_butter_init(&lo, 0, flo_dt, 3);
    if (use_hi) or_butter_init(&hi, 1, fhi_dt, 3);
    return SFX(pf_gradient_core)(nz, nx, nb, dz, dx, nt, dt, coef, interval, ns, NULL, 0, nr, r0v,
                                 r02, nr2, drv, rz, vel, NULL, dsrc, dobs, weight, grad,
                                 use_lo ? &lo : NULL, use_hi ? &hi : NULL);
}

/* preparation's attenuation parameters (wave_fwiutil.c:90-96): tmp =
 * sqrt(q^2+1), taue = (tmp+1)/(2 pi f0 q), taus = (tmp-1)/(2 pi f0 q),
 * tau = taue/taus - 1; the float instance keeps the reference's float /
 * double mix. */
static void SFX(pf_tau)(const REAL *q, size_t n, float f0, REAL *tau, REAL *taus)
{
    const double pi = 3.14159265358979323846264338328;
    for (size_t i = 0; i < n; i++) {
#if PW_F32
        float tmp = sqrtf(q[i] * q[i] + 1);
        float taue = (tmp + 1) / (2. * pi * f0 * q[i]);
        taus[i] = (tmp - 1) / (2. * pi * f0 * q[i]);
        tau[i] = taue / taus[i] - 1;
#else
        double tmp = sqrt(q[i] * q[i] + 1);
        double taue = (tmp + 1) / (2. * pi * f0 * q[i]);
        taus[i] = (tmp - 1) / (2. * pi * f0 * q[i]);
        tau[i] = taue / taus[i] - 1;
#endif
    }
}

/* One visco-acoustic step of forward_modeling (wave_fwimodeling.c:187-205;
 * whole padded grid, term persisting where laplace does not write) or of
 * gradient_v's forward pass (wave_fwigradient.c:334-345; [4, pad-4) only):
 * memory variable r2 from term and r1, term corrected, then the pfwi
 * update; rotate p and r; sponge p0, p1, r1. */
static void SFX(pf_visco_step)(REAL **p0, REAL **p1, REAL **p2, REAL **r1, REAL **r2,
                               REAL *term, const REAL *vp, const REAL *tau, const REAL *taus,
                               const REAL *rr, REAL wv, REAL dt2, REAL idt, const REAL *bc,
                               int pnx, int pnz, int nb, int inner)
{
    const int lo = inner ? 4 : 0;
    for (int ix = lo; ix < pnx - lo; ix++)
        for (int iz = lo; iz < pnz - lo; iz++) {
            size_t j = (size_t)ix * pnz + iz;
            (*r2)[j] = (tau[j] / taus[j] * term[j] + (idt - 0.5 / taus[j]) * (*r1)[j]) /
                       (idt + 0.5 / taus[j]);
            term[j] = term[j] * (1. + tau[j]) - ((*r2)[j] + (*r1)[j]) * 0.5 + rr[j] * wv;
            (*p2)[j] = 2 * (*p1)[j] - (*p0)[j] + vp[j] * vp[j] * dt2 * term[j];
        }
    REAL *t = *p0; *p0 = *p1; *p1 = *p2; *p2 = t;
    t = *r1; *r1 = *r2; *r2 = t;
    SFX(pf_apply_sponge)(*p0, bc, pnx, pnz, nb);
    SFX(pf_apply_sponge)(*p1, bc, pnx, pnz, nb);
    SFX(pf_apply_sponge)(*r1, bc, pnx, pnz, nb);
}

/* forward_modeling, visco-acoustic (wave_fwimodeling.c:116-220); q [nx][nz]
 * quality factor, f0 reference frequency; other arguments as
 * or_pfwi_forward. */
void SFX(or_pfwi_forward_visco)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                                float coef, float f0, int ns, const int *sx, int sz, int nr,
                                const int *r0v, const int *r02, const int *nr2, int drv, int rz,
                                const REAL *vel, const REAL *q, const REAL *wav, REAL *data)
{
    const int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    const size_t np = (size_t)pnz * pnx, nzx = (size_t)nz * nx;
    REAL *vp = (REAL *)calloc(np, sizeof(REAL)), *rr = (REAL *)calloc(np, sizeof(REAL));
    REAL *tp = (REAL *)calloc(np, sizeof(REAL)), *tsp = (REAL *)calloc(np, sizeof(REAL));
    REAL *t1 = (REAL *)calloc(nzx, sizeof(REAL)), *ts1 = (REAL *)calloc(nzx, sizeof(REAL));
    REAL *buf[5], *term = (REAL *)calloc(np, sizeof(REAL));
    for (int i = 0; i < 5; i++) buf[i] = (REAL *)calloc(np, sizeof(REAL));
    REAL *bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    const REAL dx2 = (REAL)dx * dx, dz2 = (REAL)dz * dz, dt2 = (REAL)dt * dt;
#if PW_F32
    const float idt = 1. / dt;
#else
    const double idt = 1. / (double)dt;
#endif
    SFX(pf_sponge_table)(nb, coef, bc);
    SFX(pf_pad)(vel, vp, nz, nx, nb);
    SFX(pf_tau)(q, nzx, f0, t1, ts1);
    SFX(pf_pad)(t1, tp, nz, nx, nb);
    SFX(pf_pad)(ts1, tsp, nz, nx, nb);
    for (int is = 0; is < ns; is++) {
        REAL *p0 = buf[0], *p1 = buf[1], *p2 = buf[2], *r1 = buf[3], *r2 = buf[4];
        for (int i = 0; i < 5; i++) memset(buf[i], 0, np * sizeof(REAL));
        REAL *dd = data + (size_t)is * nr * nt;
        memset(dd, 0, (size_t)nr * nt * sizeof(REAL));
        SFX(pf_source_map)(sx[is], sz, pnx, pnz, rr);
        for (int it = 0; it < nt; it++) {
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                dd[(size_t)(r02[is] + ir) * nt + it] = p1[(size_t)rx * pnz + rz];
            }
            SFX(pf_laplace)(p1, term, pnx, pnz, dx2, dz2);
            SFX(pf_visco_step)(&p0, &p1, &p2, &r1, &r2, term, vp, tp, tsp, rr, wav[it], dt2, idt,
                               bc, pnx, pnz, nb, 0);
        }
    }
    for (int i = 0; i < 5; i++) free(buf[i]);
    free(vp); free(rr); free(tp); free(tsp); free(t1); free(ts1); free(term); free(bc);
}

/* gradient_v (wave_fwigradient.c:264-452), raw: before the first-call
 * scaling and gradient_smooth2.  Forward: pf_visco_step on [4, pad-4) with
 * snapshots; residual and misfit as gradient_av; backward: r2 and tmp =
 * p1 (1 + tau) - 0.5 (r2 + r1) from p1 and r1, term = laplace(tmp) plus the
 * residual, the pfwi update, gradient_av's imaging; rotate; sponge. */
REAL SFX(or_pfwi_gradient_visco)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                                 float coef, float f0, int interval, int ns, const int *sx, int sz,
                                 int nr, const int *r0v, const int *r02, const int *nr2, int drv,
                                 int rz, const REAL *vel, const REAL *q, const REAL *wav,
                                 const REAL *dobs, const REAL *weight, REAL *grad)
{
    const int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    const size_t np = (size_t)pnz * pnx, nzx = (size_t)nz * nx;
    const int wnt = (nt - 1) / interval + 1;
    REAL *vp = (REAL *)calloc(np, sizeof(REAL)), *rr = (REAL *)calloc(np, sizeof(REAL));
    REAL *tp = (REAL *)calloc(np, sizeof(REAL)), *tsp = (REAL *)calloc(np, sizeof(REAL));
    REAL *t1 = (REAL *)calloc(nzx, sizeof(REAL)), *ts1 = (REAL *)calloc(nzx, sizeof(REAL));
    REAL *buf[5], *term = (REAL *)calloc(np, sizeof(REAL)), *tmp = (REAL *)calloc(np, sizeof(REAL));
    for (int i = 0; i < 5; i++) buf[i] = (REAL *)calloc(np, sizeof(REAL));
    REAL *bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    REAL *wave = (REAL *)calloc(nzx * wnt, sizeof(REAL));
    REAL *pp = (REAL *)calloc((size_t)nr * nt, sizeof(REAL));
    const REAL dx2 = (REAL)dx * dx, dz2 = (REAL)dz * dz, dt2 = (REAL)dt * dt;
#if PW_F32
    const float idt = 1. / dt;
    float wdt = dt * interval, wdt2 = wdt * wdt;
    float fcost = 0.;
#else
    const double idt = 1. / (double)dt;
    double wdt = (double)dt * interval, wdt2 = wdt * wdt;
    double fcost = 0.;
#endif
    SFX(pf_sponge_table)(nb, coef, bc);
    SFX(pf_pad)(vel, vp, nz, nx, nb);
    SFX(pf_tau)(q, nzx, f0, t1, ts1);
    SFX(pf_pad)(t1, tp, nz, nx, nb);
    SFX(pf_pad)(ts1, tsp, nz, nx, nb);
    memset(grad, 0, nzx * sizeof(REAL));
    for (int is = 0; is < ns; is++) {
        REAL *p0 = buf[0], *p1 = buf[1], *p2 = buf[2], *r1 = buf[3], *r2 = buf[4];
        for (int i = 0; i < 5; i++) memset(buf[i], 0, np * sizeof(REAL));
        memset(pp, 0, (size_t)nr * nt * sizeof(REAL));
        memset(term, 0, np * sizeof(REAL));
        memset(tmp, 0, np * sizeof(REAL));
        SFX(pf_source_map)(sx[is], sz, pnx, pnz, rr);
        int wit = 0;
        for (int it = 0; it < nt; it++) {
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                pp[(size_t)(r02[is] + ir) * nt + it] = p1[(size_t)rx * pnz + rz];
            }
            if (it % interval == 0) {
                for (int ix = 0; ix < nx; ix++)
                    for (int iz = 0; iz < nz; iz++)
                        wave[(size_t)wit * nzx + (size_t)ix * nz + iz] = p1[(size_t)(ix + nb) * pnz + iz + nb];
                wit++;
            }
            SFX(pf_laplace)(p1, term, pnx, pnz, dx2, dz2);
            SFX(pf_visco_step)(&p0, &p1, &p2, &r1, &r2, term, vp, tp, tsp, rr, wav[it], dt2, idt,
                               bc, pnx, pnz, nb, 1);
        }
        wit--;
        const REAL *dd = dobs + (size_t)is * nr * nt;
        for (int ir = 0; ir < nr; ir++)
            for (int it = 0; it < nt; it++) {
                size_t k = (size_t)ir * nt + it;
                pp[k] = dd[k] - pp[k];
                fcost += 0.5 * pp[k] * pp[k];
                pp[k] *= weight[k];
            }
        for (int i = 0; i < 5; i++) memset(buf[i], 0, np * sizeof(REAL));
        p0 = buf[0]; p1 = buf[1]; p2 = buf[2]; r1 = buf[3]; r2 = buf[4];
        memset(term, 0, np * sizeof(REAL));
        memset(tmp, 0, np * sizeof(REAL));
        for (int it = nt - 1; it >= 0; it--) {
            for (int ix = 4; ix < pnx - 4; ix++)
                for (int iz = 4; iz < pnz - 4; iz++) {
                    size_t j = (size_t)ix * pnz + iz;
                    r2[j] = (-tp[j] / tsp[j] * p1[j] + (-idt + 0.5 / tsp[j]) * r1[j]) /
                            (-idt - 0.5 / tsp[j]);
                    tmp[j] = p1[j] * (1. + tp[j]) - 0.5 * (r2[j] + r1[j]);
                }
            SFX(pf_laplace)(tmp, term, pnx, pnz, dx2, dz2);
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                term[(size_t)rx * pnz + rz] += pp[(size_t)(r02[is] + ir) * nt + it];
            }
            for (int ix = 4; ix < pnx - 4; ix++)
                for (int iz = 4; iz < pnz - 4; iz++) {
                    size_t j = (size_t)ix * pnz + iz;
                    p2[j] = 2 * p1[j] - p0[j] + vp[j] * vp[j] * dt2 * term[j];
                }
            if (it % interval == 0) {
                if (wit != wnt - 1 && wit != 0) {
                    for (int ix = 0; ix < nx; ix++)
                        for (int iz = 0; iz < nz; iz++) {
                            size_t k = (size_t)ix * nz + iz;
                            REAL temp = vp[(size_t)(ix + nb) * pnz + iz + nb];
                            temp = temp * temp * temp;
                            temp = -2. / temp;
                            grad[k] += (wave[(size_t)(wit + 1) * nzx + k] - 2. * wave[(size_t)wit * nzx + k] +
                                        wave[(size_t)(wit - 1) * nzx + k]) / wdt2 *
                                       p1[(size_t)(ix + nb) * pnz + iz + nb] * temp;
                        }
                }
                wit--;
            }
            REAL *t = p0; p0 = p1; p1 = p2; p2 = t;
            t = r1; r1 = r2; r2 = t;
            SFX(pf_apply_sponge)(p0, bc, pnx, pnz, nb);
            SFX(pf_apply_sponge)(p1, bc, pnx, pnz, nb);
            SFX(pf_apply_sponge)(r1, bc, pnx, pnz, nb);
        }
    }
    for (int i = 0; i < 5; i++) free(buf[i]);
    free(vp); free(rr); free(tp); free(tsp); free(t1); free(ts1); free(term); free(tmp); free(bc);
    free(wave); free(pp);
    return fcost;
}

/* Exact discrete adjoint of the pfwi forward scheme.
 *
 * Forward (n = 0..nt-1), a_0 = b_0 = 0, S the sponge, V = v_pad^2 dt^2:
 *   q_n = 2 a_n - b_n + V (L a_n + r w_n),  a_{n+1} = S q_n,  b_{n+1} = S a_n,
 *   d_n = R a_n (traces recorded before the step, as the reference does).
 * Misfit J = sum_s 0.5 * sum_{r,n} W (d - dobs)^2  (W = 1 when weight NULL).
 * Adjoint, phi_n = V * S * dJ/da_{n+1} (phi_{nt-1} = phi_nt = 0):
 *   phi_{n-1} = S (2 phi_n - S phi_{n+1} + V (L phi_n + R^T rho_n)),
 *   rho_n = W (d_n - dobs_n),
 * which is the forward recurrence run backwards with the residual injected.
 * Gradient: dJ/dV = sum_n (phi_n / V) (L a_n + r w_n), dJ/dv_pad = dJ/dV *
 * 2 v dt^2, folded back through pad2d's edge replication.
 * Stores the whole forward history: small cases only.  Returns J. */
REAL SFX(or_pfwi_gradient_exact)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                                 float coef, int ns, const int *sx, int sz, int nr,
                                 const int *r0v, const int *r02, const int *nr2, int drv, int rz,
                                 const REAL *vel, const REAL *wav, const REAL *dobs,
                                 const REAL *weight, REAL *grad)
{
    const int pnz = nz + 2 * nb, pnx = nx + 2 * nb;
    const size_t np = (size_t)pnz * pnx, nzx = (size_t)nz * nx;
    REAL *vp = (REAL *)calloc(np, sizeof(REAL)), *rr = (REAL *)calloc(np, sizeof(REAL));
    REAL *bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    REAL *S = (REAL *)calloc(np, sizeof(REAL)), *V = (REAL *)calloc(np, sizeof(REAL));
    REAL *hist = (REAL *)calloc(np * (size_t)(nt + 1), sizeof(REAL));
    REAL *bprev = (REAL *)calloc(np, sizeof(REAL)), *q = (REAL *)calloc(np, sizeof(REAL));
    REAL *lap = (REAL *)calloc(np, sizeof(REAL)), *gV = (REAL *)calloc(np, sizeof(REAL));
    REAL *phi0 = (REAL *)calloc(np, sizeof(REAL)), *phi1 = (REAL *)calloc(np, sizeof(REAL));
    REAL *phim = (REAL *)calloc(np, sizeof(REAL));
    REAL *d = (REAL *)calloc((size_t)nr * nt, sizeof(REAL));
    const REAL dx2 = (REAL)dx * dx, dz2 = (REAL)dz * dz, dt2 = (REAL)dt * dt;
    REAL J = 0;
    SFX(pf_sponge_table)(nb, coef, bc);
    SFX(pf_pad)(vel, vp, nz, nx, nb);
    for (int ix = 0; ix < pnx; ix++)
        for (int iz = 0; iz < pnz; iz++) {
            REAL s = 1;
            if (iz < nb) s = bc[iz] * s;
            if (iz >= pnz - nb) s = bc[pnz - iz - 1] * s;
            if (ix < nb) s = bc[ix] * s;
            if (ix >= pnx - nb) s = bc[pnx - ix - 1] * s;
            S[(size_t)ix * pnz + iz] = s;
            V[(size_t)ix * pnz + iz] = vp[(size_t)ix * pnz + iz] * vp[(size_t)ix * pnz + iz] * dt2;
        }
    for (size_t j = 0; j < np; j++) gV[j] = 0;
    for (int is = 0; is < ns; is++) {
        SFX(pf_source_map)(sx[is], sz, pnx, pnz, rr);
        memset(hist, 0, np * sizeof(REAL));
        memset(bprev, 0, np * sizeof(REAL));
        memset(d, 0, (size_t)nr * nt * sizeof(REAL));
        for (int n = 0; n < nt; n++) {
            REAL *an = hist + (size_t)n * np, *an1 = hist + (size_t)(n + 1) * np;
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                d[(size_t)(r02[is] + ir) * nt + n] = an[(size_t)rx * pnz + rz];
            }
            memset(lap, 0, np * sizeof(REAL));
            SFX(pf_laplace)(an, lap, pnx, pnz, dx2, dz2);
            for (size_t j = 0; j < np; j++) {
                REAL qj = 2 * an[j] - bprev[j] + V[j] * (lap[j] + rr[j] * wav[n]);
                an1[j] = S[j] * qj;
                bprev[j] = S[j] * an[j];
            }
        }
        const REAL *dd = dobs + (size_t)is * nr * nt;
        for (size_t k = 0; k < (size_t)nr * nt; k++) {
            REAL r = d[k] - dd[k];
            REAL w = weight ? weight[k] : 1;
            J += 0.5 * w * r * r;
            d[k] = w * r; /* d now holds rho */
        }
        /* phi1 = phi_n, phi0 = phi_{n+1} */
        memset(phi0, 0, np * sizeof(REAL));
        memset(phi1, 0, np * sizeof(REAL));
        for (int n = nt - 1; n >= 0; n--) {
            const REAL *an = hist + (size_t)n * np;
            memset(lap, 0, np * sizeof(REAL));
            SFX(pf_laplace)(an, lap, pnx, pnz, dx2, dz2);
            for (size_t j = 0; j < np; j++) gV[j] += phi1[j] / V[j] * (lap[j] + rr[j] * wav[n]);
            memset(lap, 0, np * sizeof(REAL));
            SFX(pf_laplace)(phi1, lap, pnx, pnz, dx2, dz2);
            for (int ir = 0; ir < nr2[is]; ir++) {
                int rx = r0v[is] + ir * drv;
                lap[(size_t)rx * pnz + rz] += d[(size_t)(r02[is] + ir) * nt + n];
            }
            for (size_t j = 0; j < np; j++)
                phim[j] = S[j] * (2 * phi1[j] - S[j] * phi0[j] + V[j] * lap[j]);
            REAL *t = phi0; phi0 = phi1; phi1 = phim; phim = t;
        }
    }
    memset(grad, 0, nzx * sizeof(REAL));
    for (int ix = 0; ix < pnx; ix++)
        for (int iz = 0; iz < pnz; iz++) {
            int jz = iz - nb, jx = ix - nb;
            jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
            jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
            size_t j = (size_t)ix * pnz + iz;
            grad[(size_t)jx * nz + jz] += gV[j] * 2 * vp[j] * dt2;
        }
    free(vp); free(rr); free(bc); free(S); free(V); free(hist); free(bprev); free(q);
    free(lap); free(gV); free(phi0); free(phi1); free(phim); free(d);
    return J;
}

/* Misfit J of or_pfwi_gradient_exact without the gradient (for finite
 * differences). */
REAL SFX(or_pfwi_misfit)(int nz, int nx, int nb, float dz, float dx, int nt, float dt,
                         float coef, int ns, const int *sx, int sz, int nr,
                         const int *r0v, const int *r02, const int *nr2, int drv, int rz,
                         const REAL *vel, const REAL *wav, const REAL *dobs, const REAL *weight)
{
    REAL *d = (REAL *)calloc((size_t)ns * nr * nt, sizeof(REAL));
    SFX(or_pfwi_forward)(nz, nx, nb, dz, dx, nt, dt, coef, ns, sx, sz, nr, r0v, r02, nr2, drv, rz,
                         vel, wav, d);
    REAL J = 0;
    for (size_t k = 0; k < (size_t)ns * nr * nt; k++) {
        REAL r = d[k] - dobs[k];
        REAL w = weight ? weight[k % ((size_t)nr * nt)] : 1;
        J += 0.5 * w * r * r;
    }
    free(d);
    return J;
}
