/* 3-D extension of the pfwi scheme: forward modelling, misfit and the exact
 * discrete adjoint gradient.  Test infrastructure only -- see pw_oracle.c.
 * Instantiated for REAL=float (PW_F32=1: the operation order of the 3-D GPU
 * step kernel, operation by operation, no contraction) and REAL=double (the
 * FP64 oracle).
 *
 * The reference has no 3-D FWI; this restates its 2-D acoustic scheme
 * (wave_fwimodeling.c:21-114, wave_fwiutil.c:19-223, checked bit-exactly in
 * 2-D by tests/test_oracle_golden.py) on three axes:
 *   term = (Tx / dx^2 + Tz / dz^2) + Ty / dy^2 + r w_n, each T the 8th-order
 *          sum c0 u + c1 (u+1 + u-1) + ... + c4 (u+4 + u-4) of
 *          wave_fwiutil.c:17,179-199, zero outside [4, pad-4) on every axis,
 *          the divisions as products with 1/h^2 rounded to REAL;
 *   a_{n+1} = S (2 a_n - S a_{n-1} + V term),  V = (v v) dt^2,
 *   S = Sy (Sx (Sz u)) with the sponge factors bc[i] = exp(-(coef (nb-i))^2)
 *       of each face (wave_fwiutil.c:31-36,201-223);
 *   velocity padded by edge replication on every face (pad2d, :123-147);
 *   source: a unit spike at (sz, sx, sy) smoothed by the triangle of rect 2
 *       along z and x (np_smooth2, as source_map does in 2-D) and along y;
 *   receivers at depth rz on the grid (rx[i], ry[j]), traces recorded before
 *       the step, trace index j * nrx + i.
 * Arrays: vel [ny][nx][nz]; data [ns][nry * nrx][nt]; grad [ny][nx][nz]. */

typedef struct SFX(pf3g) {
    int nz, nx, ny, nb, pnz, pnx, pny;
    size_t np;
    REAL rdz2, rdx2, rdy2, dt2;
    REAL *bc, *V, *vp;
} SFX(pf3g);

static void SFX(pf3_setup)(SFX(pf3g) *g, int nz, int nx, int ny, int nb, float dz, float dx,
                           float dy, float dt, float coef, const REAL *vel)
{
    g->nz = nz; g->nx = nx; g->ny = ny; g->nb = nb;
    g->pnz = nz + 2 * nb; g->pnx = nx + 2 * nb; g->pny = ny + 2 * nb;
    g->np = (size_t)g->pnz * g->pnx * g->pny;
#if PW_F32
    g->rdz2 = 1.f / (dz * dz); g->rdx2 = 1.f / (dx * dx); g->rdy2 = 1.f / (dy * dy);
    g->dt2 = dt * dt;
#else
    g->rdz2 = 1. / ((double)dz * dz); g->rdx2 = 1. / ((double)dx * dx);
    g->rdy2 = 1. / ((double)dy * dy); g->dt2 = (double)dt * dt;
#endif
    g->bc = (REAL *)calloc(nb > 0 ? nb : 1, sizeof(REAL));
    SFX(pf_sponge_table)(nb, coef, g->bc);
    g->vp = (REAL *)calloc(g->np, sizeof(REAL));
    g->V = (REAL *)calloc(g->np, sizeof(REAL));
    for (int iy = 0; iy < g->pny; iy++)
        for (int ix = 0; ix < g->pnx; ix++)
            for (int iz = 0; iz < g->pnz; iz++) {
                int jz = iz - nb, jx = ix - nb, jy = iy - nb;
                jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
                jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
                jy = jy < 0 ? 0 : (jy >= ny ? ny - 1 : jy);
                size_t j = ((size_t)iy * g->pnx + ix) * g->pnz + iz;
                REAL v = vel[((size_t)jy * nx + jx) * nz + jz];
                g->vp[j] = v;
                g->V[j] = (v * v) * g->dt2;
            }
}

static void SFX(pf3_free)(SFX(pf3g) *g)
{
    free(g->bc); free(g->vp); free(g->V);
}

/* sponge factor of one axis at index i of a padded extent n */
static REAL SFX(pf3_b)(const SFX(pf3g) *g, int i, int n)
{
    if (i < g->nb) return g->bc[i];
    if (i >= n - g->nb) return g->bc[n - i - 1];
    return 1;
}

static REAL SFX(pf3_sponge)(const SFX(pf3g) *g, int iz, int ix, int iy, REAL u)
{
    REAL bz = SFX(pf3_b)(g, iz, g->pnz), bx = SFX(pf3_b)(g, ix, g->pnx);
    REAL by = SFX(pf3_b)(g, iy, g->pny);
    return by * (bx * (bz * u));
}

/* 8th-order Laplacian on [4, pad-4) along every axis, 0 elsewhere */
static void SFX(pf3_laplace)(const SFX(pf3g) *g, const REAL *p, REAL *term)
{
#if PW_F32
    const float c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
#else
    const double c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
#endif
    const int pnz = g->pnz, pnx = g->pnx, pny = g->pny;
    const size_t sz = 1, sx = pnz, sy = (size_t)pnz * pnx;
    memset(term, 0, g->np * sizeof(REAL));
    for (int iy = 4; iy < pny - 4; iy++)
        for (int ix = 4; ix < pnx - 4; ix++)
            for (int iz = 4; iz < pnz - 4; iz++) {
                size_t j = ((size_t)iy * pnx + ix) * pnz + iz;
                REAL cv = p[j];
                REAL tx = c0 * cv;
                tx = tx + c1 * (p[j + sx] + p[j - sx]);
                tx = tx + c2 * (p[j + 2 * sx] + p[j - 2 * sx]);
                tx = tx + c3 * (p[j + 3 * sx] + p[j - 3 * sx]);
                tx = tx + c4 * (p[j + 4 * sx] + p[j - 4 * sx]);
                REAL tz = c0 * cv;
                tz = tz + c1 * (p[j + sz] + p[j - sz]);
                tz = tz + c2 * (p[j + 2 * sz] + p[j - 2 * sz]);
                tz = tz + c3 * (p[j + 3 * sz] + p[j - 3 * sz]);
                tz = tz + c4 * (p[j + 4 * sz] + p[j - 4 * sz]);
                REAL ty = c0 * cv;
                ty = ty + c1 * (p[j + sy] + p[j - sy]);
                ty = ty + c2 * (p[j + 2 * sy] + p[j - 2 * sy]);
                ty = ty + c3 * (p[j + 3 * sy] + p[j - 3 * sy]);
                ty = ty + c4 * (p[j + 4 * sy] + p[j - 4 * sy]);
                term[j] = (tx * g->rdx2 + tz * g->rdz2) + ty * g->rdy2;
            }
}

/* source map: spike at padded (sz, sx, sy) smoothed (triangle, rect 2) in
 * z and x by or_smooth2d and in y by the same smoothing of a line */
static void SFX(pf3_source_map)(const SFX(pf3g) *g, int sz, int sx, int sy, REAL *rr)
{
    const int pnz = g->pnz, pnx = g->pnx, pny = g->pny;
    float *f = (float *)calloc((size_t)pnz * pnx, sizeof(float));
    float *fy = (float *)calloc((size_t)pny, sizeof(float));
    f[(size_t)sx * pnz + sz] = 1.f;
    or_smooth2d(2, 2, pnz, pnx, f);
    fy[sy] = 1.f;
    or_smooth2d(2, 1, pny, 1, fy);
    for (int iy = 0; iy < pny; iy++)
        for (int ix = 0; ix < pnx; ix++)
            for (int iz = 0; iz < pnz; iz++) {
                float w = f[(size_t)ix * pnz + iz] * fy[iy];
                rr[((size_t)iy * pnx + ix) * pnz + iz] = w;
            }
    free(f);
    free(fy);
}

/* One forward step: term = Lap(a) + rr w; next = S(2a - S b + V term). */
static void SFX(pf3_step)(const SFX(pf3g) *g, const REAL *a, const REAL *b, const REAL *rr,
                          REAL w, REAL *term, REAL *next)
{
    const int pnz = g->pnz, pnx = g->pnx, pny = g->pny;
    SFX(pf3_laplace)(g, a, term);
    for (int iy = 0; iy < pny; iy++)
        for (int ix = 0; ix < pnx; ix++)
            for (int iz = 0; iz < pnz; iz++) {
                size_t j = ((size_t)iy * pnx + ix) * pnz + iz;
                REAL t = term[j];
                if (rr[j] != 0) t = t + rr[j] * w;
                term[j] = t;
                REAL p = SFX(pf3_sponge)(g, iz, ix, iy, b[j]);
                REAL v = (2 * a[j] - p) + g->V[j] * t;
                next[j] = SFX(pf3_sponge)(g, iz, ix, iy, v);
            }
}

static void SFX(pf3_record)(const SFX(pf3g) *g, const REAL *a, int nt, int it, int rz, int nrx,
                            int nry, const int *rx, const int *ry, REAL *d)
{
    for (int j = 0; j < nry; j++)
        for (int i = 0; i < nrx; i++) {
            size_t c = ((size_t)(ry[j] + g->nb) * g->pnx + rx[i] + g->nb) * g->pnz + rz + g->nb;
            d[((size_t)j * nrx + i) * nt + it] = a[c];
        }
}

/* Forward modelling of ns shots; src [ns][3] interior (z, x, y). */
void SFX(or_pf3_forward)(int nz, int nx, int ny, int nb, float dz, float dx, float dy, int nt,
                         float dt, float coef, int ns, const int *src, int rz, int nrx, int nry,
                         const int *rx, const int *ry, const REAL *vel, const REAL *wav,
                         REAL *data)
{
    SFX(pf3g) g;
    SFX(pf3_setup)(&g, nz, nx, ny, nb, dz, dx, dy, dt, coef, vel);
    REAL *rr = (REAL *)calloc(g.np, sizeof(REAL)), *term = (REAL *)calloc(g.np, sizeof(REAL));
    REAL *a = (REAL *)calloc(g.np, sizeof(REAL)), *b = (REAL *)calloc(g.np, sizeof(REAL));
    REAL *c = (REAL *)calloc(g.np, sizeof(REAL));
    const size_t nr = (size_t)nrx * nry;
    for (int is = 0; is < ns; is++) {
        memset(a, 0, g.np * sizeof(REAL));
        memset(b, 0, g.np * sizeof(REAL));
        SFX(pf3_source_map)(&g, src[3 * is] + nb, src[3 * is + 1] + nb, src[3 * is + 2] + nb, rr);
        REAL *d = data + (size_t)is * nr * nt;
        for (int it = 0; it < nt; it++) {
            SFX(pf3_record)(&g, a, nt, it, rz, nrx, nry, rx, ry, d);
            SFX(pf3_step)(&g, a, b, rr, wav[it], term, c);
            REAL *t = b; b = a; a = c; c = t;
            /* b now holds the old a: the step's S b reads S(old a) */
        }
    }
    free(rr); free(term); free(a); free(b); free(c);
    SFX(pf3_free)(&g);
}

/* Exact discrete adjoint (the 2-D derivation of or_pfwi_gradient_exact on
 * three axes).  With b_{n+1} = a_n stored unsponged here, the forward is
 * a_{n+1} = S(2 a_n - S a_{n-1} + V term_n); the adjoint
 *   phi_{n-1} = S (2 phi_n - S phi_{n+1} + V (L phi_n + R^T rho_n)),
 * rho_n = W (d_n - dobs_n), and dJ/dV = sum_n (phi_n / V) term_n, folded
 * through the edge-replicated padding with dV/dv = 2 v dt^2.  weight [nr][nt]
 * or NULL (1).  Stores the whole forward history: small cases only.
 * Returns J = 0.5 sum W (d - dobs)^2. */
REAL SFX(or_pf3_gradient_exact)(int nz, int nx, int ny, int nb, float dz, float dx, float dy,
                                int nt, float dt, float coef, int ns, const int *src, int rz,
                                int nrx, int nry, const int *rx, const int *ry, const REAL *vel,
                                const REAL *wav, const REAL *dobs, const REAL *weight, REAL *grad)
{
    SFX(pf3g) g;
    SFX(pf3_setup)(&g, nz, nx, ny, nb, dz, dx, dy, dt, coef, vel);
    const size_t np = g.np, nr = (size_t)nrx * nry;
    REAL *rr = (REAL *)calloc(np, sizeof(REAL)), *term = (REAL *)calloc(np, sizeof(REAL));
    REAL *hist = (REAL *)calloc(np * (size_t)(nt + 2), sizeof(REAL));
    REAL *lap = (REAL *)calloc(np, sizeof(REAL)), *gV = (REAL *)calloc(np, sizeof(REAL));
    REAL *phi0 = (REAL *)calloc(np, sizeof(REAL)), *phi1 = (REAL *)calloc(np, sizeof(REAL));
    REAL *phim = (REAL *)calloc(np, sizeof(REAL));
    REAL *d = (REAL *)calloc(nr * nt, sizeof(REAL));
    REAL J = 0;
    for (int is = 0; is < ns; is++) {
        SFX(pf3_source_map)(&g, src[3 * is] + nb, src[3 * is + 1] + nb, src[3 * is + 2] + nb, rr);
        /* hist[n + 1] = a_n, hist[0] = a_{-1} = 0 */
        memset(hist, 0, 2 * np * sizeof(REAL));
        for (int n = 0; n < nt; n++) {
            REAL *an = hist + (size_t)(n + 1) * np;
            SFX(pf3_record)(&g, an, nt, n, rz, nrx, nry, rx, ry, d);
            SFX(pf3_step)(&g, an, an - np, rr, wav[n], term, an + np);
        }
        const REAL *dd = dobs + (size_t)is * nr * nt;
        for (size_t k = 0; k < nr * nt; k++) {
            REAL r = d[k] - dd[k];
            REAL w = weight ? weight[k] : 1;
            J += 0.5 * w * r * r;
            d[k] = w * r; /* d now holds rho */
        }
        memset(phi0, 0, np * sizeof(REAL));
        memset(phi1, 0, np * sizeof(REAL));
        for (int n = nt - 1; n >= 0; n--) {
            const REAL *an = hist + (size_t)(n + 1) * np;
            SFX(pf3_laplace)(&g, an, lap);
            for (size_t j = 0; j < np; j++) gV[j] += phi1[j] / g.V[j] * (lap[j] + rr[j] * wav[n]);
            SFX(pf3_laplace)(&g, phi1, lap);
            for (int jy = 0; jy < nry; jy++)
                for (int ix = 0; ix < nrx; ix++) {
                    size_t c = ((size_t)(ry[jy] + nb) * g.pnx + rx[ix] + nb) * g.pnz + rz + nb;
                    lap[c] += d[((size_t)jy * nrx + ix) * nt + n];
                }
            for (int iy = 0; iy < g.pny; iy++)
                for (int ix = 0; ix < g.pnx; ix++)
                    for (int iz = 0; iz < g.pnz; iz++) {
                        size_t j = ((size_t)iy * g.pnx + ix) * g.pnz + iz;
                        REAL s0 = SFX(pf3_sponge)(&g, iz, ix, iy, phi0[j]);
                        REAL v = 2 * phi1[j] - s0 + g.V[j] * lap[j];
                        phim[j] = SFX(pf3_sponge)(&g, iz, ix, iy, v);
                    }
            REAL *t = phi0; phi0 = phi1; phi1 = phim; phim = t;
        }
    }
    memset(grad, 0, (size_t)nz * nx * ny * sizeof(REAL));
    for (int iy = 0; iy < g.pny; iy++)
        for (int ix = 0; ix < g.pnx; ix++)
            for (int iz = 0; iz < g.pnz; iz++) {
                int jz = iz - nb, jx = ix - nb, jy = iy - nb;
                jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
                jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
                jy = jy < 0 ? 0 : (jy >= ny ? ny - 1 : jy);
                size_t j = ((size_t)iy * g.pnx + ix) * g.pnz + iz;
                grad[((size_t)jy * nx + jx) * nz + jz] += gV[j] * 2 * g.vp[j] * g.dt2;
            }
    free(rr); free(term); free(hist); free(lap); free(gV); free(phi0); free(phi1); free(phim);
    free(d);
    SFX(pf3_free)(&g);
    return J;
}

/* J of or_pf3_gradient_exact alone (finite differences) */
REAL SFX(or_pf3_misfit)(int nz, int nx, int ny, int nb, float dz, float dx, float dy, int nt,
                        float dt, float coef, int ns, const int *src, int rz, int nrx, int nry,
                        const int *rx, const int *ry, const REAL *vel, const REAL *wav,
                        const REAL *dobs, const REAL *weight)
{
    const size_t nr = (size_t)nrx * nry;
    REAL *d = (REAL *)calloc((size_t)ns * nr * nt, sizeof(REAL));
    SFX(or_pf3_forward)(nz, nx, ny, nb, dz, dx, dy, nt, dt, coef, ns, src, rz, nrx, nry, rx, ry,
                        vel, wav, d);
    REAL J = 0;
    for (size_t k = 0; k < (size_t)ns * nr * nt; k++) {
        REAL r = d[k] - dobs[k];
        REAL w = weight ? weight[k % (nr * nt)] : 1;
        J += 0.5 * w * r * r;
    }
    free(d);
    return J;
}
