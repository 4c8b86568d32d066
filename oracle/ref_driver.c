/* Thin C driver around the reference's own FWI and wavelet routines.
 *
 * Test infrastructure only: compiled by oracle/Makefile together with the
 * UNMODIFIED reference sources (pywave/src/*.c, read in place) into
 * oracle/_ref/libpwref.so.  It exposes entry points the reference's Python
 * glue never returns -- the raw gradients of gradient_av and gradient_pas_av,
 * the unscaled Ricker table of fdm2d -- so the oracle restatement can be
 * pinned against them.
 *
 * Parameter set-up mirrors pywave/src/pfwi.c:743-860 (fwic) and
 * pfwi.c:260-300 (forward_modeling_ac).
 */
#include <stdio.h>
#include <string.h>
#include <stdbool.h>
#include "wave_alloc.h"
#include "wave_fwiutil.h"
#include "wave_fwimodeling.h"
#include "wave_fwigradient.h"
#include "wave_butter.h"
#include "wave_komplex.h" /* pulls in wave_kissfft.h once */
#include "wave_ricker.h"
#include "wave_freqfilt.h"

/* Ricker table exactly as fdm2d builds it (pywave/src/wave_fdm.c:502-516). */
void refdrv_ricker(int nt, float dt, float f0, float t0, float A, float *out)
{
    int it, fft_size;
    float freq;
    for (it = 0; it < nt; it++) out[it] = 0.f;
    out[(int)(t0 / dt)] = A;
    freq = f0 * dt;
    fft_size = 2 * kiss_fft_next_fast_size((nt + 1) / 2);
    ricker_init(fft_size, freq, 0);
    np_freqfilt(nt, out);
    ricker_close();
}

int refdrv_next_fast(int n) { return kiss_fft_next_fast_size(n); }

static void fill_acpar(np_acqui acpar, np_sou soupar, const float *par)
{
    /* par: nz,nx,dz,dx,oz,ox,nt,dt,ot,ns,ds,os,nb,coef,f0,acqui_type,interval */
    acpar->nz = (int)par[0];
    acpar->nx = (int)par[1];
    acpar->dz = par[2];
    acpar->dx = par[3];
    acpar->z0 = par[4];
    acpar->x0 = par[5];
    acpar->nt = (int)par[6];
    acpar->dt = par[7];
    acpar->t0 = par[8];
    acpar->ns = (int)par[9];
    acpar->ds = par[10];
    acpar->s0 = par[11];
    acpar->nb = (int)par[12];
    acpar->coef = par[13];
    acpar->f0 = par[14];
    acpar->acqui_type = (int)par[15];
    acpar->interval = (int)par[16];
    acpar->sz = 5;
    acpar->nr = acpar->nx;
    acpar->dr = acpar->dx;
    acpar->r0 = acpar->x0;
    acpar->rz = 1;
    soupar->fhi = 0.5 / acpar->dt;
    soupar->flo = 0.;
    soupar->rectx = 2;
    soupar->rectz = 2;
}

/* forward_modeling_a (pywave/src/wave_fwimodeling.c:21-114).
 * vel/q: [nx][nz]; wav: [nt]; data out: [ns][nr=nx][nt]. */
void refdrv_forward(const float *par, float *vel, float *q, float *wav, float *data)
{
    np_sou soupar = (np_sou)np_alloc(1, sizeof(*soupar));
    np_acqui acpar = (np_acqui)np_alloc(1, sizeof(*acpar));
    np_vec array = (np_vec)np_alloc(1, sizeof(*array));
    fill_acpar(acpar, soupar, par);
    preparation(vel, q, wav, acpar, soupar, array);
    float ***d = np_floatalloc3(acpar->nt, acpar->nx, acpar->ns);
    forward_modeling_a(d, soupar, acpar, array, false);
    memcpy(data, d[0][0], sizeof(float) * acpar->nt * acpar->nx * acpar->ns);
}

/* gradient_init + one gradient_av call (pywave/src/wave_fwigradient.c:20-262)
 * with the fwic settings (pfwi.c:843-860) except the smoothing radius, which
 * the caller picks (rect=1 disables gradient_smooth2's triangle smoothing).
 * The output includes gradient_av's first-call 0.1/max|g| scaling. */
void refdrv_gradient(const float *par, float *vel, float *q, float *wav,
                     float *dobs, int rect, float *grad, float *fcost)
{
    np_sou soupar = (np_sou)np_alloc(1, sizeof(*soupar));
    np_acqui acpar = (np_acqui)np_alloc(1, sizeof(*acpar));
    np_vec array = (np_vec)np_alloc(1, sizeof(*array));
    np_fwi fwipar = (np_fwi)np_alloc(1, sizeof(*fwipar));
    fill_acpar(acpar, soupar, par);
    preparation(vel, q, wav, acpar, soupar, array);
    float ***d = np_floatalloc3(acpar->nt, acpar->nx, acpar->ns);
    memcpy(d[0][0], dobs, sizeof(float) * acpar->nt * acpar->nx * acpar->ns);
    fwipar->onlygrad = false;
    fwipar->grad_type = 1;
    fwipar->misfit_type = 1;
    fwipar->opt_type = 1;
    fwipar->wt1 = acpar->t0;
    fwipar->wt2 = acpar->t0 + (acpar->nt - 1) * acpar->dt;
    fwipar->woff1 = acpar->r0;
    fwipar->woff2 = acpar->r0 + (acpar->nr - 1) * acpar->dr;
    fwipar->oreo = false;
    fwipar->waterz = 0;
    fwipar->waterzb = 0;
    fwipar->rectx = rect;
    fwipar->rectz = rect;
    gradient_init(d, soupar, acpar, array, fwipar, false);
    gradient_av(array->vv, fcost, grad);
}

/* gradient_pas_init + one gradient_pas_av call (wave_fwigradient.c:528-870)
 * as pfwic sets them up (pfwi.c:1780-1890: velocity only, so the source
 * weight is 1 and no source inversion runs), with the caller's smoothing
 * radius and multiscale cutoffs.  src: [ns][nt][nx][nz] source fields.  The output includes the
 * first-call 0.1/max|g| scaling. */
void refdrv_gradient_pas(const float *par, float *vel, float *q, float *wav, float *dobs,
                         float *src, int rect, float flo, float fhi, float *grad, float *fcost)
{
    np_sou soupar = (np_sou)np_alloc(1, sizeof(*soupar));
    np_acqui acpar = (np_acqui)np_alloc(1, sizeof(*acpar));
    np_vec array = (np_vec)np_alloc(1, sizeof(*array));
    np_fwi fwipar = (np_fwi)np_alloc(1, sizeof(*fwipar));
    fill_acpar(acpar, soupar, par);
    /* multiscale cutoffs in Hz (pfwic: flo 0, fhi 0.5/dt, i.e. no filter) */
    soupar->flo = flo;
    soupar->fhi = fhi;
    np_pas paspar = passive_init(acpar);
    paspar->inv = true;
    paspar->onlysrc = false;
    paspar->onlyvel = true;
    preparation(vel, q, wav, acpar, soupar, array);
    const int nz = acpar->nz, nx = acpar->nx, nt = acpar->nt, ns = acpar->ns;
    float ***d = np_floatalloc3(nt, nx, ns);
    memcpy(d[0][0], dobs, sizeof(float) * nt * nx * ns);
    float ****w = np_floatalloc4(nz, nx, nt, ns);
    memcpy(w[0][0][0], src, sizeof(float) * (size_t)nz * nx * nt * ns);
    fwipar->onlygrad = false;
    fwipar->grad_type = 1;
    fwipar->misfit_type = 1;
    fwipar->opt_type = 1;
    fwipar->wt1 = acpar->t0;
    fwipar->wt2 = acpar->t0 + (acpar->nt - 1) * acpar->dt;
    fwipar->woff1 = acpar->r0;
    fwipar->woff2 = acpar->r0 + (acpar->nr - 1) * acpar->dr;
    fwipar->oreo = false;
    fwipar->waterz = 0;
    fwipar->waterzb = 0;
    fwipar->rectx = rect;
    fwipar->rectz = rect;
    gradient_pas_init(d, w, NULL, soupar, acpar, array, fwipar, paspar, false);
    gradient_pas_av(array->vv, fcost, grad);
}

/* np_butter_init + np_butter_apply over n samples (wave_butter.c) */
void refdrv_butter(int low, float cutoff, int nn, int n, float *x)
{
    np_butter bw = np_butter_init(low != 0, cutoff, nn);
    np_butter_apply(bw, n, x);
    np_butter_close(bw);
}

/* residual_weighting (wave_fwiutil.c:225-296); w: [nr][nt] */
void refdrv_residual_weights(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2,
                             int oreo, float *w)
{
    float **ww = np_floatalloc2(nt, nr);
    residual_weighting(ww, nt, nr, wtn1, wtn2, woffn1, woffn2, oreo != 0);
    memcpy(w, ww[0], sizeof(float) * nt * nr);
    free(ww[0]);
    free(ww);
}

/* visco-acoustic forward_modeling (wave_fwimodeling.c:116-220): the
 * memory-variable scheme with tau, taus from q and f0 (preparation,
 * wave_fwiutil.c:90-96).  data out: [ns][nr=nx][nt]. */
void refdrv_forward_visco(const float *par, float *vel, float *q, float *wav, float *data)
{
    np_sou soupar = (np_sou)np_alloc(1, sizeof(*soupar));
    np_acqui acpar = (np_acqui)np_alloc(1, sizeof(*acpar));
    np_vec array = (np_vec)np_alloc(1, sizeof(*array));
    fill_acpar(acpar, soupar, par);
    preparation(vel, q, wav, acpar, soupar, array);
    float ***d = np_floatalloc3(acpar->nt, acpar->nx, acpar->ns);
    forward_modeling(d, soupar, acpar, array, false);
    memcpy(data, d[0][0], sizeof(float) * acpar->nt * acpar->nx * acpar->ns);
}

/* gradient_init + one gradient_v call (wave_fwigradient.c:20-92, 264-452),
 * set up as refdrv_gradient; output after the first-call scaling and the
 * caller's smoothing radius. */
void refdrv_gradient_visco(const float *par, float *vel, float *q, float *wav, float *dobs,
                           int rect, float *grad, float *fcost)
{
    np_sou soupar = (np_sou)np_alloc(1, sizeof(*soupar));
    np_acqui acpar = (np_acqui)np_alloc(1, sizeof(*acpar));
    np_vec array = (np_vec)np_alloc(1, sizeof(*array));
    np_fwi fwipar = (np_fwi)np_alloc(1, sizeof(*fwipar));
    fill_acpar(acpar, soupar, par);
    preparation(vel, q, wav, acpar, soupar, array);
    float ***d = np_floatalloc3(acpar->nt, acpar->nx, acpar->ns);
    memcpy(d[0][0], dobs, sizeof(float) * acpar->nt * acpar->nx * acpar->ns);
    fwipar->onlygrad = false;
    fwipar->grad_type = 1;
    fwipar->misfit_type = 1;
    fwipar->opt_type = 1;
    fwipar->wt1 = acpar->t0;
    fwipar->wt2 = acpar->t0 + (acpar->nt - 1) * acpar->dt;
    fwipar->woff1 = acpar->r0;
    fwipar->woff2 = acpar->r0 + (acpar->nr - 1) * acpar->dr;
    fwipar->oreo = false;
    fwipar->waterz = 0;
    fwipar->waterzb = 0;
    fwipar->rectx = rect;
    fwipar->rectz = rect;
    gradient_init(d, soupar, acpar, array, fwipar, false);
    gradient_v(array->vv, fcost, grad);
}
