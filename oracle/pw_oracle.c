/* CPU oracle for the pywave acoustic FD / TRI / FWI-gradient hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker
 * or the timed CPU baseline -- never as the thing measured or shipped.
 *
 * It restates, in plain C, the algorithms of:
 *   fdm2d / fdm              pywave/src/wave_fdm.c:28-381, 397-686
 *   vel_expand / abc_*       pywave/src/wave_abc.c:14-294
 *   Ricker table             pywave/src/wave_fdm.c:502-516, wave_ricker.c:22-58,
 *                            wave_freqfilt.c:76-99 (closed form of the same DFT)
 *   padding-size rule        pywave/src/wave_fft2.c:45-51, wave_fft3.c:44-60,
 *                            wave_kissfft.c:412-424
 *   pfwi acoustic modelling  pywave/src/wave_fwimodeling.c:21-114,
 *                            wave_fwiutil.c:19-223
 *   gradient_av              pywave/src/wave_fwigradient.c:93-262
 *   triangle smoothing       pywave/src/wave_triangle.c:177-238 (np_smooth2)
 *   residual weighting       pywave/src/wave_fwiutil.c:225-296 (both branches)
 *   Butterworth filter       pywave/src/wave_butter.c:18-116
 * plus the exact discrete adjoint of the pfwi forward step (FP64), derived
 * for this project and checked against finite differences in tests/, and
 * the 3-D extension of the pfwi scheme with its exact adjoint
 * (pw_oracle3d_body.h; the reference has no 3-D FWI), and pfwi's passive
 * mode 4 (pw_oracle_lstri_body.h): the time-reversal operator timerev_lop
 * (pywave/src/wave_triutil.c:48-316) and the LS-TRI source inversion by
 * np_solver / np_cgstep (wave_fwi.c:121, wave_bigsolver.c:1170,
 * wave_cgstep.c:16).
 *
 * The body is instantiated twice (pw_oracle_body.h): REAL=float reproduces
 * the reference's float evaluation order operation by operation (no FMA
 * contraction: built with -ffp-contract=off), REAL=double is the FP64 oracle
 * against which every FP32 result's error is stated.
 *
 * Parity pins: tests/test_oracle_golden.py checks the float instance against
 * golden vectors produced by the reference itself (tests/golden/, generated
 * by tests/golden/make_golden.py from the reference compiled under oracle/_ref).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

/* kiss_fft_next_fast_size (pywave/src/wave_kissfft.c:412-424): smallest
 * n' >= n whose only prime factors are 2, 3 and 5. */
int or_next_fast(int n)
{
    for (;; n++) {
        int m = n;
        while (m % 2 == 0) m /= 2;
        while (m % 3 == 0) m /= 3;
        while (m % 5 == 0) m /= 5;
        if (m <= 1) return n;
    }
}

/* Padded sizes of fft2_init/fft3_init with cmplx=0, pad1=1: the first (z)
 * axis becomes 2*next_fast((n+1)/2), the others next_fast(n). */
int or_pad_first(int n) { return 2 * or_next_fast((n + 1) / 2); }

/* Ricker table of fdm2d (wave_fdm.c:502-516): a spike of height A at sample
 * (int)(t0/dt), zero-phase filtered by shape(w) = w*exp(1-w)/nfft,
 * w = (k*dw)^2, dw = 1/(nfft*f0*dt), nfft = 2*next_fast((nt+1)/2).  The
 * reference does forward FFT -> multiply -> inverse FFT with KISS FFT in
 * float; with a single spike that is the cosine sum below, evaluated here in
 * double with the shape samples rounded to float as the reference stores
 * them. */
void or_ricker(int nt, float dt, float f0, float t0, float A, double *out)
{
    int nfft = 2 * or_next_fast((nt + 1) / 2);
    int nw = nfft / 2 + 1;
    int k0 = (int)(t0 / dt);
    float freq = f0 * dt;
    float dw = (float)(1. / (nfft * freq));
    double *shape = (double *)malloc(sizeof(double) * nw);
    double *ctab = (double *)malloc(sizeof(double) * nfft);
    for (int k = 0; k < nw; k++) {
        float w = k * dw;
        w *= w;
        shape[k] = (double)(w * expf(1 - w) / nfft);
    }
    for (int j = 0; j < nfft; j++) ctab[j] = cos(2.0 * M_PI * (double)j / (double)nfft);
    for (int n = 0; n < nt; n++) {
        long m = n - k0;
        double s = shape[0];
        for (int k = 1; k < nfft / 2; k++) {
            long ph = ((long)k * m) % nfft;
            if (ph < 0) ph += nfft;
            s += 2.0 * shape[k] * ctab[ph];
        }
        {
            long ph = ((long)(nfft / 2) * m) % nfft;
            if (ph < 0) ph += nfft;
            s += shape[nfft / 2] * ctab[ph];
        }
        out[n] = (double)A * s;
    }
    free(shape);
    free(ctab);
}

/* One line of np_smooth2 (adjoint triangle smoothing, box=false, der=false;
 * wave_triangle.c:177-238): spread with (-w, 2w, -w) at offsets (0, nb, 2nb),
 * integrate forward then backward, fold the 2*nb extension back with
 * half-sample mirror reflections.  Float arithmetic in the reference's order. */
void or_smooth2_line(int nb, int n, float *x, int o, int d, float *tmp)
{
    int np = n + 2 * nb;
    float wt = (float)(1.0 / (nb * nb));
    float t;
    for (int i = 0; i < np; i++) tmp[i] = 0;
    for (int i = 0; i < n; i++) tmp[i] += (-wt) * x[o + i * d];
    for (int i = 0; i < n; i++) tmp[i + nb] += ((float)(2. * wt)) * x[o + i * d];
    for (int i = 0; i < n; i++) tmp[i + 2 * nb] += (-wt) * x[o + i * d];
    t = 0.f;
    for (int i = 0; i < np; i++) { t += tmp[i]; tmp[i] = t; }
    t = 0.f;
    for (int i = np - 1; i >= 0; i--) { t += tmp[i]; tmp[i] = t; }
    for (int i = 0; i < n; i++) x[o + i * d] = tmp[i + nb];
    /* right extension: blocks alternate mirrored / direct */
    for (int m = 0; m < nb; m++) {
        int b = m / n, i = m % n;
        int dst = (b % 2 == 0) ? (n - 1 - i) : i;
        x[o + dst * d] += tmp[nb + n + m];
    }
    /* left extension: blocks alternate direct / mirrored */
    for (int m = 0; m < nb; m++) {
        int b = m / n, i = m % n;
        int dst = (b % 2 == 0) ? i : (n - 1 - i);
        x[o + dst * d] += tmp[nb - 1 - m];
    }
}

/* 2-D smoothing of an [n1 fast][n2] array along axis 0 with rect1 and along
 * axis 1 with rect2 (rect<=1 skips the axis), as source_map and
 * gradient_smooth2 apply it (wave_fwiutil.c:149-177, 298-335). */
void or_smooth2d(int rect1, int rect2, int n1, int n2, float *a)
{
    int nmax = (n1 > n2 ? n1 : n2) + 2 * ((rect1 > rect2 ? rect1 : rect2) + 1);
    float *tmp = (float *)malloc(sizeof(float) * nmax);
    if (rect1 > 1)
        for (int j = 0; j < n2; j++) or_smooth2_line(rect1, n1, a, j * n1, 1, tmp);
    if (rect2 > 1)
        for (int j = 0; j < n1; j++) or_smooth2_line(rect2, n2, a, j, n1, tmp);
    free(tmp);
}

/* residual_weighting with oreo=false (wave_fwiutil.c:225-296, else branch):
 * 1 on [woffn1,woffn2]x[wtn1,wtn2], 10-sample sine tapers at both ends of
 * both axes.  w: [nr][nt]. */
void or_residual_weights(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2, float *w)
{
    float s[10];
    for (int i = 0; i < 10; i++) s[i] = sinf(0.5 * M_PI * (i + 1) / 11.);
    for (int i = 0; i < nr * nt; i++) w[i] = 0.f;
    for (int ir = woffn1; ir <= woffn2; ir++)
        for (int it = wtn1; it <= wtn2; it++) w[ir * nt + it] = 1.f;
    for (int ir = 0; ir < 10; ir++)
        for (int it = wtn1; it <= wtn2; it++) {
            w[(woffn1 + ir) * nt + it] *= s[ir];
            w[(woffn2 - ir) * nt + it] *= s[ir];
        }
    for (int it = 0; it < 10; it++)
        for (int ir = woffn1; ir <= woffn2; ir++) {
            w[ir * nt + wtn1 + it] *= s[it];
            w[ir * nt + wtn2 - it] *= s[it];
        }
}

/* residual_weighting with oreo = true (wave_fwiutil.c:236-265): 1 outside
 * [woffn1,woffn2]x[wtn1,wtn2], 0 inside, 10-sample sine tapers on the
 * outer sides.  w: [nr][nt]. */
void or_residual_weights_oreo(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2,
                              float *w)
{
    float s[10];
    for (int i = 0; i < 10; i++) s[i] = sinf(0.5 * M_PI * (i + 1) / 11.);
    for (int i = 0; i < nr * nt; i++) w[i] = 1.f;
    for (int ir = woffn1; ir <= woffn2; ir++)
        for (int it = wtn1; it <= wtn2; it++) w[ir * nt + it] = 0.f;
    for (int ir = 0; ir < 10; ir++)
        for (int it = wtn1; it <= wtn2; it++) {
            if (woffn1 - ir > 0) w[(woffn1 - ir) * nt + it] *= s[ir];
            if (woffn2 + ir < nr) w[(woffn2 + ir) * nt + it] *= s[ir];
        }
    for (int it = 0; it < 10; it++) {
        for (int ir = 0; ir < woffn1; ir++) {
            w[ir * nt + wtn1 + it] *= s[it];
            w[ir * nt + wtn2 - it] *= s[it];
        }
        for (int ir = woffn2 + 1; ir < nr; ir++) {
            w[ir * nt + wtn1 + it] *= s[it];
            w[ir * nt + wtn2 - it] *= s[it];
        }
    }
}

/* np_butter_init (wave_butter.c:18-62): a Butterworth filter of nn poles as
 * one first-order section (odd nn) and nn/2 second-order sections, cutoff in
 * cycles per sample, every coefficient rounded to float as the reference
 * stores it (its double/float mix kept). */
typedef struct {
    int nn, low;
    float den[16][2];
    float mid;
} or_butter_t;

static void or_butter_init(or_butter_t *bw, int low, float cutoff, int nn)
{
    const double pi = 3.14159265358979323846264338328;
    float arg = 2. * pi * cutoff;
    float sinw = sinf(arg), cosw = cosf(arg), fact, ss;
    bw->nn = nn;
    bw->low = low;
    if (nn % 2) {
        if (low) {
            fact = (1. + cosw) / sinw;
            bw->den[nn / 2][0] = 1. / (1. + fact);
            bw->den[nn / 2][1] = 1. - fact;
        } else {
            fact = sinw / (1. + cosw);
            bw->den[nn / 2][0] = 1. / (fact + 1.);
            bw->den[nn / 2][1] = fact - 1.;
        }
    }
    fact = low ? sinf(0.5 * arg) : cosf(0.5 * arg);
    fact *= fact;
    for (int j = 0; j < nn / 2; j++) {
        ss = sinf(pi * (2 * j + 1) / (2 * nn)) * sinw;
        bw->den[j][0] = fact / (1. + ss);
        bw->den[j][1] = (1. - ss) / fact;
    }
    bw->mid = -2. * cosw / fact;
}

/* the coefficients, for the GPU tests: den [nn/2 + nn%2][2], mid */
void or_butter_coefs(int low, float cutoff, int nn, float *den, float *mid)
{
    or_butter_t bw;
    or_butter_init(&bw, low, cutoff, nn);
    for (int j = 0; j < nn / 2 + nn % 2; j++) {
        den[2 * j] = bw.den[j][0];
        den[2 * j + 1] = bw.den[j][1];
    }
    *mid = bw.mid;
}

#define REAL float
#define SFX(name) name##_f32
#define PW_F32 1
#include "pw_oracle_body.h"
#include "pw_oracle3d_body.h"
#include "pw_oracle_lstri_body.h"
#undef REAL
#undef SFX
#undef PW_F32

#define REAL double
#define SFX(name) name##_f64
#define PW_F32 0
#include "pw_oracle_body.h"
#include "pw_oracle3d_body.h"
#include "pw_oracle_lstri_body.h"
#undef REAL
#undef SFX
#undef PW_F32
