/* pywave_b200 -- C ABI of the B200-native acoustic FD / TRI / FWI-gradient path.
 *
 * Plain C: pointers, sizes and status codes; no torch or CUDA types in the
 * signatures (streams are passed as `void *`, a cudaStream_t; NULL = the
 * legacy default stream).  Every entry point returns PW_OK (0) or a negative
 * PW_ERR_* status; pw_last_error() gives the message of the calling thread's
 * last failure.
 *
 * Array conventions follow the reference: column-major, z fastest
 * (pywave/afd2d.py:48 `vel.flatten(order='F')`); traces with time fastest
 * ([ny][nx][nt], pywave/src/afd.c:202-206,473-486); pfwi data [ns][nr][nt]
 * (pywave/pfwi.py:74).  Pointers are device pointers unless the args carry
 * PW_HOST_PTRS, in which case the library stages host<->device copies on the
 * given stream itself (the drop-in path of the reference's Python glue).
 */
#ifndef PYWAVE_B200_H
#define PYWAVE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PW_OK 0
#define PW_ERR_SHAPE (-1)     /* inconsistent or unsupported sizes / indices */
#define PW_ERR_CFL (-2)       /* time step violates the scheme's stability limit */
#define PW_ERR_OOM (-3)       /* device allocation failed */
#define PW_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up */
#define PW_ERR_CUDA (-5)      /* a CUDA runtime call failed */
#define PW_ERR_VALUE (-6)     /* NaN/Inf or non-positive velocity, bad flag */

#define PW_HOST_PTRS 1        /* all array pointers are host memory */
#define PW_NO_CFL_CHECK 2     /* skip the host-side stability check */
#define PW_PER_SHOT 4         /* pfwi: one shot at a time (the reference's summation order) */

/* ---------------------------------------------------------------- afd --- */

/* Arguments of the afd propagator: afd2dc / afd3dc of the reference
 * (pywave/src/afd.c:23-314 and 316-578; parse formats afd.c:73,366), with
 * abc forced on and every face using nbt/ct as afd.c:98-116,389-402 do. */
typedef struct pw_afd_args {
  int dim;        /* 2 or 3 */
  int nz, nx, ny; /* interior model size (ny = 1 for 2-D) */
  int nt;         /* time samples */
  int nbt;        /* absorbing taper width on every face (afd.c:101-116) */
  float ct;       /* taper coefficient, w = exp(-(ct*(nbt-1-i))^2) (wave_abc.c:142) */
  float dt, dz, dx, dy;
  int ns;         /* forward: number of point sources */
  int tri;        /* 0: forward modelling, 1: time-reversal (reverse time, inject traces) */
  int jsnap;      /* snapshot interval (0 = no snapshots), wave_fdm.c:652-661 */
  int gz;         /* receiver depth in interior rows below the top (0 = the reference's z=0) */
  int flags;      /* PW_HOST_PTRS | PW_NO_CFL_CHECK */
} pw_afd_args;

/* Forward modelling or time reversal with the afd scheme.
 * Replaces afd2dc / afd3dc (pywave/src/afd.c:316, :23) and the time loops of
 * fdm2d / fdm (pywave/src/wave_fdm.c:397-686, 28-381).
 *   vel     [ny][nx][nz]                 interior velocity
 *   src     forward: [k][ns] with k rows sx,sz,f,t,A (2-D) or sx,sy,sz,f,t,A
 *           (3-D), exactly afd2d.py:68 / afd3d.py:70's packing;
 *           tri: traces [ny][nx][nt] injected at the receiver row
 *   wavelet optional [ns][nt] source time functions; NULL = the reference's
 *           Ricker table built from f,t,A (wave_fdm.c:502-516)
 *   dat     forward: recorded traces [ny][nx][nt] (may be NULL); unused in tri
 *   wfd     snapshots [ntsnap][ny][nx][nz], ntsnap = #{it < nt : it % jsnap == 0}
 *           (may be NULL); the reference's afd2dc returns dat then wfd. */
int pw_afd(const pw_afd_args *a, const float *vel, const float *src, const float *wavelet,
           float *dat, float *wfd, void *stream);

/* Forward modelling of nshot 2-D shots of uneven size and length in one
 * lockstep time loop: the reference's afd2d forward (afd.c:316, wave_fdm.c:
 * 397-686) run for many shots at once, one kernel launch per time step over
 * the tiles of every shot still running (shots end at their own nt), with
 * the tile shape picked by timing candidates on the first steps and the
 * remaining steps replayed as one CUDA graph (when `stream` is not the
 * legacy default stream).  Traces are bit-identical to pw_afd per shot.
 *   args[k]      each shot's pw_afd_args (dim 2, tri 0, jsnap 0; one
 *                PW_HOST_PTRS setting for all shots)
 *   vel[k], src[k], wavelet[k] (wavelet may be NULL, or wavelet[k] NULL:
 *                the Ricker table), dat[k] [nx][nt] traces, as in pw_afd */
int pw_afd_batch(int nshot, const pw_afd_args *args, const float *const *vel,
                 const float *const *src, const float *const *wavelet, float *const *dat,
                 void *stream);

/* Size of the fixed device scratch array behind pw_afd_noalloc (32 MiB). */
#define PW_NOALLOC_SCRATCH_BYTES (32u << 20)

/* pw_afd's forward modelling (tri = 0) that allocates no device memory.
 * No counterpart in the reference.  For callers that run inside a host
 * framework owning every device allocation (a caching pool that must not be
 * bypassed, a memory budget that a hidden allocation would break): pw_afd grows
 * a cached workspace with cudaMalloc on first use, this entry point never does.
 * Its wavefields, padded velocity, taper tables and trace buffer are carved
 * from one file-scope __device__ array of PW_NOALLOC_SCRATCH_BYTES per device,
 * whose address comes from cudaGetSymbolAddress; a model that needs more is
 * rejected with PW_ERR_SHAPE before any device work (a 1000 x 1000 2-D model
 * with nbt 30 and nt 2000 needs 21 MiB; a 50^3 3-D model with nbt 30 and
 * nt 1000 needs 29 MiB).
 *   Same arguments and results as pw_afd, with these differences: every
 *   pointer is device memory (PW_HOST_PTRS is rejected); with ns > 0 both
 *   src and wavelet [ns][nt] are required (no Ricker table is built);
 *   pw_last_timing is not updated.
 *   The wavefields and the halo of the padded velocity must start at zero:
 *   each call clears the part of the array it uses on `stream` first.  Calls
 *   whose GPU work overlapped would race on the one array; a per-device lock
 *   held until the call's stream has drained (on error returns as well) keeps
 *   calls of one process from overlapping.  Every call waits on `stream`: it
 *   reads the source positions back to the host and returns only after its
 *   work has finished.  The first call on a device loads the module holding
 *   the array and takes its address.  The array is reserved when that module
 *   loads: on the first call under lazy module loading
 *   (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2), or when each
 *   context loads the library under EAGER loading, whether or not
 *   pw_afd_noalloc is ever called. */
int pw_afd_noalloc(const pw_afd_args *a, const float *vel, const float *src,
                   const float *wavelet, float *dat, float *wfd, void *stream);

/* Time-reversal source imaging with G receiver groups propagated in lockstep
 * and the image fused into the time loop:
 *   img = sum_{it % jsnap == 0} prod_g u_g(it)^2        (then / max if normalize)
 * This is what the TRI demos assemble in Python from G afd2d/afd3d(tri=True)
 * runs (demos/test_third_tri.py:61-77, demos/test_mod2d_tri_psVSfd.py:166-190);
 * the reference's own C image (wave_fdm.c:666-672) is never returned
 * (afd.c:562-574).
 *   group   [ny][nx] group id (0..ngroups-1) of each receiver, -1 = unused;
 *           NULL = the demos' x-bands of width nx/ngroups
 *   dat     traces [ny][nx][nt] (every group reads its own receivers)
 *   img     [ny][nx][nz] */
int pw_tri_image(const pw_afd_args *a, int ngroups, const int *group, const float *vel,
                 const float *dat, float *img, int normalize, void *stream);

/* --------------------------------------------------------------- pfwi --- */

/* pfwi's 20-float parameter array (pywave/pfwi.py:40-61) decoded, plus the
 * settings pfwi.c hard-codes (sz=5, rz=1, nr=nx, dr=dx, r0=ox: pfwi.c:796-801). */
typedef struct pw_fwi_args {
  int nz, nx;
  float dz, dx, oz, ox;
  int nt;
  float dt, ot;
  int ns;
  float ds, os;
  int nb;          /* sponge width (wave_fwiutil.c:31-36) */
  float coef;      /* sponge coefficient, bc[i] = expf(-(coef*(nb-i))^2) */
  float f0;        /* reference frequency (unused by the acoustic path) */
  int acqui_type;  /* 1 fixed spread, otherwise moving spread (wave_fwiutil.c:55-71) */
  int interval;    /* snapshot interval of the reference-mode gradient */
  int niter;       /* L-BFGS iterations (pw_fwi) */
  int sz, rz;      /* source / receiver depth below the top (pfwi.c: 5 and 1) */
  int flags;       /* PW_HOST_PTRS | PW_NO_CFL_CHECK | PW_PER_SHOT */
  long long hbm_budget; /* bytes of device memory the exact gradient's checkpoints, segment
                           buffer and wavefields may hold; 0 = a quarter of the device */
  float flo, fhi;       /* multiscale residual filter of the REFERENCE-mode gradients (Hz):
                           a 3-pole zero-phase Butterworth high-pass at flo when flo*dt >
                           0.0001 and low-pass at fhi when 0 < fhi*dt < 0.4999
                           (gradient_pas_init / gradient_pas_av, wave_fwigradient.c:657-658,
                           767-780); 0, 0 = off, as pfwic and fwic run it */
} pw_fwi_args;

/* Fills a pw_fwi_args from pfwi's float parameter array (pfwi.c:691-713
 * reads it; only the first 20 entries are meaningful). */
int pw_fwi_args_from_pararray(const float *pararray, int n, pw_fwi_args *out);

/* Acoustic forward modelling of all shots: forward_modeling_ac
 * (pywave/src/pfwi.c:27) -> forward_modeling_a (wave_fwimodeling.c:21-114).
 *   vel [nx][nz], wav [nt], data [ns][nr][nt]. */
int pw_pfwi_forward(const pw_fwi_args *a, const float *vel, const float *wav, float *data,
                    void *stream);

#define PW_GRAD_REFERENCE 0  /* gradient_av's imaging: snapshot-difference u_tt, interior only */
#define PW_GRAD_EXACT 1      /* exact discrete adjoint of the forward scheme, incl. the sponge
                                and the edge-replicated padding; checkpointed */

/* One FWI gradient over all shots: gradient_av (wave_fwigradient.c:93-242)
 * without its post-processing (see pw_gradient_postprocess).
 *   weight  [nr][nt] residual weights; NULL = residual_weighting as fwic sets
 *           it up (wave_fwiutil.c:225-296, pfwi.c:849-855)
 *   grad    [nx][nz] dJ/dv (EXACT) or the reference's raw gradient (REFERENCE)
 *   misfit  0.5*sum(r^2) in FP64 (REFERENCE: unweighted residual as the
 *           reference; EXACT: 0.5*sum(w r^2), consistent with grad)
 *   ckpt_k  checkpoint interval of the EXACT mode (0 = planned under a->hbm_budget,
 *           see pw_last_fwi_plan) */
int pw_pfwi_gradient(const pw_fwi_args *a, int mode, const float *vel, const float *wav,
                     const float *dobs, const float *weight, float *grad, double *misfit,
                     int ckpt_k, void *stream);

/* The same gradient with distributed sources instead of the point source
 * and wavelet (pfwi's passive mode 4 with velocity update): gradient_pas_av
 * (wave_fwigradient.c:667-870, set up by gradient_pas_init :528-663 as pfwic
 * does: velocity only, source weight 1, no multiscale filter).  Each
 * forward step adds src[shot][it][ix][iz] to the term of the interior
 * cell (ix, iz).  src [ns][nt][nx][nz]; the other arguments as above. */
int pw_pfwi_gradient_passive(const pw_fwi_args *a, int mode, const float *vel, const float *src,
                             const float *dobs, const float *weight, float *grad, double *misfit,
                             int ckpt_k, void *stream);

/* Visco-acoustic pfwi (media 2), which the reference implements but its
 * Python glue never reaches (pfwi.c:864 always takes the acoustic path):
 * the pfwi scheme with a memory variable whose relaxation times come from
 * the quality factor q [nx][nz] and a->f0 (preparation, wave_fwiutil.c:90-96).
 * pw_pfwi_forward_visco: forward_modeling (wave_fwimodeling.c:116-220),
 * data [ns][nr][nt].  pw_pfwi_gradient_visco: gradient_v
 * (wave_fwigradient.c:264-452) before its post-processing, shots summed in
 * the reference's order; weight, grad, misfit as pw_pfwi_gradient's
 * REFERENCE mode.  Source maps must stay clear of the grid's 4-cell rim. */
int pw_pfwi_forward_visco(const pw_fwi_args *a, const float *vel, const float *q,
                          const float *wav, float *data, void *stream);
int pw_pfwi_gradient_visco(const pw_fwi_args *a, const float *vel, const float *q,
                           const float *wav, const float *dobs, const float *weight, float *grad,
                           double *misfit, void *stream);

/* Checkpoint plan of the calling thread's last PW_GRAD_EXACT gradient: the
 * interval k, the shots per batch, the device bytes the call held and the
 * recompute factor (forward steps run / nt; 1 = nothing recomputed).  The
 * planner fits pw_fwi_args.hbm_budget and minimises recompute.  No
 * counterpart in the reference, which stores every snapshot
 * (wave_fwigradient.c:116). */
int pw_last_fwi_plan(int *ckpt_k, int *shots_per_batch, long long *bytes, double *recompute);

/* ------------------------------------------------------------ pfwi 3-D --- */

/* The 3-D extension of pfwi's acoustic scheme (the reference has no 3-D FWI:
 * its 2-D step, wave_fwimodeling.c:21-114 and wave_fwiutil.c:19-223, on
 * three axes with an 8th-order Laplacian per axis, a sponge on all six faces
 * and edge-replicated padding; oracle/pw_oracle3d_body.h states it in full). */
typedef struct pw_fwi3d_args {
  int nz, nx, ny;       /* interior model size */
  float dz, dx, dy;
  int nt;
  float dt;
  int nb;               /* sponge width on every face (>= 5) */
  float coef;           /* sponge coefficient, bc[i] = expf(-(coef*(nb-i))^2) */
  int ns;               /* shots */
  const int *src;       /* host [ns][3]: source (z, x, y), interior indices; the
                           spike is smoothed by the rect-2 triangle on each axis */
  int nrx, nry;         /* receivers on the grid (rx[i], ry[j]), trace j*nrx + i */
  const int *rx, *ry;   /* host, interior indices */
  int rz;               /* receiver depth, interior index */
  int flags;            /* PW_HOST_PTRS | PW_NO_CFL_CHECK */
  long long hbm_budget; /* as pw_fwi_args.hbm_budget */
} pw_fwi3d_args;

/* 3-D forward modelling of all shots.  vel [ny][nx][nz], wav [nt],
 * data [ns][nry*nrx][nt] (traces recorded before each step, as pfwi does). */
int pw_pfwi3d_forward(const pw_fwi3d_args *a, const float *vel, const float *wav, float *data,
                      void *stream);

/* 3-D exact-adjoint FWI gradient of J = 0.5 sum w (d - dobs)^2 over all
 * shots (J in FP64), checkpointed as pw_pfwi_gradient's EXACT mode under
 * a->hbm_budget (pw_last_fwi_plan reports the plan).  No reference
 * counterpart.  weight [nr][nt] or NULL (1); grad [ny][nx][nz] = dJ/dv. */
int pw_pfwi3d_gradient(const pw_fwi3d_args *a, const float *vel, const float *wav,
                       const float *dobs, const float *weight, float *grad, double *misfit,
                       int ckpt_k, void *stream);

/* gradient_av's tail (wave_fwigradient.c:244-255): triangle smoothing
 * rect x rect (wave_fwiutil.c:298-335) and the scale factor; *scaling <= 0 on
 * entry means "first call": it is set to 0.1/max|grad| as the reference's
 * static does. */
int pw_gradient_postprocess(int nz, int nx, int rect, int waterz, float *grad, float *scaling,
                            int flags, void *stream);

/* Full-waveform inversion as fwic runs it (pywave/src/pfwi.c:497-1029 ->
 * fwi, wave_fwi.c:24-119): gradient_av + gradient_smooth2 (rect 3, first-call
 * scale), L-BFGS with 20 pairs and the Wolfe line search of
 * wave_fwilbfgs.c:108-165 (20 trials, c1 1e-4, c2 0.9, factor 10, clip [0,10]),
 * stopping when misfit/misfit0 < 0.01.  Inner products run in FP64 on the GPU.
 *   vel0 [nx][nz] starting model, dobs [ns][nr][nt],
 *   vinv [niter][nx][nz] model after each iteration (zero after an early stop),
 *   iters_done number of completed iterations. */
int pw_fwi(const pw_fwi_args *a, const float *vel0, const float *wav, const float *dobs,
           float *vinv, int *iters_done, void *stream);

/* Passive-source FWI as pfwic runs it (pywave/src/pfwi.c:1507-2036 -> pfwi,
 * wave_fwi.c:212-322): pw_fwi's optimiser with gradient_pas_av on the
 * source fields src [ns][nt][nx][nz] and the line-search step reset to 1
 * every 5 iterations (optpar->repeat).  vinv and iters_done as pw_fwi. */
int pw_pfwi_passive(const pw_fwi_args *a, const float *vel0, const float *src, const float *dobs,
                    float *vinv, int *iters_done, void *stream);

/* ------------------------------------------------- pseudo-spectral --- */

/* Forward modelling or time reversal with the pseudo-spectral method: the
 * reference's apscfun.aps2dc / aps3dc (pywave/src/aps.c:315, :22) and the
 * time loops of psm2d / psm (wave_psp.c:367-635, 25-352).  Arguments exactly
 * as pw_afd's (the two modules share their argument tuples and outputs);
 * the Laplacian is -(2 pi |k|)^2 applied through cuFFT on the reference's
 * FFT-padded grid with its centring, so results agree with the reference to
 * float rounding (its KISS FFT rounds differently), not bit for bit.  No
 * stability check (the reference has none). */
int pw_aps(const pw_afd_args *a, const float *vel, const float *src, const float *wavelet,
           float *dat, float *wfd, void *stream);

/* ---------------------------------------------- pfwi mode 4: LS-TRI --- */

/* pfwi's passive mode 4 without velocity update (pfwicfun.lstric,
 * pywave/src/pfwi.c:1031-1444).  Geometry from pw_fwi_args: nz, nx, dz, dx,
 * nt, dt, ns, nb (>= 4), coef, rz (the data row is padded row rz + nb; the
 * pararray parser sets rz = 1 as pfwi.c:1319 does), niter (CG iterations),
 * flags (PW_HOST_PTRS).  vel [nx][nz]; a shot's source field
 * [nt][nx][nz]; a shot's data [nx][nt].  Fields and data are bit-identical
 * to the reference's timerev_lop (wave_triutil.c:48-316). */

/* timerev_lop with add = 0, one shot (wave_triutil.c:86-180): adj = 0 maps
 * mod to dat, adj = 1 maps dat to mod. */
int pw_timerev(const pw_fwi_args *a, int adj, const float *vel, float *mod, float *dat,
               void *stream);

/* lstric with inv = 0 (lstri, wave_fwi.c:121-175): data [ns][nx][nt] of the
 * source fields src [ns][nt][nx][nz]; every shot in one launch. */
int pw_lstri_forward(const pw_fwi_args *a, const float *vel, const float *src, float *data,
                     void *stream);

/* lstric with inv = 1 (lstri_op, wave_fwigradient.c:454-520): per shot,
 * a->niter conjugate-gradient iterations of np_solver / np_cgstep
 * (wave_bigsolver.c:1170, wave_cgstep.c:16) from a zero source field;
 * src [ns][nt][nx][nz] out, data [ns][nx][nt] in.  The CG step vectors carry
 * over from one shot to the next within the call, as the reference's do;
 * dot products run in FP64 in a fixed block order. */
int pw_lstri_invert(const pw_fwi_args *a, const float *vel, const float *data, float *src,
                    void *stream);

/* ---------------------------------------------- residual utilities --- */

/* np_butter_init + np_butter_apply (wave_butter.c:18-102): every one of the
 * ntr traces x [ntr][n] filtered in place, causally, by a Butterworth
 * low-pass (low = 1) or high-pass (low = 0) of npoles (1..16) poles at
 * cutoff cycles per sample.  flags: PW_HOST_PTRS. */
int pw_butter_apply(int n, int ntr, int low, float cutoff, int npoles, float *x, int flags,
                    void *stream);

/* residual_weighting (wave_fwiutil.c:225-296), host only: w [nr][nt] is 1 on
 * the window [woffn1, woffn2] x [wtn1, wtn2] with 10-sample sine tapers
 * inside its edges (oreo = 0, as fwic and pfwic use it), or 0 on the window
 * and 1 outside with the tapers outside its edges (oreo = 1).  Taper samples
 * beyond the array (a window closer than 10 samples to an edge, where the
 * reference writes out of bounds) are skipped. */
int pw_residual_weights(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2, int oreo,
                        float *w);

/* ------------------------------------------------------------ utility --- */

const char *pw_last_error(void);
const char *pw_version(void);
/* Releases the calling device's cached device memory: the workspace and
 * the cached cuFFT plans of pw_aps. */
int pw_release_cache(void);
/* Device time of the calling thread's last completed call: the time loop
 * alone (CUDA events recorded on the call's stream around its step kernels),
 * the number of step-kernel launches in it, and the whole call's kernel
 * launches.  Used by the benchmark to time the dominant kernel live. */
int pw_last_timing(double *loop_ms, long long *step_launches, long long *total_launches);

#ifdef __cplusplus
}
#endif
#endif
