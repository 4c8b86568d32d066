// pfwi acoustic path (forward modelling, FWI gradient, post-processing).
#include "pw_common.cuh"

extern "C" int pw_fwi_args_from_pararray(const float *p, int n, pw_fwi_args *o) {
  PW_CHECK(p && o && n >= 20, PW_ERR_VALUE, "pararray needs 20 values");
  memset(o, 0, sizeof *o);
  o->nz = (int)p[0]; o->nx = (int)p[1]; o->dz = p[2]; o->dx = p[3]; o->oz = p[4]; o->ox = p[5];
  o->nt = (int)p[6]; o->dt = p[7]; o->ot = p[8]; o->ns = (int)p[10]; o->ds = p[11];
  o->os = p[12]; o->nb = (int)p[14]; o->coef = p[15]; o->f0 = p[16];
  o->acqui_type = (int)p[17]; o->interval = (int)p[18]; o->niter = (int)p[19];
  o->sz = 5; o->rz = 1;
  return PW_OK;
}

extern "C" int pw_pfwi_forward(const pw_fwi_args *, const float *, const float *, float *, void *) {
  pw::set_error("pw_pfwi_forward: not built yet");
  return PW_ERR_SHAPE;
}

extern "C" int pw_pfwi_gradient(const pw_fwi_args *, int, const float *, const float *,
                                const float *, const float *, float *, double *, int, void *) {
  pw::set_error("pw_pfwi_gradient: not built yet");
  return PW_ERR_SHAPE;
}

extern "C" int pw_gradient_postprocess(int, int, int, int, float *, float *, int, void *) {
  pw::set_error("pw_gradient_postprocess: not built yet");
  return PW_ERR_SHAPE;
}
