// Pseudo-spectral acoustic propagation: the apscfun module (pywave/src/aps.c,
// aps2dc / aps3dc) and psm2d / psm (pywave/src/wave_psp.c:25-635), forward
// modelling and time reversal, on cuFFT.
//
// The reference's step on its FFT-padded grid (nz2 = 2*next_fast((nz+1)/2),
// nx2 = next_fast(nx), ny2 = next_fast(ny) around the expanded nz x nx x ny
// grid):
//   wave = sign * wwt * IFFT(lapl * FFT(sign * curr)),  sign = (-1)^(ix+iy),
//     lapl = -(2 pi |k|)^2 on the centred grid, wwt = 1/(nz2 nx2 ny2);
//   on the expanded grid: c = curr, curr = (c + (c - prev)) + wave vv,
//     prev = c; sources (3x3(x3) spread, / (|dx|+|dz|(+|dy|)+1)) or the
//     time-reversed traces on the receiver row; abc_apply on curr and prev
//     (face by face over the padded grid); traces; snapshots.
// Here the state is kept modulated, S = sign * curr and P = sign * prev:
// negation is exact, so S feeds the forward FFT directly, sign * wave =
// wwt * (the inverse FFT), and S, P are updated in place by one pointwise
// kernel per step (P' = taper(S), S' = taper(S + (S - P) + ...)).  Per step:
// R2C, multiply by lapl, C2R, update: four launches.  The FFTs are cuFFT's
// (float, a different rounding than the reference's KISS FFT): results
// agree with the reference to float rounding, not bit for bit.
#include "pw_common.cuh"

#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

namespace pw {
namespace ps {

constexpr int MAXSRC_PS = 64;

struct Args {
  int dim;
  int nz, nx, ny;        // expanded grid
  int nz2, nx2, ny2;     // FFT grid (real layout [ny2][nx2][nz2])
  int nb, nby;           // taper width on z / x faces, and on y faces (0 in 2-D)
  int nz1, nx1, ny1;     // interior
  float wwt;             // 1 / (nz2 nx2 ny2), float as the reference stores it
  const float *vv;       // [ny][nx][nz] expanded v^2 dt^2
  const float *wz, *wx, *wy;  // taper factor per padded index (1 off the faces)
  float *S, *P;          // modulated current / previous fields, padded layout
  const float *F;        // C2R output (unnormalised), padded layout
  int it, nt;
  int ns;
  int sz[MAXSRC_PS], sx[MAXSRC_PS], sy[MAXSRC_PS];  // expanded-grid source cells
  const float *rick;     // [ns][nt]
  int rz;                // receiver row (expanded grid)
  const float *tri_dat;  // [ny1][nx1][nt] or null
  float *rec;            // forward traces [ny1][nx1][nt] or null
  float *wfd;            // this step's snapshot [ny1][nx1][nz1] or null
};

__global__ void lapl_mul_kernel(cufftComplex *spec, const float *lapl, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float l = lapl[i];
    cufftComplex c = spec[i];
    c.x = fmul(c.x, l);
    c.y = fmul(c.y, l);
    spec[i] = c;
  }
}

__global__ void update_kernel(const Args a) {
  const long long n = (long long)a.nz * a.nx * a.ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(q % a.nz);
    const int ix = (int)((q / a.nz) % a.nx);
    const int iy = (int)(q / ((long long)a.nz * a.nx));
    const long long j = ((long long)iy * a.nx2 + ix) * a.nz2 + iz;
    const bool neg = (ix + iy) & 1;
    const float vve = a.vv[q];
    const float s = a.S[j], p = a.P[j];
    // sign * wave = wwt * F (the reference multiplies the signed wwt by F)
    float c = fadd(fadd(s, fsub(s, p)), fmul(fmul(a.wwt, a.F[j]), vve));
    if (a.tri_dat) {
      if (iz == a.rz && ix >= a.nb && ix < a.nb + a.nx1 && iy >= a.nby && iy < a.nby + a.ny1) {
        const float d = a.tri_dat[((size_t)(iy - a.nby) * a.nx1 + (ix - a.nb)) * a.nt + a.it];
        const float inj = fmul(vve, d);
        c = fadd(c, neg ? -inj : inj);
      }
    } else {
      for (int i = 0; i < a.ns; i++) {
        const int ddz = iz - a.sz[i], ddx = ix - a.sx[i], ddy = iy - a.sy[i];
        if (ddz < -1 || ddz > 1 || ddx < -1 || ddx > 1 || (a.dim == 3 && (ddy < -1 || ddy > 1)) ||
            (a.dim == 2 && ddy != 0))
          continue;
        const float den = (float)(abs(ddx) + abs(ddz) + (a.dim == 3 ? abs(ddy) : 0) + 1);
        const float inj = fdiv(fmul(vve, a.rick[(size_t)i * a.nt + a.it]), den);
        c = fadd(c, neg ? -inj : inj);
      }
    }
    const float tz = a.wz[iz], tx = a.wx[ix], ty = a.wy[iy];
    c = fmul(fmul(fmul(c, tz), tx), ty);
    a.S[j] = c;
    a.P[j] = fmul(fmul(fmul(s, tz), tx), ty);
    const float cur = neg ? -c : c;
    if (a.rec && iz == a.rz && ix >= a.nb && ix < a.nb + a.nx1 && iy >= a.nby &&
        iy < a.nby + a.ny1)
      a.rec[((size_t)(iy - a.nby) * a.nx1 + (ix - a.nb)) * a.nt + a.it] = cur;
    if (a.wfd && iz >= a.nb && iz < a.nb + a.nz1 && ix >= a.nb && ix < a.nb + a.nx1 &&
        iy >= a.nby && iy < a.nby + a.ny1)
      a.wfd[((size_t)(iy - a.nby) * a.nx1 + (ix - a.nb)) * a.nz1 + (iz - a.nb)] = cur;
  }
}

// edge-replicated expansion of the interior velocity, v^2 dt^2 as
// psm2d / psm form it ((v v) dt) dt (wave_psp.c:164-166, 484-486)
__global__ void expand_kernel(const float *vel, int nz1, int nx1, int ny1, int nb, int nby, int nz,
                              int nx, int ny, float dt, float *vv) {
  const long long n = (long long)nz * nx * ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(q % nz), ix = (int)((q / nz) % nx), iy = (int)(q / ((long long)nz * nx));
    const int jz = min(max(iz - nb, 0), nz1 - 1), jx = min(max(ix - nb, 0), nx1 - 1);
    const int jy = min(max(iy - nby, 0), ny1 - 1);
    const float v = vel[((size_t)jy * nx1 + jx) * nz1 + jz];
    vv[q] = fmul(fmul(fmul(v, v), dt), dt);
  }
}

__global__ void finite_kernel(const float *v, long long n, unsigned *bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (!(v[i] > 0.f) || !isfinite(v[i])) atomicOr(bad, 1u);
}

// abc_cal / abc_apply (wave_abc.c:134-294): per padded index the top / left
// face weight, the bottom / right one counted from the padded size, or 1
static void taper_table(int n, int n2, int nb, const std::vector<float> &w, std::vector<float> &f) {
  f.assign(n, 1.f);
  for (int i = 0; i < nb && i < n; i++) f[i] = w[i];
  for (int i = 0; i < nb; i++) {
    const int cell = n2 - 1 - i;
    if (cell >= 0 && cell < n) f[cell] = w[i];
  }
}

// -(2 pi |k|)^2 on psm2d / psm's centred grid, each quantity rounded as the
// reference rounds it (wave_psp.c:180-192, 497-508)
static void build_lapl(int dim, int nz2, int nx2, int ny2, int nkz, float dz, float dx, float dy,
                       std::vector<float> &lapl) {
  const double pi = 3.14159265358979323846264338328;
  const float dkz = 1. / (nz2 * dz), kz0 = 0.f;
  const float dkx = 1. / (nx2 * dx), kx0 = -0.5 / dx;
  const float dky = dim == 3 ? (float)(1. / (ny2 * dy)) : 0.f;
  const float ky0 = dim == 3 ? (float)(-0.5 / dy) : 0.f;
  lapl.resize((size_t)nkz * nx2 * ny2);
  for (int iy = 0; iy < ny2; iy++) {
    const float ky = ky0 + iy * dky;
    for (int ix = 0; ix < nx2; ix++) {
      const float kx = kx0 + ix * dkx;
      for (int iz = 0; iz < nkz; iz++) {
        const float kz = kz0 + iz * dkz;
        const float k = dim == 3 ? 2 * pi * std::hypot((double)ky, std::hypot((double)kx, (double)kz))
                                 : 2 * pi * std::hypot((double)kx, (double)kz);
        lapl[((size_t)iy * nx2 + ix) * nkz + iz] = -k * k;
      }
    }
  }
}

// The last grid's cuFFT plans, kept per device between calls (planning a
// 270^3 transform costs ~0.1 s); used and replaced under the device's
// workspace lock.
struct FftPlans {
  int dim = 0, nz2 = 0, nx2 = 0, ny2 = 0;
  cufftHandle fwd = 0, inv = 0;
  void reset() {
    if (fwd) cufftDestroy(fwd);
    if (inv) cufftDestroy(inv);
    fwd = inv = 0;
    dim = 0;
  }
};
static FftPlans &plans_for_device() {
  static std::mutex mu;
  static std::map<int, FftPlans> reg;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(mu);
  return reg[dev];
}

}  // namespace ps

void release_fft_plans() {
  ps::plans_for_device().reset();
}

namespace ps {

// waits for the call's stream on every return path, before the workspace
// lock (declared earlier) is released
struct DrainOnExit {
  cudaStream_t st;
  ~DrainOnExit() { cudaStreamSynchronize(st); }
};

}  // namespace ps
}  // namespace pw

using namespace pw;
using namespace pw::ps;

#define PW_CUFFT(call)                                                                  \
  do {                                                                                  \
    cufftResult r_ = (call);                                                            \
    if (r_ != CUFFT_SUCCESS) {                                                          \
      ::pw::set_error("%s:%d: %s: cuFFT error %d", __FILE__, __LINE__, #call, (int)r_); \
      return r_ == CUFFT_ALLOC_FAILED ? PW_ERR_OOM : PW_ERR_CUDA;                       \
    }                                                                                   \
  } while (0)

// aps2dc / aps3dc (aps.c:315, :22) -> psm2d / psm: arguments as pw_afd's.
extern "C" int pw_aps(const pw_afd_args *a, const float *vel, const float *src,
                      const float *wavelet, float *dat, float *wfd, void *stream) {
  PW_CHECK(a != nullptr && vel != nullptr, PW_ERR_VALUE, "null argument");
  PW_CHECK(a->dim == 2 || a->dim == 3, PW_ERR_VALUE, "dim must be 2 or 3");
  const int dim = a->dim;
  const bool tri = a->tri != 0;
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  cudaStream_t st = (cudaStream_t)stream;
  const int nz1 = a->nz, nx1 = a->nx, ny1 = dim == 3 ? a->ny : 1, nt = a->nt, nb = a->nbt;
  PW_CHECK(nz1 >= 1 && nx1 >= 1 && ny1 >= 1 && nt >= 1 && nb >= 0, PW_ERR_SHAPE,
           "sizes must be positive");
  PW_CHECK(a->jsnap >= 0, PW_ERR_VALUE, "jsnap must be >= 0");
  PW_CHECK(a->gz >= 0 && a->gz < nz1, PW_ERR_SHAPE, "receiver depth gz=%d outside [0,%d)", a->gz,
           nz1);
  const int nby = dim == 3 ? nb : 0;
  const int nz = nz1 + 2 * nb, nx = nx1 + 2 * nb, ny = ny1 + 2 * nby;
  // fft2_init / fft3_init with cmplx = 0, pad1 = 1 (wave_fft2.c:45-52, wave_fft3.c:44-60)
  const int nz2 = pad_first(nz), nx2 = next_fast(nx), ny2 = dim == 3 ? next_fast(ny) : 1;
  const int nkz = nz2 / 2 + 1;
  const size_t nreal = (size_t)nz2 * nx2 * ny2, ncplx = (size_t)nkz * nx2 * ny2;
  const size_t nexp = (size_t)nz * nx * ny, nvel = (size_t)nz1 * nx1 * ny1;
  const size_t nrec = (size_t)nx1 * ny1;
  int ntsnap = 0;
  if (a->jsnap > 0)
    for (int it = 0; it < nt; it++)
      if (it % a->jsnap == 0) ntsnap++;

  // sources (aps.c:384-412 / 93-121: positions truncated to int) and wavelets
  Args g{};
  std::vector<float> rick;
  if (!tri) {
    const int ns = a->ns;
    PW_CHECK(ns >= 0 && ns <= MAXSRC_PS, PW_ERR_SHAPE, "ns must be in [0,%d]", MAXSRC_PS);
    const int rows = dim == 2 ? 5 : 6;
    std::vector<float> s((size_t)rows * ns);
    if (ns > 0) {
      PW_CHECK(src != nullptr, PW_ERR_VALUE, "source array is null");
      if (host) memcpy(s.data(), src, s.size() * 4);
      else PW_CUDA(cudaMemcpy(s.data(), src, s.size() * 4, cudaMemcpyDeviceToHost));
    }
    rick.assign((size_t)std::max(ns, 1) * nt, 0.f);
    for (int i = 0; i < ns; i++) {
      const int spx = (int)s[i];
      const int spy = dim == 2 ? 0 : (int)s[ns + i];
      const int spz = (int)s[(dim == 2 ? 1 : 2) * ns + i];
      const float f0 = s[(rows - 3) * ns + i], t0 = s[(rows - 2) * ns + i], A = s[(rows - 1) * ns + i];
      PW_CHECK(spx >= 0 && spx < nx1 && spz >= 0 && spz < nz1 && spy >= 0 && spy < ny1,
               PW_ERR_SHAPE, "source %d at (z=%d,x=%d,y=%d) outside the model", i, spz, spx, spy);
      PW_CHECK(nb >= 1 || (spx > 0 && spx < nx1 - 1 && spz > 0 && spz < nz1 - 1 &&
                           (dim == 2 || (spy > 0 && spy < ny1 - 1))),
               PW_ERR_SHAPE, "source %d spread leaves the grid", i);
      g.sz[i] = spz + nb;
      g.sx[i] = spx + nb;
      g.sy[i] = dim == 3 ? spy + nby : 0;
      if (!wavelet) {
        PW_CHECK(t0 >= 0.f && (int)(t0 / a->dt) < nt, PW_ERR_VALUE,
                 "source %d onset t=%g outside [0, nt*dt)", i, t0);
        ricker_table(nt, a->dt, f0, t0, A, rick.data() + (size_t)i * nt);
      }
    }
    if (wavelet && ns > 0) {
      if (host) memcpy(rick.data(), wavelet, (size_t)ns * nt * 4);
      else PW_CUDA(cudaMemcpy(rick.data(), wavelet, (size_t)ns * nt * 4, cudaMemcpyDeviceToHost));
    }
    g.ns = ns;
  }
  // taper tables (abc_cal: float exponent, double exp, stored as float)
  std::vector<float> w(std::max(nb, 1));
  for (int ib = 0; ib < nb; ib++)
    w[ib] = (float)exp(-a->ct * a->ct * (nb - 1 - ib) * (nb - 1 - ib));
  std::vector<float> twz, twx, twy;
  taper_table(nz, nz2, nb, w, twz);
  taper_table(nx, nx2, nb, w, twx);
  if (dim == 3) taper_table(ny, ny2, nby, w, twy);
  else twy.assign(1, 1.f);
  std::vector<float> lapl;
  build_lapl(dim, nz2, nx2, ny2, nkz, a->dz, a->dx, a->dy, lapl);

  Carve cv;
  const size_t o_S = cv.add(nreal * 4), o_P = cv.add(nreal * 4), o_F = cv.add(nreal * 4);
  const size_t o_spec = cv.add(ncplx * sizeof(cufftComplex));
  const size_t o_lapl = cv.add(ncplx * 4);
  const size_t o_vv = cv.add(nexp * 4);
  const size_t o_tab = cv.add((twz.size() + twx.size() + twy.size()) * 4);
  const size_t o_rick = cv.add(rick.size() * 4 + 4);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_tri = cv.add(tri ? (size_t)nt * nrec * 4 : 0);
  const size_t o_rec = cv.add(!tri && dat && host ? (size_t)nt * nrec * 4 : 0);
  const size_t o_wfd = cv.add(wfd && host ? (size_t)ntsnap * nvel * 4 : 0);
  const size_t o_bad = cv.add(16);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  DrainOnExit drain{st};  // declared after the lock: drains before it is released
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  const float *d_vel = vel;
  if (host) {
    PW_TRY(to_device(base + o_vel, vel, nvel * 4, true, st));
    d_vel = at<float>(base, o_vel);
  }
  {
    unsigned *bad = at<unsigned>(base, o_bad);
    finite_kernel<<<592, 256, 0, st>>>(d_vel, (long long)nvel, bad);
    PW_CUDA(cudaGetLastError());
    unsigned hbad = 0;
    PW_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
    PW_CHECK(hbad == 0, PW_ERR_VALUE, "velocity has non-finite or non-positive values");
  }
  float *tab = at<float>(base, o_tab);
  {
    std::vector<float> all;
    for (auto *v : {&twz, &twx, &twy}) all.insert(all.end(), v->begin(), v->end());
    PW_CUDA(cudaMemcpyAsync(tab, all.data(), all.size() * 4, cudaMemcpyHostToDevice, st));
    PW_CUDA(cudaMemcpyAsync(base + o_lapl, lapl.data(), lapl.size() * 4, cudaMemcpyHostToDevice,
                            st));
    if (!tri && g.ns > 0)
      PW_CUDA(cudaMemcpyAsync(base + o_rick, rick.data(), (size_t)g.ns * nt * 4,
                              cudaMemcpyHostToDevice, st));
  }
  expand_kernel<<<592, 256, 0, st>>>(d_vel, nz1, nx1, ny1, nb, nby, nz, nx, ny, a->dt,
                                     at<float>(base, o_vv));
  PW_CUDA(cudaGetLastError());
  if (tri) {
    PW_CHECK(src != nullptr, PW_ERR_VALUE, "TRI traces are null");
    PW_TRY(to_device(base + o_tri, src, (size_t)nt * nrec * 4, host, st));
  }

  FftPlans &pl = plans_for_device();
  if (!(pl.dim == dim && pl.nz2 == nz2 && pl.nx2 == nx2 && pl.ny2 == ny2)) {
    PW_CUDA(cudaStreamSynchronize(st));  // the old plans may still be in use on a stream
    pl.reset();
    if (dim == 2) {
      PW_CUFFT(cufftPlan2d(&pl.fwd, nx2, nz2, CUFFT_R2C));
      PW_CUFFT(cufftPlan2d(&pl.inv, nx2, nz2, CUFFT_C2R));
    } else {
      PW_CUFFT(cufftPlan3d(&pl.fwd, ny2, nx2, nz2, CUFFT_R2C));
      PW_CUFFT(cufftPlan3d(&pl.inv, ny2, nx2, nz2, CUFFT_C2R));
    }
    pl.dim = dim;
    pl.nz2 = nz2;
    pl.nx2 = nx2;
    pl.ny2 = ny2;
  }
  PW_CUFFT(cufftSetStream(pl.fwd, st));
  PW_CUFFT(cufftSetStream(pl.inv, st));

  g.dim = dim;
  g.nz = nz; g.nx = nx; g.ny = ny;
  g.nz2 = nz2; g.nx2 = nx2; g.ny2 = ny2;
  g.nb = nb; g.nby = nby;
  g.nz1 = nz1; g.nx1 = nx1; g.ny1 = ny1;
  g.wwt = (float)(1.0 / ((double)nz2 * nx2 * ny2));
  g.vv = at<float>(base, o_vv);
  g.wz = tab;
  g.wx = tab + twz.size();
  g.wy = tab + twz.size() + twx.size();
  g.S = at<float>(base, o_S);
  g.P = at<float>(base, o_P);
  g.F = at<float>(base, o_F);
  g.nt = nt;
  g.rick = at<float>(base, o_rick);
  g.rz = nb + a->gz;
  g.tri_dat = tri ? at<float>(base, o_tri) : nullptr;
  float *rec = (!tri && dat) ? (host ? at<float>(base, o_rec) : dat) : nullptr;
  float *wfd_dev = wfd ? (host ? at<float>(base, o_wfd) : wfd) : nullptr;
  g.rec = rec;
  cufftComplex *spec = at<cufftComplex>(base, o_spec);
  const float *d_lapl = at<float>(base, o_lapl);
  const int ublocks = (int)std::min<long long>(ceil_div((long long)nexp, 256), 148LL * 16);
  const int mblocks = (int)std::min<long long>(ceil_div((long long)ncplx, 256), 148LL * 16);
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  for (int k = 0; k < nt; k++) {
    const int it = tri ? nt - 1 - k : k;
    PW_CUFFT(cufftExecR2C(pl.fwd, g.S, spec));
    lapl_mul_kernel<<<mblocks, 256, 0, st>>>(spec, d_lapl, (long long)ncplx);
    PW_CUDA(cudaGetLastError());
    PW_CUFFT(cufftExecC2R(pl.inv, spec, at<float>(base, o_F)));
    g.it = it;
    g.wfd = (wfd_dev && a->jsnap > 0 && it % a->jsnap == 0)
                ? wfd_dev + (size_t)(it / a->jsnap) * nvel : nullptr;
    update_kernel<<<ublocks, 256, 0, st>>>(g);
    PW_CUDA(cudaGetLastError());
    launches += 4;
  }
  timer.stop();
  if (host && rec) PW_TRY(to_host(dat, rec, (size_t)nt * nrec * 4, true, st));
  if (host && wfd_dev) PW_TRY(to_host(wfd, wfd_dev, (size_t)ntsnap * nvel * 4, true, st));
  timer.finish(launches, launches + 3);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}
