// FWI driver: L-BFGS with the reference's Wolfe line search
// (pywave/src/wave_fwi.c:24-119, wave_fwilbfgs.c:9-165), every inner product
// and norm in FP64 on the GPU; model, gradient and L-BFGS pairs stay float32
// in HBM as the reference keeps them.
#include "pw_common.cuh"

#include <cmath>
#include <vector>

namespace pw {
namespace lb {

// sum(a[i]*b[i]) in FP64, deterministic: a fixed grid of DOT_BLOCKS blocks
// of DOT_THREADS threads, each thread a grid-stride partial sum, each block a
// fixed shared-memory tree into part[block]; dot_final_kernel then adds the
// block sums in block order.  The same inputs give the same bits on every run
// (no atomics), so the line search takes the same decisions every time.
constexpr int DOT_BLOCKS = 296, DOT_THREADS = 256;

__global__ void __launch_bounds__(DOT_THREADS) dot_kernel(const float *a, const float *b,
                                                          long long n, double *part) {
  __shared__ double sh[DOT_THREADS];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)DOT_THREADS + threadIdx.x; i < n;
       i += (long long)DOT_BLOCKS * DOT_THREADS)
    s = __dadd_rn(s, __dmul_rn((double)a[i], (double)b[i]));
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = DOT_THREADS / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void dot_final_kernel(const double *part, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < DOT_BLOCKS; k++) s = __dadd_rn(s, part[k]);
    *out = s;
  }
}

// y = a*x + b*y (FP64 coefficients and arithmetic, no contraction; float32 storage)
__global__ void axpby_kernel(double a, const float *x, double b, float *y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)__dadd_rn(__dmul_rn(a, (double)x[i]), __dmul_rn(b, (double)y[i]));
}

// x = clip(xk + alpha*d, lo, hi) (line_search, wave_fwilbfgs.c:125-128)
__global__ void trial_kernel(const float *xk, const float *d, float alpha, float lo, float hi,
                             float *x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    // the product rounded on its own, as the reference's C evaluates it
    float v = __fadd_rn(xk[i], __fmul_rn(alpha, d[i]));
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    x[i] = v;
  }
}

__global__ void sub_kernel(const float *a, float *b, long long n) {  // b = a - b
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i] - b[i];
}

struct Dev {
  cudaStream_t st;
  long long n;
  double *acc;  // device scalars: DOT_BLOCKS block sums, then the total
  int dot(const float *a, const float *b, double *out) {
    dot_kernel<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(a, b, n, acc);
    dot_final_kernel<<<1, 32, 0, st>>>(acc, acc + DOT_BLOCKS);
    PW_CUDA(cudaGetLastError());
    PW_CUDA(cudaMemcpyAsync(out, acc + DOT_BLOCKS, 8, cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
    return PW_OK;
  }
  int axpby(double a, const float *x, double b, float *y) {
    axpby_kernel<<<592, 256, 0, st>>>(a, x, b, y, n);
    PW_CUDA(cudaGetLastError());
    return PW_OK;
  }
  int copy(const float *src, float *dst) {
    PW_CUDA(cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToDevice, st));
    return PW_OK;
  }
};

struct Buffers {
  std::vector<void *> ptrs;
  ~Buffers() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <class T>
  int alloc(T **p, size_t count) {
    void *q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      set_error("device allocation of %zu bytes failed", count * sizeof(T));
      return PW_ERR_OOM;
    }
    ptrs.push_back(q);
    *p = static_cast<T *>(q);
    return PW_OK;
  }
};

}  // namespace lb
}  // namespace pw

using namespace pw;
using namespace pw::lb;

// fwi (wave_fwi.c:24-119; wav: point sources, gradient_av) and pfwi
// (wave_fwi.c:212-322; dsrc: a source field per shot, gradient_pas_av, and
// alpha reset to 1 every `repeat` iterations, optpar->repeat = 5 in pfwic)
static int fwi_impl(const pw_fwi_args *a, const float *vel0, const float *wav, const float *dsrc,
                    const float *dobs, float *vinv, int *iters_done, int repeat, void *stream) {
  PW_CHECK(a && vel0 && (wav || dsrc) && dobs && vinv, PW_ERR_VALUE, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const long long n = (long long)a->nz * a->nx;
  const int niter = a->niter;
  // fwic's optimiser settings (pfwi.c:834-860)
  const int npair = 20, nls = 20, rect = 3, waterz = 0;
  const float c1 = 1e-4f, c2 = 0.9f, factor = 10.f, v1 = 0.f, v2 = 10.f, conv_error = 0.01f;
  Buffers B;
  float *x, *g, *d, *xk, *sk, *yk, *q, *wav_d = nullptr, *dobs_d = nullptr, *dsrc_d = nullptr;
  double *acc;
  PW_TRY(B.alloc(&x, n));
  PW_TRY(B.alloc(&g, n));
  PW_TRY(B.alloc(&d, n));
  PW_TRY(B.alloc(&xk, n));
  PW_TRY(B.alloc(&q, n));
  PW_TRY(B.alloc(&sk, n * npair));
  PW_TRY(B.alloc(&yk, n * npair));
  PW_TRY(B.alloc(&acc, DOT_BLOCKS + 1));
  const long long nd = (long long)a->ns * a->nx * a->nt;
  const long long nsf = (long long)a->ns * n * a->nt;  // passive source fields
  if (host) {
    if (wav) {
      PW_TRY(B.alloc(&wav_d, a->nt));
      PW_CUDA(cudaMemcpyAsync(wav_d, wav, a->nt * 4, cudaMemcpyHostToDevice, st));
    }
    if (dsrc) {
      PW_TRY(B.alloc(&dsrc_d, nsf));
      PW_CUDA(cudaMemcpyAsync(dsrc_d, dsrc, (size_t)nsf * 4, cudaMemcpyHostToDevice, st));
    }
    PW_TRY(B.alloc(&dobs_d, nd));
    PW_CUDA(cudaMemcpyAsync(dobs_d, dobs, nd * 4, cudaMemcpyHostToDevice, st));
  }
  PW_TRY(to_device(x, vel0, n * 4, host, st));
  pw_fwi_args ga = *a;
  ga.flags &= ~PW_HOST_PTRS;
  const float *gwav = host ? wav_d : wav, *gdobs = host ? dobs_d : dobs;
  const float *gdsrc = host ? dsrc_d : dsrc;
  float scaling = 0.f;  // gradient_av's static: set by the first gradient
  float *dsc;
  PW_TRY(B.alloc(&dsc, 1));
  Dev D{st, n, acc};
  // gradient_av + gradient_smooth2 (wave_fwigradient.c:93-255), or
  // gradient_pas_av + gradient_smooth2b (:667-870; waterz = waterzb = 0
  // there, so the two smoothings coincide)
  auto gradient = [&](float *xv, float *fcost) -> int {
    double J = 0.0;
    if (gdsrc)
      PW_TRY(pw_pfwi_gradient_passive(&ga, PW_GRAD_REFERENCE, xv, gdsrc, gdobs, nullptr, g, &J, 0,
                                      st));
    else
      PW_TRY(pw_pfwi_gradient(&ga, PW_GRAD_REFERENCE, xv, gwav, gdobs, nullptr, g, &J, 0, st));
    PW_CUDA(cudaMemcpyAsync(dsc, &scaling, 4, cudaMemcpyHostToDevice, st));
    PW_TRY(pw_gradient_postprocess(a->nz, a->nx, rect, waterz, g, dsc, 0, st));
    PW_CUDA(cudaMemcpyAsync(&scaling, dsc, 4, cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
    *fcost = (float)J;
    return PW_OK;
  };
  float fcost = 0.f;
  PW_TRY(gradient(x, &fcost));
  float fk = fcost;
  const float f0 = fcost;
  float alpha = 1.f;
  int ipair = 0;
  int iter = 0;
  if (!host) PW_CUDA(cudaMemsetAsync(vinv, 0, (size_t)n * niter * 4, st));
  else memset(vinv, 0, (size_t)n * niter * 4);
  for (iter = 0; iter < niter; iter++) {
    if (repeat > 0 && iter % repeat == 0) alpha = 1.f;
    if (iter == 0) {
      PW_TRY(D.axpby(-1.0, g, 0.0, d));
    } else {
      // lbfgs_update (wave_fwilbfgs.c:27-36)
      const int j = ipair - 1;
      sub_kernel<<<592, 256, 0, st>>>(x, sk + (size_t)j * n, n);
      sub_kernel<<<592, 256, 0, st>>>(g, yk + (size_t)j * n, n);
      PW_CUDA(cudaGetLastError());
      // lbfgs_direction (wave_fwilbfgs.c:38-95), FP64 inner products
      double ss, yy;
      PW_TRY(D.dot(sk + (size_t)j * n, sk + (size_t)j * n, &ss));
      PW_TRY(D.dot(yk + (size_t)j * n, yk + (size_t)j * n, &yy));
      if (ss == 0.0 || yy == 0.0) {
        PW_TRY(D.axpby(-1.0, g, 0.0, d));
      } else {
        std::vector<double> rho(ipair), al(ipair);
        PW_TRY(D.copy(g, q));
        for (int i = ipair - 1; i >= 0; i--) {
          double ys, sq;
          PW_TRY(D.dot(yk + (size_t)i * n, sk + (size_t)i * n, &ys));
          rho[i] = 1.0 / ys;
          PW_TRY(D.dot(sk + (size_t)i * n, q, &sq));
          al[i] = rho[i] * sq;
          PW_TRY(D.axpby(-al[i], yk + (size_t)i * n, 1.0, q));
        }
        const double gamma = 1.0 / yy / rho[ipair - 1];
        PW_TRY(D.axpby(gamma, q, 0.0, d));
        for (int i = 0; i < ipair; i++) {
          double yr;
          PW_TRY(D.dot(yk + (size_t)i * n, d, &yr));
          const double beta = yr * rho[i];
          PW_TRY(D.axpby(al[i] - beta, sk + (size_t)i * n, 1.0, d));
        }
        PW_TRY(D.axpby(0.0, d, -1.0, d));
      }
    }
    // lbfgs_save (wave_fwilbfgs.c:9-25)
    if (ipair < npair) {
      PW_TRY(D.copy(x, sk + (size_t)ipair * n));
      PW_TRY(D.copy(g, yk + (size_t)ipair * n));
      ipair++;
    } else {
      for (int i = 0; i < npair - 1; i++) {
        PW_TRY(D.copy(sk + (size_t)(i + 1) * n, sk + (size_t)i * n));
        PW_TRY(D.copy(yk + (size_t)(i + 1) * n, yk + (size_t)i * n));
      }
      PW_TRY(D.copy(x, sk + (size_t)(npair - 1) * n));
      PW_TRY(D.copy(g, yk + (size_t)(npair - 1) * n));
    }
    // line_search (wave_fwilbfgs.c:108-165)
    PW_TRY(D.copy(x, xk));
    double m1d;
    PW_TRY(D.dot(g, d, &m1d));
    const double m2 = m1d * c2, m1 = m1d * c1;
    float alpha1 = 0.f, alpha2 = 0.f;
    int flag = 0, i;
    for (i = 0; i < nls; i++) {
      trial_kernel<<<592, 256, 0, st>>>(xk, d, alpha, v1, v2, x, n);
      PW_CUDA(cudaGetLastError());
      PW_TRY(gradient(x, &fcost));
      double m3;
      PW_TRY(D.dot(g, d, &m3));
      if (fcost <= fk + alpha * m1 && m3 >= m2) {
        fk = fcost;
        flag = 0;
        break;
      } else if (fcost > fk + alpha * m1) {
        alpha2 = alpha;
        alpha = 0.5f * (alpha1 + alpha2);
      } else {
        alpha1 = alpha;
        if (alpha2 == 0.f) alpha *= factor;
        else alpha = 0.5f * (alpha1 + alpha2);
      }
    }
    if (i == nls) flag = fcost <= fk ? 1 : 2;
    if (flag == 2) break;            // "Line Search Failed"
    if (fk / f0 < conv_error) break;  // "Convergence Criterion Reached"
    PW_TRY(to_host(vinv + (size_t)iter * n, x, n * 4, host, st));
  }
  PW_CUDA(cudaStreamSynchronize(st));
  if (iters_done) *iters_done = iter;
  return PW_OK;
}

extern "C" int pw_fwi(const pw_fwi_args *a, const float *vel0, const float *wav, const float *dobs,
                      float *vinv, int *iters_done, void *stream) {
  PW_CHECK(wav != nullptr, PW_ERR_VALUE, "null wavelet");
  return fwi_impl(a, vel0, wav, nullptr, dobs, vinv, iters_done, 0, stream);
}

extern "C" int pw_pfwi_passive(const pw_fwi_args *a, const float *vel0, const float *src,
                               const float *dobs, float *vinv, int *iters_done, void *stream) {
  PW_CHECK(src != nullptr, PW_ERR_VALUE, "null source field");
  return fwi_impl(a, vel0, nullptr, src, dobs, vinv, iters_done, 5, stream);
}
