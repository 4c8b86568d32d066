// Status, workspace and host-side helpers of libpywave_b200.
#include "pw_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <map>
#include <memory>
#include <thread>

namespace pw {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

Workspace &Workspace::for_current_device() {
  static std::mutex reg_mu;
  static std::map<int, std::unique_ptr<Workspace>> reg;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(reg_mu);
  auto &p = reg[dev];
  if (!p) p.reset(new Workspace());
  return *p;
}

int Workspace::reserve(size_t bytes) {
  if (bytes <= cap_) return PW_OK;
  if (base_) {
    cudaFree(base_);
    base_ = nullptr;
    cap_ = 0;
  }
  size_t want = bytes + bytes / 8;  // headroom for slightly larger repeats
  if (cudaMalloc(&base_, want) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMalloc(&base_, bytes) != cudaSuccess) {
      cudaGetLastError();
      base_ = nullptr;
      set_error("device allocation of %zu bytes failed", bytes);
      return PW_ERR_OOM;
    }
    want = bytes;
  }
  cap_ = want;
  return PW_OK;
}

void Workspace::release() {
  if (base_) cudaFree(base_);
  base_ = nullptr;
  cap_ = 0;
}

int next_fast(int n) {
  for (;; n++) {
    int m = n;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    while (m % 5 == 0) m /= 5;
    if (m <= 1) return n;
  }
}

void ricker_table(int nt, float dt, float f0, float t0, float A, float *out) {
  // Spike of height A at k0 = (int)(t0/dt), real FFT of length nfft, times the
  // real even shape s_k = w exp(1-w)/nfft with w = (k dw)^2, inverse real FFT
  // (both unnormalised).  For one spike this is
  //   x[n] = A (s_0 + 2 sum_{0<k<nfft/2} s_k cos(2 pi k (n-k0)/nfft)
  //             + s_{nfft/2} cos(pi (n-k0)))
  const int nfft = 2 * next_fast((nt + 1) / 2);
  const int nw = nfft / 2 + 1;
  const int k0 = (int)(t0 / dt);
  const float freq = f0 * dt;
  const float dw = (float)(1. / (nfft * freq));
  std::vector<double> shape(nw), ctab(nfft);
  for (int k = 0; k < nw; k++) {
    float w = k * dw;
    w *= w;
    shape[k] = (double)(w * expf(1 - w) / nfft);
  }
  for (int j = 0; j < nfft; j++) ctab[j] = std::cos(2.0 * M_PI * (double)j / (double)nfft);
  std::vector<double> two_shape(nw);
  for (int k = 0; k < nw; k++) two_shape[k] = 2.0 * shape[k];  // exact
  // the shape underflows to exactly 0 beyond some k (expf(1-w) < 2^-149):
  // those terms add +-0, which leaves every partial sum unchanged (a sum
  // starting at +0 never becomes -0), so the loops stop at the last nonzero
  int kend = nfft / 2;
  while (kend > 1 && two_shape[kend - 1] == 0.0) kend--;
  // samples are independent: split them over host threads, and sum four
  // samples side by side (four independent chains); the phase k*m mod nfft
  // advances by m mod nfft per term (same terms, same order per sample)
  auto rows = [&](int n0, int n1) {
    int n = n0;
    for (; n + 4 <= n1; n += 4) {
      long mm[4], ph[4];
      double s[4];
      for (int i = 0; i < 4; i++) {
        const long m = n + i - k0;
        mm[i] = ((m % nfft) + nfft) % nfft;
        ph[i] = 0;
        s[i] = shape[0];
      }
      for (int k = 1; k < kend; k++) {
        const double t = two_shape[k];
        for (int i = 0; i < 4; i++) {
          ph[i] += mm[i];
          if (ph[i] >= nfft) ph[i] -= nfft;
          s[i] += t * ctab[ph[i]];
        }
      }
      for (int i = 0; i < 4; i++) {
        const long m = n + i - k0;
        long ph2 = ((long)(nfft / 2) * m) % nfft;
        if (ph2 < 0) ph2 += nfft;
        s[i] += shape[nfft / 2] * ctab[ph2];
        out[n + i] = (float)((double)A * s[i]);
      }
    }
    for (; n < n1; n++) {
      const long m = n - k0;
      const long mm = ((m % nfft) + nfft) % nfft;
      double s = shape[0];
      long ph = 0;
      for (int k = 1; k < kend; k++) {
        ph += mm;
        if (ph >= nfft) ph -= nfft;
        s += two_shape[k] * ctab[ph];
      }
      long ph2 = ((long)(nfft / 2) * m) % nfft;
      if (ph2 < 0) ph2 += nfft;
      s += shape[nfft / 2] * ctab[ph2];
      out[n] = (float)((double)A * s);
    }
  };
  const long long work = (long long)nt * kend * 2;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nthr = (int)std::min<long long>(std::min(hw, 32), std::max(1LL, work >> 19));
  if (nthr <= 1) {
    rows(0, nt);
  } else {
    std::vector<std::thread> th;
    const int chunk = (nt + nthr - 1) / nthr;
    for (int i = 0; i < nthr; i++) {
      const int n0 = i * chunk, n1 = std::min(nt, n0 + chunk);
      if (n0 < n1) th.emplace_back(rows, n0, n1);
    }
    for (auto &t : th) t.join();
  }
}

Timing &timing() {
  static thread_local Timing t;
  return t;
}

LoopTimer::LoopTimer(cudaStream_t s) : s_(s) {
  cudaEventCreate(&a_);
  cudaEventCreate(&b_);
}
LoopTimer::~LoopTimer() {
  if (a_) cudaEventDestroy(a_);
  if (b_) cudaEventDestroy(b_);
}
void LoopTimer::start() { cudaEventRecord(a_, s_); }
void LoopTimer::stop() { cudaEventRecord(b_, s_); }
void LoopTimer::finish(long long step_launches, long long total_launches) {
  float ms = 0.f;
  cudaEventSynchronize(b_);
  cudaEventElapsedTime(&ms, a_, b_);
  timing().loop_ms = ms;
  timing().step_launches = step_launches;
  timing().total_launches = total_launches;
}

int to_device(void *dst, const void *src, size_t bytes, bool host, cudaStream_t s) {
  if (bytes == 0) return PW_OK;
  PW_CUDA(cudaMemcpyAsync(dst, src, bytes, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  return PW_OK;
}

int to_host(void *dst, const void *src, size_t bytes, bool host, cudaStream_t s) {
  if (bytes == 0) return PW_OK;
  PW_CUDA(cudaMemcpyAsync(dst, src, bytes, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
  return PW_OK;
}

}  // namespace pw

extern "C" const char *pw_last_error(void) { return pw::g_last_error.c_str(); }

extern "C" const char *pw_version(void) { return "pywave_b200 0.1 (sm_100a)"; }

extern "C" int pw_last_timing(double *loop_ms, long long *step_launches,
                              long long *total_launches) {
  if (loop_ms) *loop_ms = pw::timing().loop_ms;
  if (step_launches) *step_launches = pw::timing().step_launches;
  if (total_launches) *total_launches = pw::timing().total_launches;
  return PW_OK;
}

extern "C" int pw_release_cache(void) {
  auto &ws = pw::Workspace::for_current_device();
  std::lock_guard<std::mutex> g(ws.mutex());
  cudaDeviceSynchronize();
  pw::release_fft_plans();
  ws.release();
  return PW_OK;
}
