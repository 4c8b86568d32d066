// Shared internals of libpywave_b200: status handling, the per-device
// workspace, exact-rounding float helpers and small host utilities.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <mutex>

#include "../../include/pywave_b200.h"

namespace pw {

// ---------------------------------------------------------------- errors --
void set_error(const char *fmt, ...);

struct Status {
  int code = PW_OK;
  bool ok() const { return code == PW_OK; }
};

#define PW_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      ::pw::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,             \
                      cudaGetErrorString(e_));                                \
      return e_ == cudaErrorMemoryAllocation ? PW_ERR_OOM : PW_ERR_CUDA;      \
    }                                                                         \
  } while (0)

#define PW_CHECK(cond, code, ...)                                             \
  do {                                                                        \
    if (!(cond)) {                                                            \
      ::pw::set_error(__VA_ARGS__);                                           \
      return (code);                                                          \
    }                                                                         \
  } while (0)

#define PW_TRY(expr)                                                          \
  do {                                                                        \
    int rc_ = (expr);                                                         \
    if (rc_ != PW_OK) return rc_;                                             \
  } while (0)

// ------------------------------------------------------------ workspace --
// One grow-only device allocation per device, carved into 256-byte aligned
// slices per call.  A call holds the device's lock from carve to its final
// stream synchronisation, so concurrent calls serialise instead of aliasing.
class Workspace {
 public:
  static Workspace &for_current_device();
  // Reserve `bytes` (rounded); returns PW_OK or PW_ERR_OOM.
  int reserve(size_t bytes);
  char *base() const { return base_; }
  size_t capacity() const { return cap_; }
  void release();
  std::mutex &mutex() { return mu_; }

 private:
  char *base_ = nullptr;
  size_t cap_ = 0;
  std::mutex mu_;
};

// Builds a slice layout first (sizes), then binds to the workspace base.
class Carve {
 public:
  size_t add(size_t bytes) {
    size_t off = total_;
    total_ += (bytes + 255) & ~size_t(255);
    return off;
  }
  size_t total() const { return total_; }

 private:
  size_t total_ = 0;
};

template <class T>
inline T *at(char *base, size_t off) { return reinterpret_cast<T *>(base + off); }

// ------------------------------------------------------------- helpers ----
inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }
inline long long round_up(long long a, long long b) { return (a + b - 1) / b * b; }

// kiss_fft_next_fast_size (pywave/src/wave_kissfft.c:412-424): the smallest
// n' >= n with no prime factor other than 2, 3, 5.
int next_fast(int n);
// First-axis padding of fft2_init/fft3_init with cmplx=0, pad1=1
// (pywave/src/wave_fft2.c:45-46): 2*next_fast((n+1)/2).
inline int pad_first(int n) { return 2 * next_fast((n + 1) / 2); }

// The Ricker table of fdm2d/fdm (pywave/src/wave_fdm.c:502-516; shape
// wave_ricker.c:22-58; zero-phase filter wave_freqfilt.c:76-99), evaluated as
// the closed-form cosine sum of the spike's filtered spectrum in double, with
// the spectral shape samples rounded to float as the reference stores them.
void ricker_table(int nt, float dt, float f0, float t0, float A, float *out);

// Per-thread record of the last call's device timing (pw_last_timing).
struct Timing {
  double loop_ms = 0;
  long long step_launches = 0;
  long long total_launches = 0;
};
Timing &timing();
// RAII pair of CUDA events bracketing a time loop on a stream.
class LoopTimer {
 public:
  explicit LoopTimer(cudaStream_t s);
  ~LoopTimer();
  void start();
  void stop();
  // Synchronises on the stop event and stores the elapsed time in timing().
  void finish(long long step_launches, long long total_launches);

 private:
  cudaStream_t s_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
};

// Destroys the calling device's cached cuFFT plans (psm.cu); the caller
// holds the device's workspace lock.
void release_fft_plans();

// Copy helper honouring PW_HOST_PTRS.
int to_device(void *dst, const void *src, size_t bytes, bool host, cudaStream_t s);
int to_host(void *dst, const void *src, size_t bytes, bool host, cudaStream_t s);

}  // namespace pw

// ------------------------------------------------- device-side helpers ----
// Explicitly rounded float ops: the parity-critical expressions are written
// with these so that nvcc never contracts a*b+c into an FMA, which keeps the
// evaluation order (and rounding) of the reference's C code.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// Packed pairs of floats for sm_100's f32x2 pipe: add / sub / mul.rn.f32x2
// round each lane exactly as the scalar __fadd_rn / __fsub_rn / __fmul_rn.
// Unlike the scalar .rn forms, a packed multiply whose result feeds a packed
// add is fused by the assembler into one FMA (one rounding instead of two,
// with or without -fmad=false), so every product that is added is first
// multiplied by a runtime 1.0 (a kernel argument the compiler cannot fold):
// the fused form p * 1 + t then rounds exactly as the separate add.
typedef unsigned long long f2;
__device__ __forceinline__ f2 pk2(float a, float b) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void up2(f2 r, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// fused a * b + c per lane, one rounding (fma.rn.f32x2)
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ f2 lo2(const float4 &v) { return pk2(v.x, v.y); }
__device__ __forceinline__ f2 hi2(const float4 &v) { return pk2(v.z, v.w); }
__device__ __forceinline__ float4 join2(f2 l, f2 h) {
  float4 r;
  up2(l, r.x, r.y);
  up2(h, r.z, r.w);
  return r;
}
