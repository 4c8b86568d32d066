// afd propagator on sm_100a: forward modelling, time reversal, and lockstep
// multi-group TRI imaging.  One fused kernel per time step covers
//   4th-order Laplacian -> leapfrog -> injection -> double taper ->
//   receiver sampling -> snapshot / image accumulation
// of the reference's fdm2d / fdm time loop (pywave/src/wave_fdm.c:551-662,
// 209-354) with its exact float evaluation order.
//
// Device layout ("field layout"): every field is a zero-haloed array
//   off(iz,ix,iy) = (iz + HZ) + lz*(ix + hx) + sy*(iy + hy),
// z fastest, lz a multiple of 32 floats, so each thread owns one aligned
// float4 of 4 consecutive z cells.  The halo cells are never written and stay
// zero, which reproduces the reference's zero border beyond the expanded grid.
//
// Two buffers per wavefield: at step k the kernel reads A = u_k and B =
// u_{k-1} (as stored, tapered once) and overwrites B with u_{k+1}.  The
// reference's `prev` array is taper(u_{k-1}) (wave_fdm.c:595-597,633-636); it
// is recomputed on the fly from B with the same multiplications, so the scheme
// moves 16 bytes per point update (read A, B, vv; write B).
#include "pw_common.cuh"

#include <algorithm>
#include <cmath>

namespace pw {
namespace afd {

constexpr int HZ = 4;       // z halo (cells) in front of iz = 0
constexpr int MAXG = 4;     // receiver groups propagated in lockstep per launch
constexpr int MAXSRC = 16;  // point sources resolved inside the kernel

struct Geo {
  int nz, nx, ny;                    // expanded extents (interior + 2*nbt)
  int lz, px, py;                    // allocation: leading dim, x extent, y extent
  int hx, hy;                        // x / y halo widths
  long long sy;                      // y-plane stride = lz*px
  int lz0, lz1, lx0, lx1, ly0, ly1;  // Laplacian is non-zero on [lo,hi) per axis
};

__host__ __device__ inline long long foff(const Geo &g, int iz, int ix, int iy) {
  return (long long)(iz + HZ) + (long long)g.lz * (ix + g.hx) + g.sy * (iy + g.hy);
}

struct StepArgs {
  Geo g;
  int tz4, tx, ych;  // tile: float4 columns along z, columns along x, planes per CTA along y
  float c0, c1, c2, idx, idy, idz, k0;
  const float *cur[MAXG];
  float *nxt[MAXG];
  const float *vv;
  const float *wz1, *wz2, *wx1, *wx2, *wy1, *wy2;  // taper factors (1 outside the faces)
  int it, nt;
  int ns;
  int sz[MAXSRC], sx[MAXSRC], sy[MAXSRC];
  const float *rick;  // [ns][nt]
  int rz, rx0, ry0, nrx, nry;
  const float *tri_dat;  // [nt][nry][nrx]
  const int *gid;        // [nry][nrx] or null: every receiver feeds group 0
  float *rec;            // forward traces [nt][nry][nrx] or null
  int nb, nz1, nx1, ny1, nby;
  float *wfd;            // this step's snapshot [ny1][nx1][nz1] (group 0) or null
  float *img;            // image accumulator (field layout) or null
};

__device__ __forceinline__ float4 ld4(const float *base, const Geo &g, int z4, int ix, int iy) {
  if (z4 < -1 || z4 * 4 >= g.nz || ix < -g.hx || ix >= g.nx + g.hx || iy < -g.hy ||
      iy >= g.ny + g.hy)
    return make_float4(0.f, 0.f, 0.f, 0.f);
  return __ldg(reinterpret_cast<const float4 *>(base + foff(g, z4 * 4, ix, iy)));
}

__device__ __forceinline__ float el(const float4 &v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_el(float4 &v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}

template <int DIM, int G, bool TRI>
__global__ void __launch_bounds__(DIM == 3 ? 256 : 512) step_kernel(const StepArgs a) {
  extern __shared__ float4 smem[];
  const Geo &g = a.g;
  const int tz4 = a.tz4, tx = a.tx;
  const int W = tz4 + 2;
  const int plane4 = W * (tx + 4);
  const int tid = threadIdx.x;
  const int zl = tid % tz4, xl = tid / tz4;
  const int z4 = blockIdx.x * tz4 + zl;
  const int iz0 = z4 * 4;
  const int ix = blockIdx.y * tx + xl;
  const bool live = (iz0 < g.nz) && (ix < g.nx);
  const int y_begin = DIM == 3 ? blockIdx.z * a.ych : 0;
  const int y_end = DIM == 3 ? min(g.ny, y_begin + a.ych) : 1;
  const int nh = 4 * W + 2 * tx;

  float wz1[4], wz2[4];
  bool lzok[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = iz0 + e;
    const bool in = live && iz < g.nz;
    wz1[e] = in ? a.wz1[iz] : 1.f;
    wz2[e] = in ? a.wz2[iz] : 1.f;
    lzok[e] = iz >= g.lz0 && iz < g.lz1;
  }
  const float wx1 = live ? a.wx1[ix] : 1.f, wx2 = live ? a.wx2[ix] : 1.f;
  const bool lxok = ix >= g.lx0 && ix < g.lx1;
  const bool rec_x = ix >= a.rx0 && ix < a.rx0 + a.nrx;
  const bool rec_z = a.rz >= iz0 && a.rz < iz0 + 4;

  float4 q[G][5];
#pragma unroll
  for (int gi = 0; gi < G; gi++)
#pragma unroll
    for (int k = 0; k < 5; k++) q[gi][k] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (DIM == 3) {
#pragma unroll
    for (int gi = 0; gi < G; gi++)
#pragma unroll
      for (int k = 0; k < 4; k++) q[gi][k] = ld4(a.cur[gi], g, z4, ix, y_begin - 2 + k);
  }

  int parity = 0;
  for (int y = y_begin; y < y_end; y++, parity ^= 1) {
    float4 *buf = smem + parity * G * plane4;
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      if (DIM == 3) q[gi][4] = ld4(a.cur[gi], g, z4, ix, y + 2);
      else q[gi][2] = ld4(a.cur[gi], g, z4, ix, y);
      buf[gi * plane4 + (xl + 2) * W + zl + 1] = q[gi][2];
    }
    for (int h = tid; h < nh; h += blockDim.x) {
      int r, c;
      if (h < 4 * W) {
        const int rr = h / W;
        r = rr < 2 ? rr : tx + rr;
        c = h % W;
      } else {
        const int h2 = h - 4 * W;
        r = 2 + (h2 >> 1);
        c = (h2 & 1) ? tz4 + 1 : 0;
      }
      const int z4g = blockIdx.x * tz4 + c - 1;
      const int xg = blockIdx.y * tx + r - 2;
#pragma unroll
      for (int gi = 0; gi < G; gi++) buf[gi * plane4 + r * W + c] = ld4(a.cur[gi], g, z4g, xg, y);
    }
    float4 pv[G];
    float4 vvv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
#pragma unroll
      for (int gi = 0; gi < G; gi++)
        pv[gi] = *reinterpret_cast<const float4 *>(a.nxt[gi] + foff(g, iz0, ix, y));
      vvv = ld4(a.vv, g, z4, ix, y);
    }
    __syncthreads();
    if (live) {
      const bool lyok = DIM == 2 || (y >= g.ly0 && y < g.ly1);
      const float wy1 = DIM == 3 ? a.wy1[y] : 1.f, wy2 = DIM == 3 ? a.wy2[y] : 1.f;
      const long long o = foff(g, iz0, ix, y);
      const bool rec_here = rec_z && rec_x && (DIM == 2 || (y >= a.ry0 && y < a.ry0 + a.nry));
      const int r_idx = rec_here ? (DIM == 3 ? (y - a.ry0) * a.nrx : 0) + (ix - a.rx0) : 0;
      const bool interior = (ix >= a.nb && ix < a.nb + a.nx1) &&
                            (DIM == 2 || (y >= a.nby && y < a.nby + a.ny1));
      float4 outv[G];
#pragma unroll
      for (int gi = 0; gi < G; gi++) {
        const float4 *row = buf + gi * plane4;
        const float4 c = q[gi][2];
        const float4 L = row[(xl + 2) * W + zl];
        const float4 Rr = row[(xl + 2) * W + zl + 2];
        const float4 xm1 = row[(xl + 1) * W + zl + 1], xp1 = row[(xl + 3) * W + zl + 1];
        const float4 xm2 = row[xl * W + zl + 1], xp2 = row[(xl + 4) * W + zl + 1];
        float4 res;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          const float cv = el(c, e);
          const float zm1 = e == 0 ? L.w : el(c, e - 1);
          const float zp1 = e == 3 ? Rr.x : el(c, e + 1);
          const float zm2 = e == 0 ? L.z : (e == 1 ? L.w : el(c, e - 2));
          const float zp2 = e == 2 ? Rr.x : (e == 3 ? Rr.y : el(c, e + 2));
          float t = fmul(fmul(a.c0, cv), a.k0);
          if (DIM == 3) {
            t = fadd(t, fmul(fmul(a.c1, fadd(el(q[gi][1], e), el(q[gi][3], e))), a.idy));
            t = fadd(t, fmul(fmul(a.c2, fadd(el(q[gi][0], e), el(q[gi][4], e))), a.idy));
          }
          t = fadd(t, fmul(fmul(a.c1, fadd(el(xm1, e), el(xp1, e))), a.idx));
          t = fadd(t, fmul(fmul(a.c2, fadd(el(xm2, e), el(xp2, e))), a.idx));
          t = fadd(t, fmul(fmul(a.c1, fadd(zm1, zp1)), a.idz));
          t = fadd(t, fmul(fmul(a.c2, fadd(zm2, zp2)), a.idz));
          const float lap = (lzok[e] && lxok && lyok) ? t : 0.f;
          // prev = taper(u_{k-1} as stored)
          float p = el(pv[gi], e);
          p = fmul(fmul(fmul(fmul(p, wz1[e]), wz2[e]), wx1), wx2);
          if (DIM == 3) p = fmul(fmul(p, wy1), wy2);
          const float vve = el(vvv, e);
          float v = fadd(cv, fsub(cv, p));
          v = fadd(v, fmul(lap, vve));
          if (TRI) {
            if (rec_here && iz == a.rz && (a.gid == nullptr ? gi == 0 : a.gid[r_idx] == gi))
              v = fadd(v, fmul(vve, a.tri_dat[(size_t)a.it * a.nrx * a.nry + r_idx]));
          } else {
            for (int s = 0; s < a.ns; s++) {
              const int dz = iz - a.sz[s], dxs = ix - a.sx[s], dys = DIM == 3 ? y - a.sy[s] : 0;
              if (dz >= -1 && dz <= 1 && dxs >= -1 && dxs <= 1 && dys >= -1 && dys <= 1) {
                const float den = (float)(abs(dxs) + abs(dys) + abs(dz) + 1);
                v = fadd(v, fdiv(fmul(vve, a.rick[(size_t)s * a.nt + a.it]), den));
              }
            }
          }
          v = fmul(fmul(fmul(fmul(v, wz1[e]), wz2[e]), wx1), wx2);
          if (DIM == 3) v = fmul(fmul(v, wy1), wy2);
          if (iz >= g.nz) v = 0.f;
          set_el(res, e, v);
          if (!TRI && gi == 0 && rec_here && iz == a.rz && a.rec)
            a.rec[(size_t)a.it * a.nrx * a.nry + r_idx] = v;
          if (gi == 0 && a.wfd && interior && iz >= a.nb && iz < a.nb + a.nz1)
            a.wfd[((size_t)(DIM == 3 ? y - a.nby : 0) * a.nx1 + (ix - a.nb)) * a.nz1 + (iz - a.nb)] = v;
        }
        outv[gi] = res;
        *reinterpret_cast<float4 *>(a.nxt[gi] + o) = res;
      }
      if (a.img && interior) {
        float4 im = *reinterpret_cast<const float4 *>(a.img + o);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          if (iz >= a.nb && iz < a.nb + a.nz1) {
            float prod = 1.f;
#pragma unroll
            for (int gi = 0; gi < G; gi++) prod = fmul(fmul(prod, el(outv[gi], e)), el(outv[gi], e));
            set_el(im, e, fadd(el(im, e), prod));
          }
        }
        *reinterpret_cast<float4 *>(a.img + o) = im;
      }
    }
    if (DIM == 3) {
#pragma unroll
      for (int gi = 0; gi < G; gi++) {
        q[gi][0] = q[gi][1];
        q[gi][1] = q[gi][2];
        q[gi][2] = q[gi][3];
        q[gi][3] = q[gi][4];
      }
    }
  }
}

// vv = ((v*v)*dt)*dt on the expanded grid with edge replication of the
// interior velocity (vel_expand, wave_abc.c:14-125; wave_fdm.c:173-175).
__global__ void expand_vv_kernel(Geo g, const float *vel, int nz1, int nx1, int ny1, int nb,
                                 int nby, float dt, float *vv) {
  const long long n = (long long)g.nz * g.nx * g.ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % g.nz);
    const int ix = int((i / g.nz) % g.nx);
    const int iy = int(i / ((long long)g.nz * g.nx));
    int jz = min(max(iz - nb, 0), nz1 - 1);
    int jx = min(max(ix - nb, 0), nx1 - 1);
    int jy = min(max(iy - nby, 0), ny1 - 1);
    const float v = vel[((size_t)jy * nx1 + jx) * nz1 + jz];
    vv[foff(g, iz, ix, iy)] = fmul(fmul(fmul(v, v), dt), dt);
  }
}

// [rows][cols] -> [cols][rows] through a 32x33 shared tile.
__global__ void transpose_kernel(const float *in, float *out, long long rows, long long cols) {
  __shared__ float t[32][33];
  const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long r = r0 + j, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[j][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long c = c0 + j, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = t[threadIdx.x][j];
  }
}

// interior cells of a field-layout array -> [ny1][nx1][nz1]
__global__ void extract_kernel(Geo g, const float *f, int nb, int nby, int nz1, int nx1, int ny1,
                               float *out) {
  const long long n = (long long)nz1 * nx1 * ny1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % nz1);
    const int ix = int((i / nz1) % nx1);
    const int iy = int(i / ((long long)nz1 * nx1));
    out[i] = f[foff(g, iz + nb, ix + nb, iy + nby)];
  }
}

__global__ void absmax_kernel(const float *x, long long n, unsigned int *out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void scale_by_max_kernel(float *x, long long n, const unsigned int *mx) {
  const float m = __uint_as_float(*mx);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = m > 0.f ? fdiv(x[i], m) : x[i];
}

// ------------------------------------------------------------------ host --

struct Plan {
  int dim;
  int nz1, nx1, ny1, nb, nby;
  Geo g;
  int nz2, nx2, ny2;
  int tz4, tx, ych;
  dim3 grid;
  int threads;
  size_t smem_per_g;
};

static int make_plan(const pw_afd_args *a, Plan &p) {
  PW_CHECK(a->dim == 2 || a->dim == 3, PW_ERR_SHAPE, "dim must be 2 or 3 (got %d)", a->dim);
  PW_CHECK(a->nz >= 1 && a->nx >= 1 && a->ny >= 1 && a->nt >= 1 && a->nbt >= 0, PW_ERR_SHAPE,
           "sizes must be positive (nz=%d nx=%d ny=%d nt=%d nbt=%d)", a->nz, a->nx, a->ny, a->nt,
           a->nbt);
  PW_CHECK(a->dim == 3 || a->ny == 1, PW_ERR_SHAPE, "2-D runs need ny = 1 (got %d)", a->ny);
  p.dim = a->dim;
  p.nz1 = a->nz;
  p.nx1 = a->nx;
  p.ny1 = a->ny;
  p.nb = a->nbt;
  p.nby = a->dim == 3 ? a->nbt : 0;
  Geo &g = p.g;
  g.nz = p.nz1 + 2 * p.nb;
  g.nx = p.nx1 + 2 * p.nb;
  g.ny = a->dim == 3 ? p.ny1 + 2 * p.nb : 1;
  p.nz2 = pad_first(g.nz);
  p.nx2 = next_fast(g.nx);
  p.ny2 = a->dim == 3 ? next_fast(g.ny) : 1;
  // faces must not overlap inside the padded grid (abc_apply's top/bottom
  // and left/right strips are disjoint whenever the interior is non-empty)
  PW_CHECK(p.nz2 >= 2 * p.nb && p.nx2 >= 2 * p.nb && (a->dim == 2 || p.ny2 >= 2 * p.nb),
           PW_ERR_SHAPE, "taper faces overlap");
  g.hx = 2;
  g.hy = a->dim == 3 ? 2 : 0;
  g.lz = (int)round_up(HZ + round_up(g.nz, 4) + 4, 32);
  g.px = g.nx + 2 * g.hx;
  g.py = g.ny + 2 * g.hy;
  g.sy = (long long)g.lz * g.px;
  g.lz0 = 2;
  g.lz1 = std::min(g.nz, p.nz2 - 2);
  g.lx0 = 2;
  g.lx1 = std::min(g.nx, p.nx2 - 2);
  g.ly0 = a->dim == 3 ? 2 : 0;
  g.ly1 = a->dim == 3 ? std::min(g.ny, p.ny2 - 2) : 1;
  // tile shape: z float4 columns x x columns, <= 512 threads
  const int nz4 = ceil_div(g.nz, 4);
  int ztiles = ceil_div(nz4, 32);
  p.tz4 = ceil_div(nz4, ztiles);
  p.tx = std::max(1, std::min(a->dim == 3 ? 8 : 16, 256 / p.tz4));
  if (a->dim == 3) {
    const long long zx = (long long)ztiles * ceil_div(g.nx, p.tx);
    int ych = 32;
    while (ych > 8 && zx * ceil_div(g.ny, ych) < 148 * 3) ych /= 2;
    p.ych = ych;
  } else {
    p.ych = 1;
  }
  p.threads = p.tz4 * p.tx;
  p.grid = dim3(ztiles, ceil_div(g.nx, p.tx), a->dim == 3 ? ceil_div(g.ny, p.ych) : 1);
  p.smem_per_g = 2ull * (p.tz4 + 2) * (p.tx + 4) * sizeof(float4);
  return PW_OK;
}

static void taper_tables(const Plan &p, float ct, std::vector<float> &wz1, std::vector<float> &wz2,
                         std::vector<float> &wx1, std::vector<float> &wx2,
                         std::vector<float> &wy1, std::vector<float> &wy2) {
  const int nb = p.nb;
  std::vector<float> w(std::max(nb, 1));
  // abc_cal (wave_abc.c:141-143): float product, double exp, stored as float
  for (int ib = 0; ib < nb; ib++) w[ib] = (float)exp(-ct * ct * (nb - 1 - ib) * (nb - 1 - ib));
  auto axis = [&](int n, int n2, std::vector<float> &first, std::vector<float> &second) {
    first.assign(n, 1.f);
    second.assign(n, 1.f);
    for (int i = 0; i < nb && i < n; i++) first[i] = w[i];          // top / left face
    for (int i = 0; i < nb; i++) {                                   // bottom / right face,
      const int cell = n2 - 1 - i;                                   // indexed from the padded end
      if (cell >= 0 && cell < n) second[cell] = w[i];
    }
  };
  axis(p.g.nz, p.nz2, wz1, wz2);
  axis(p.g.nx, p.nx2, wx1, wx2);
  if (p.dim == 3) axis(p.g.ny, p.ny2, wy1, wy2);
  else { wy1.assign(1, 1.f); wy2.assign(1, 1.f); }
}

template <int DIM, int G, bool TRI>
static int launch_step(const Plan &p, const StepArgs &s, cudaStream_t st) {
  const size_t smem = p.smem_per_g * G;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(step_kernel<DIM, G, TRI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    attr_set = true;
  }
  step_kernel<DIM, G, TRI><<<p.grid, p.threads, smem, st>>>(s);
  PW_CUDA(cudaGetLastError());
  return PW_OK;
}

static int launch_any(const Plan &p, int G, bool tri, const StepArgs &s, cudaStream_t st) {
#define PW_L(D, GG, T) \
  if (p.dim == D && G == GG && tri == T) return launch_step<D, GG, T>(p, s, st);
  PW_L(2, 1, false) PW_L(3, 1, false)
  PW_L(2, 1, true) PW_L(2, 2, true) PW_L(2, 3, true) PW_L(2, 4, true)
  PW_L(3, 1, true) PW_L(3, 2, true) PW_L(3, 3, true) PW_L(3, 4, true)
#undef PW_L
  set_error("unsupported kernel variant dim=%d G=%d tri=%d", p.dim, G, (int)tri);
  return PW_ERR_SHAPE;
}

static int check_cfl(const pw_afd_args *a, const float *vel_host_max) {
  if (a->flags & PW_NO_CFL_CHECK) return PW_OK;
  // 4th-order leapfrog: v dt / h <= 0.612 (2-D) / 0.5 (3-D) (measured limits)
  const float h = std::min(a->dz, std::min(a->dx, a->dim == 3 ? a->dy : a->dx));
  const float lim = a->dim == 3 ? 0.5f : 0.612f;
  const float cfl = (*vel_host_max) * a->dt / h;
  PW_CHECK(cfl <= lim, PW_ERR_CFL, "unstable: vmax*dt/h = %g exceeds %g", cfl, lim);
  return PW_OK;
}

__global__ void vel_stats_kernel(const float *v, long long n, unsigned int *out) {
  float mx = 0.f, mn = 3.0e38f;
  unsigned int bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float x = v[i];
    if (!(x > 0.f) || !isfinite(x)) bad = 1;
    else { mx = fmaxf(mx, x); mn = fminf(mn, x); }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, __float_as_uint(mx));
    atomicMin(out + 1, __float_as_uint(mn));
    if (bad) atomicOr(out + 2, 1u);
  }
}

// Finite positive velocities and the stability limit, checked on the device
// copy before the time loop starts.
static int check_velocity(const pw_afd_args *a, const float *vel_dev, size_t n, unsigned int *mx,
                          cudaStream_t st) {
  const unsigned int init[3] = {0u, 0x7f7fffffu, 0u};
  PW_CUDA(cudaMemcpyAsync(mx, init, sizeof init, cudaMemcpyHostToDevice, st));
  vel_stats_kernel<<<592, 256, 0, st>>>(vel_dev, (long long)n, mx);
  PW_CUDA(cudaGetLastError());
  unsigned int h[3];
  PW_CUDA(cudaMemcpyAsync(h, mx, sizeof h, cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  PW_CHECK(h[2] == 0, PW_ERR_VALUE, "velocity has non-finite or non-positive values");
  float vmax;
  memcpy(&vmax, &h[0], 4);
  return check_cfl(a, &vmax);
}

struct Run {
  Plan p;
  int G;
  bool tri;
  int ntsnap;
  // device slices
  float *vv, *wz1, *wz2, *wx1, *wx2, *wy1, *wy2;
  float *A[MAXG], *B[MAXG];
  float *rick, *trid, *rec, *img, *vel;
  int *gid;
  unsigned int *mx;
};

// Shared driver of pw_afd / pw_tri_image.
static int run(const pw_afd_args *a, int G, const int *group_host_or_dev, const float *vel,
               const float *src, const float *wavelet, float *dat, float *wfd, float *img_out,
               int normalize, cudaStream_t st) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  Run r{};
  PW_TRY(make_plan(a, r.p));
  const Plan &p = r.p;
  const Geo &g = p.g;
  r.G = G;
  r.tri = a->tri != 0 || img_out != nullptr;
  PW_CHECK(G >= 1 && G <= MAXG, PW_ERR_SHAPE, "ngroups must be in [1,%d] (got %d)", MAXG, G);
  PW_CHECK(a->jsnap >= 0, PW_ERR_VALUE, "jsnap must be >= 0");
  PW_CHECK(a->gz >= 0 && a->gz < a->nz, PW_ERR_SHAPE, "receiver depth gz=%d outside [0,%d)", a->gz,
           a->nz);
  PW_CHECK(!img_out || a->jsnap > 0, PW_ERR_VALUE, "TRI imaging needs jsnap > 0");
  const int nt = a->nt;
  r.ntsnap = 0;
  if (a->jsnap > 0)
    for (int it = 0; it < nt; it++)
      if (it % a->jsnap == 0) r.ntsnap++;
  const size_t nvel = (size_t)p.nz1 * p.nx1 * p.ny1;
  const size_t nrec = (size_t)p.nx1 * p.ny1;
  const size_t nfield = (size_t)g.sy * g.py + 64;

  // host-side parameters: sources, wavelets, tables
  int ns = 0;
  std::vector<int> sz, sx, sy;
  std::vector<float> rick;
  if (!r.tri) {
    ns = a->ns;
    PW_CHECK(ns >= 0 && ns <= MAXSRC, PW_ERR_SHAPE, "ns must be in [0,%d] (got %d)", MAXSRC, ns);
    const int rows = a->dim == 3 ? 6 : 5;
    std::vector<float> s((size_t)rows * ns);
    if (ns > 0) {
      PW_CHECK(src != nullptr, PW_ERR_VALUE, "source array is null");
      if (host) memcpy(s.data(), src, s.size() * sizeof(float));
      else PW_CUDA(cudaMemcpy(s.data(), src, s.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    rick.resize((size_t)std::max(ns, 1) * nt);
    for (int i = 0; i < ns; i++) {
      // afd.c:416-425 (2-D) / 136-147 (3-D): positions are truncated to int
      const int spx = (int)s[i];
      const int spy = a->dim == 3 ? (int)s[ns + i] : 0;
      const int spz = (int)s[(a->dim == 3 ? 2 : 1) * ns + i];
      const float f0 = s[(rows - 3) * ns + i], t0 = s[(rows - 2) * ns + i], A = s[(rows - 1) * ns + i];
      PW_CHECK(spx >= 0 && spx < p.nx1 && spz >= 0 && spz < p.nz1 && spy >= 0 && spy < p.ny1,
               PW_ERR_SHAPE, "source %d at (z=%d,x=%d,y=%d) outside the model", i, spz, spx, spy);
      PW_CHECK(p.nb >= 1 || (spx > 0 && spx < p.nx1 - 1 && spz > 0 && spz < p.nz1 - 1),
               PW_ERR_SHAPE, "source %d stencil leaves the grid", i);
      sx.push_back(spx + p.nb);
      sy.push_back(a->dim == 3 ? spy + p.nb : 0);
      sz.push_back(spz + p.nb);
      if (wavelet == nullptr) {
        PW_CHECK(t0 >= 0.f && (int)(t0 / a->dt) < nt, PW_ERR_VALUE,
                 "source %d onset t=%g outside [0, nt*dt)", i, t0);
        ricker_table(nt, a->dt, f0, t0, A, rick.data() + (size_t)i * nt);
      }
    }
    if (wavelet != nullptr && ns > 0) {
      if (host) memcpy(rick.data(), wavelet, (size_t)ns * nt * sizeof(float));
      else PW_CUDA(cudaMemcpy(rick.data(), wavelet, (size_t)ns * nt * sizeof(float), cudaMemcpyDeviceToHost));
    }
  }
  std::vector<float> wz1, wz2, wx1, wx2, wy1, wy2;
  taper_tables(p, a->ct, wz1, wz2, wx1, wx2, wy1, wy2);

  // workspace layout
  Carve cv;
  const size_t o_vv = cv.add(nfield * 4);
  size_t o_A[MAXG], o_B[MAXG];
  for (int i = 0; i < G; i++) { o_A[i] = cv.add(nfield * 4); o_B[i] = cv.add(nfield * 4); }
  const size_t o_t = cv.add((wz1.size() * 2 + wx1.size() * 2 + wy1.size() * 2) * 4);
  const size_t o_rick = cv.add(rick.size() * 4 + 4);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_trid = cv.add(r.tri ? (size_t)nt * nrec * 4 : 0);
  const size_t o_trin = cv.add((r.tri && host) ? (size_t)nt * nrec * 4 : 0);
  const size_t o_rec = cv.add(!r.tri && dat ? (size_t)nt * nrec * 4 : 0);
  const size_t o_dat = cv.add(!r.tri && dat && host ? (size_t)nt * nrec * 4 : 0);
  const size_t o_img = cv.add(img_out ? nfield * 4 : 0);
  const size_t o_imgx = cv.add(img_out && host ? nvel * 4 : 0);
  const size_t o_gid = cv.add(group_host_or_dev || G > 1 ? nrec * 4 : 0);
  const size_t o_wfd = cv.add(wfd && host ? (size_t)r.ntsnap * nvel * 4 : 0);
  const size_t o_mx = cv.add(16);

  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  r.vv = at<float>(base, o_vv);
  for (int i = 0; i < G; i++) { r.A[i] = at<float>(base, o_A[i]); r.B[i] = at<float>(base, o_B[i]); }
  float *tb = at<float>(base, o_t);
  r.wz1 = tb; r.wz2 = r.wz1 + wz1.size(); r.wx1 = r.wz2 + wz2.size(); r.wx2 = r.wx1 + wx1.size();
  r.wy1 = r.wx2 + wx2.size(); r.wy2 = r.wy1 + wy1.size();
  r.rick = at<float>(base, o_rick);
  r.vel = host ? at<float>(base, o_vel) : const_cast<float *>(vel);
  r.trid = at<float>(base, o_trid);
  r.rec = at<float>(base, o_rec);
  r.img = img_out ? at<float>(base, o_img) : nullptr;
  r.gid = (group_host_or_dev || G > 1) ? at<int>(base, o_gid) : nullptr;
  r.mx = at<unsigned int>(base, o_mx);

  // inputs
  PW_CHECK(vel != nullptr, PW_ERR_VALUE, "velocity is null");
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  if (host) PW_TRY(to_device(r.vel, vel, nvel * 4, true, st));
  PW_TRY(check_velocity(a, r.vel, nvel, r.mx, st));
  {
    std::vector<float> all;
    all.insert(all.end(), wz1.begin(), wz1.end()); all.insert(all.end(), wz2.begin(), wz2.end());
    all.insert(all.end(), wx1.begin(), wx1.end()); all.insert(all.end(), wx2.begin(), wx2.end());
    all.insert(all.end(), wy1.begin(), wy1.end()); all.insert(all.end(), wy2.begin(), wy2.end());
    PW_CUDA(cudaMemcpyAsync(tb, all.data(), all.size() * 4, cudaMemcpyHostToDevice, st));
  }
  if (!r.tri && ns > 0)
    PW_CUDA(cudaMemcpyAsync(r.rick, rick.data(), (size_t)ns * nt * 4, cudaMemcpyHostToDevice, st));
  expand_vv_kernel<<<1184, 256, 0, st>>>(g, r.vel, p.nz1, p.nx1, p.ny1, p.nb, p.nby, a->dt, r.vv);
  PW_CUDA(cudaGetLastError());
  if (r.tri) {
    PW_CHECK(src != nullptr, PW_ERR_VALUE, "TRI traces are null");
    const float *din = src;
    if (host) {
      float *tmp = at<float>(base, o_trin);
      PW_TRY(to_device(tmp, src, (size_t)nt * nrec * 4, true, st));
      din = tmp;
    }
    dim3 tb2(32, 8), tg(ceil_div(nt, 32), ceil_div((long long)nrec, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(din, r.trid, (long long)nrec, nt);
    PW_CUDA(cudaGetLastError());
  }
  if (r.gid) {
    if (group_host_or_dev) {
      PW_TRY(to_device(r.gid, group_host_or_dev, nrec * 4, host, st));
    } else {
      // the demos' x-bands: dg = nx/G, columns >= G*dg unused
      std::vector<int> gh(nrec);
      const int dg = p.nx1 / G;
      for (int iy = 0; iy < p.ny1; iy++)
        for (int ix = 0; ix < p.nx1; ix++) gh[(size_t)iy * p.nx1 + ix] = dg > 0 && ix / dg < G ? ix / dg : -1;
      PW_CUDA(cudaMemcpyAsync(r.gid, gh.data(), nrec * 4, cudaMemcpyHostToDevice, st));
    }
  }

  // time loop
  StepArgs s{};
  s.g = g;
  s.tz4 = p.tz4; s.tx = p.tx; s.ych = p.ych;
  {
    const float c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;  // wave_fdm.c:15
    s.c0 = c0; s.c1 = c1; s.c2 = c2;
    s.idz = 1 / (a->dz * a->dz);
    s.idx = 1 / (a->dx * a->dx);
    s.idy = a->dim == 3 ? 1 / (a->dy * a->dy) : 0.f;
    s.k0 = a->dim == 3 ? (s.idy + s.idx) + s.idz : s.idx + s.idz;
  }
  s.vv = r.vv;
  s.wz1 = r.wz1; s.wz2 = r.wz2; s.wx1 = r.wx1; s.wx2 = r.wx2; s.wy1 = r.wy1; s.wy2 = r.wy2;
  s.nt = nt;
  s.ns = ns;
  for (int i = 0; i < ns; i++) { s.sz[i] = sz[i]; s.sx[i] = sx[i]; s.sy[i] = sy[i]; }
  s.rick = r.rick;
  s.rz = p.nb + a->gz;
  s.rx0 = p.nb; s.ry0 = p.nby; s.nrx = p.nx1; s.nry = p.ny1;
  s.tri_dat = r.tri ? r.trid : nullptr;
  s.gid = r.gid;
  s.rec = (!r.tri && dat) ? r.rec : nullptr;
  s.nb = p.nb; s.nz1 = p.nz1; s.nx1 = p.nx1; s.ny1 = p.ny1; s.nby = p.nby;
  float *wfd_dev = wfd ? (host ? at<float>(base, o_wfd) : wfd) : nullptr;
  float *A[MAXG], *B[MAXG];
  for (int i = 0; i < G; i++) { A[i] = r.A[i]; B[i] = r.B[i]; }
  LoopTimer timer(st);
  timer.start();
  for (int k = 0; k < nt; k++) {
    const int it = r.tri ? nt - 1 - k : k;
    s.it = it;
    for (int i = 0; i < G; i++) { s.cur[i] = A[i]; s.nxt[i] = B[i]; }
    const bool snap = a->jsnap > 0 && it % a->jsnap == 0;
    s.wfd = (snap && wfd_dev) ? wfd_dev + (size_t)(it / a->jsnap) * nvel : nullptr;
    s.img = (snap && r.img) ? r.img : nullptr;
    PW_TRY(launch_any(p, G, r.tri, s, st));
    for (int i = 0; i < G; i++) std::swap(A[i], B[i]);
  }
  timer.stop();

  // outputs
  if (!r.tri && dat) {
    float *dst = host ? at<float>(base, o_dat) : dat;
    dim3 tb2(32, 8), tg(ceil_div((long long)nrec, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(r.rec, dst, nt, (long long)nrec);
    PW_CUDA(cudaGetLastError());
    if (host) PW_TRY(to_host(dat, dst, (size_t)nt * nrec * 4, true, st));
  }
  if (wfd && host) PW_TRY(to_host(wfd, wfd_dev, (size_t)r.ntsnap * nvel * 4, true, st));
  if (img_out) {
    float *dst = host ? at<float>(base, o_imgx) : img_out;
    extract_kernel<<<1184, 256, 0, st>>>(g, r.img, p.nb, p.nby, p.nz1, p.nx1, p.ny1, dst);
    PW_CUDA(cudaGetLastError());
    if (normalize) {
      absmax_kernel<<<592, 256, 0, st>>>(dst, (long long)nvel, r.mx);
      scale_by_max_kernel<<<1184, 256, 0, st>>>(dst, (long long)nvel, r.mx);
      PW_CUDA(cudaGetLastError());
    }
    if (host) PW_TRY(to_host(img_out, dst, nvel * 4, true, st));
  }
  PW_CUDA(cudaStreamSynchronize(st));
  // launches: velocity check, vv expansion, [trace transpose], time loop,
  // [trace transpose | image extract (+2 for normalisation)]
  const long long aux = 2 + (r.tri ? 1 : 0) + ((!r.tri && dat) ? 1 : 0) +
                        (img_out ? (normalize ? 3 : 1) : 0);
  timer.finish(nt, nt + aux);
  return PW_OK;
}

}  // namespace afd
}  // namespace pw

extern "C" int pw_afd(const pw_afd_args *a, const float *vel, const float *src,
                      const float *wavelet, float *dat, float *wfd, void *stream) {
  return pw::afd::run(a, 1, nullptr, vel, src, wavelet, dat, wfd, nullptr, 0,
                      (cudaStream_t)stream);
}

extern "C" int pw_tri_image(const pw_afd_args *a, int ngroups, const int *group,
                            const float *vel, const float *dat, float *img, int normalize,
                            void *stream) {
  PW_CHECK(img != nullptr, PW_ERR_VALUE, "img is null");
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  pw_afd_args b = *a;
  b.tri = 1;
  return pw::afd::run(&b, ngroups, group, vel, dat, nullptr, nullptr, nullptr, img, normalize,
                      (cudaStream_t)stream);
}
