// afd propagator on sm_100a: forward modelling, time reversal, and lockstep
// multi-group TRI imaging.  One fused kernel per time step covers
//   4th-order Laplacian -> leapfrog -> injection -> double taper ->
//   receiver sampling -> snapshot / image accumulation
// of the reference's fdm2d / fdm time loop (pywave/src/wave_fdm.c:551-662,
// 209-354) with its exact float evaluation order (no FMA contraction).
//
// Kernel axes.  z is contiguous; x is the tile axis; y is the marched axis.
// 3-D maps (z,x,y) to the model's (z,x,y).  2-D maps the model's x to the
// marched axis y and uses a dummy x axis of extent 1, so one field layout
// serves both.  Field layout: a zero-haloed array
//   off(iz,ix,iy) = (iz + HZ) + sx*(ix + hx) + sy*(iy + hy),
// leading dimension a multiple of 32 floats; each thread owns one aligned
// float4 of 4 consecutive z cells.  Halo cells are never written and stay
// zero: that is the reference's zero border beyond the expanded grid.
//
// Kernels.  Each thread owns one float4 of z cells and marches it along y
// with a 5-deep register queue of its own cells (the y neighbours).  3-D runs
// use tile_kernel: a warp owns an 8-slot x 4-column patch and stages it (with
// its z and x halo) per plane in a private cp.async ring in shared memory,
// together with each lane's B and vv cells, several planes ahead; lanes read
// their z / x neighbours there after a warp-level sync only.  2-D runs (no x
// neighbours) use march_kernel: z neighbours by warp shuffle, the leading
// plane, B and vv by a per-thread cp.async ring.  The TRI image of G receiver
// groups is formed by image_kernel after each imaging step (3-D) or by
// shuffles between the groups' lanes (2-D).
//
// Two buffers per wavefield: at step k the kernel reads A = u_k and B =
// u_{k-1} (as stored, tapered once) and overwrites B with u_{k+1}.  The
// reference's `prev` array is taper(u_{k-1}) (wave_fdm.c:595-597,633-636); it
// is recomputed on the fly from B with the same multiplications, so one
// group-point update moves 16 bytes (read A, B, vv; write B), vv shared by
// all groups.
#include "pw_common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <tuple>

namespace pw {
namespace afd {

constexpr int HZ = 4;       // z halo (cells) in front of iz = 0
constexpr int MAXG = 8;     // receiver groups per lockstep launch
constexpr int MAXSRC = 16;  // point sources resolved inside the kernel

struct Geo {
  int nz, nx, ny;                    // extents in kernel axes
  int lz;                            // leading dimension (floats)
  long long sx, sy;                  // x / y strides (floats)
  int hx, hy;                        // x / y halo widths
  int py;                            // allocated y extent (ny + 2*hy)
  int lz0, lz1, lx0, lx1, ly0, ly1;  // Laplacian is non-zero on [lo,hi) per axis
};

__host__ __device__ inline long long foff(const Geo &g, int iz, int ix, int iy) {
  return (long long)(iz + HZ) + g.sx * (ix + g.hx) + g.sy * (iy + g.hy);
}

struct StepArgs {
  Geo g;
  int ych;  // planes per CTA along y
  int ngroups;
  int S, ZS, KX, nzc, WPC;  // march tile: slots per column, slots / columns per CTA, z chunks,
                            // warps per column chunk
  int WZ, WX;               // warp-tile kernel: warps per CTA along z and x (per group)
  float c0, c1, c2, idx, idy, idz, k0;
  // 1.0f, as a runtime value: each packed product is multiplied by it
  // before it is added, so that a product and its add fused into one FMA
  // (p * one + t) still round as the separate multiply and add
  float one;
  const float *cur[MAXG];
  float *nxt[MAXG];
  const float *vv;
  // taper factor per cell along each axis: the top/left face weight, the
  // bottom/right one, or 1 (faces of one axis are disjoint, and x*1 is exact,
  // so one product per axis equals abc_apply's face-by-face products)
  const float *wz, *wx, *wy;
  int it, nt;
  int ns;
  int sz[MAXSRC], sx[MAXSRC], sy[MAXSRC];
  const float *rick;  // [ns][nt]
  int rz, rx0, ry0, nrx, nry;  // receivers: row rz, x in [rx0,rx0+nrx), y in [ry0,ry0+nry)
  const float *tri_dat;        // [nt][nry][nrx]
  const int *gid;              // [nry][nrx] or null: every receiver feeds group 0
  float *rec;                  // forward traces [nt][nry][nrx] or null
  int nbz, nbx, nby, nz1, nx1, ny1;  // interior = [nb, nb+n1) per kernel axis
  float *wfd;                  // this step's snapshot [ny1][nx1][nz1] (group 0) or null
  float *img;                  // image accumulator (field layout) or null
  // warp-plane counts of the 3-D step paths, or null (warp-tile kernels
  // only): [0..3] TRI paths 0..3, [4..7] forward paths 0..3
  unsigned long long *stats;
  int *err;  // set to nonzero by a warp-tile kernel whose bounded wait gave up
};

__device__ __forceinline__ float el(const float4 &v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_el(float4 &v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}

// 16-byte global -> shared async copy; src_bytes = 0 zero-fills the slot.
__device__ __forceinline__ void cp16(float4 *dst, const float *src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Two cells per f32x2 op for the march and resident kernels (pk2 helpers;
// k1 is the runtime 1.0 of StepArgs::one).  lap_quad: the 4th-order
// Laplacian of the float4 c in the reference's order (y, then x when XT,
// then z terms), with (Lz, Lw) the two cells below c and (Rx, Ry) the two
// above; y1 / y2 are the float4s at y +- 1 / y +- 2.
template <bool XT>
__device__ __forceinline__ float4 lap_quad(const StepArgs &a, f2 k1, const float4 &c,
                                           const float4 &ym1, const float4 &yp1,
                                           const float4 &ym2, const float4 &yp2,
                                           const float4 &xm1, const float4 &xp1,
                                           const float4 &xm2, const float4 &xp2, float Lz,
                                           float Lw, float Rx, float Ry) {
  const f2 kc0 = pk2(a.c0, a.c0), kc1 = pk2(a.c1, a.c1), kc2 = pk2(a.c2, a.c2);
  const f2 kk0 = pk2(a.k0, a.k0), kx = pk2(a.idx, a.idx), ky = pk2(a.idy, a.idy);
  const f2 kz = pk2(a.idz, a.idz);
  const f2 zb = pk2(c.y, c.z);
  const f2 z1[2] = {add2(pk2(Lw, c.x), zb), add2(zb, pk2(c.w, Rx))};
  const f2 z2[2] = {add2(pk2(Lz, Lw), hi2(c)), add2(lo2(c), pk2(Rx, Ry))};
  f2 t[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    auto P = [h](const float4 &v) { return h ? hi2(v) : lo2(v); };
    f2 tt = mul2(mul2(mul2(kc0, P(c)), kk0), k1);
    tt = add2(tt, mul2(mul2(mul2(kc1, add2(P(ym1), P(yp1))), ky), k1));
    tt = add2(tt, mul2(mul2(mul2(kc2, add2(P(ym2), P(yp2))), ky), k1));
    if (XT) {
      tt = add2(tt, mul2(mul2(mul2(kc1, add2(P(xm1), P(xp1))), kx), k1));
      tt = add2(tt, mul2(mul2(mul2(kc2, add2(P(xm2), P(xp2))), kx), k1));
    }
    tt = add2(tt, mul2(mul2(mul2(kc1, z1[h]), kz), k1));
    tt = add2(tt, mul2(mul2(mul2(kc2, z2[h]), kz), k1));
    t[h] = tt;
  }
  return join2(t[0], t[1]);
}
// The leapfrog update before any injection, c + (c - b) + lap vv, with b the
// stored u_{k-1} tapered face by face (wz per cell, then wx when XT, then wy).
template <bool XT>
__device__ __forceinline__ float4 update_quad(f2 k1, const float4 &c, const float4 &pv,
                                              const float4 &lap, const float4 &vv,
                                              const float (&wz)[4], float wx, float wy) {
  const f2 wx2 = pk2(wx, wx), wy2 = pk2(wy, wy);
  f2 r[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    auto P = [h](const float4 &v) { return h ? hi2(v) : lo2(v); };
    f2 b = mul2(P(pv), pk2(wz[2 * h], wz[2 * h + 1]));
    if (XT) b = mul2(b, wx2);
    b = mul2(mul2(b, wy2), k1);
    r[h] = add2(add2(P(c), sub2(P(c), b)), mul2(mul2(P(lap), P(vv)), k1));
  }
  return join2(r[0], r[1]);
}
// The taper of the updated cells, face by face (wz, then wx when XT, then wy).
template <bool XT>
__device__ __forceinline__ float4 taper_quad(const float4 &v, const float (&wz)[4], float wx,
                                             float wy) {
  const f2 wx2 = pk2(wx, wx), wy2 = pk2(wy, wy);
  f2 r[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    f2 t = mul2(h ? hi2(v) : lo2(v), pk2(wz[2 * h], wz[2 * h + 1]));
    if (XT) t = mul2(t, wx2);
    r[h] = mul2(t, wy2);
  }
  return join2(r[0], r[1]);
}

// March kernel: register-marched, one float4 of z cells per thread.
//
// Lanes map onto (z float4 slot, group) with the G receiver groups of a TRI
// launch interleaved (lane = slot_in_warp * G + group), warps onto z chunks
// and x columns.  Slots of one column are contiguous in memory and the x
// stride is the column length, so a warp touches G runs of consecutive 16-B
// cells.  Each thread marches its float4 along y:
//   * y neighbours: a 5-deep register queue;
//   * z neighbours: shuffles from the adjacent slot's lane (loads at warp and
//     chunk edges);
//   * x neighbours (3-D): loads through L1 / L2;
//   * the leading plane of A, the previous field B and vv: cp.async copies
//     into a per-thread ring in shared memory, MARCH_NS - 1 planes ahead.
// A thread only reads ring slots it filled itself, so no barrier is needed;
// the TRI image product meets the groups of a cell in adjacent lanes and is
// formed by shuffles.  Same float evaluation order as the reference.
constexpr int MARCH_MAXT = 512;  // threads per CTA (launch bound)
constexpr int MARCH_NS = 4;      // ring slots per stream: MARCH_NS - 1 planes in flight

// 16-byte async copy allocating in L1 as well (cp.async.ca).
__device__ __forceinline__ void cp16ca(float4 *dst, const float *src, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(n)
               : "memory");
}

// One CTA's work: (bx, by) = (z chunk + x tile, y chunk) of the field that
// `a` describes; `ring` is the CTA's dynamic shared memory.
template <bool TWO_D, bool TRI, bool SNAP>
__device__ __forceinline__ void march_body(const StepArgs &a, int bx, int by, float4 *ring) {
  constexpr int NS = MARCH_NS, D = NS - 1;
  const Geo &g = a.g;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int nth = blockDim.x;
  const int G = a.ngroups;
  const int spw = 32 / G;
  const int gi = lane % G;
  const int sl = lane / G;
  const int xl = w / a.WPC;
  const int zs = (w - xl * a.WPC) * spw + sl;
  const int slot = (bx % a.nzc) * a.ZS + zs;
  const int ix = TWO_D ? 0 : (bx / a.nzc) * a.KX + xl;
  const bool valid = sl < spw && zs < a.ZS && slot < a.S && xl < a.KX && ix < g.nx;
  const int iz0 = 4 * slot - HZ;
  const bool live = valid && slot >= 1 && iz0 < g.nz;
  const float *A = a.cur[0];
  float *B = a.nxt[0];
#pragma unroll
  for (int k = 1; k < MAXG; k++)
    if (gi == k) {
      A = a.cur[k];
      B = a.nxt[k];
    }
  const long long sx = g.sx, sy = g.sy;
  const long long base = valid ? 4LL * slot + sx * (ix + g.hx) + sy * g.hy : 0;
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);

  float wz[4];
  bool lzm[4], keep[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = iz0 + e;
    wz[e] = (live && iz < g.nz) ? a.wz[iz] : 1.f;
    lzm[e] = iz >= g.lz0 && iz < g.lz1;
    keep[e] = iz < g.nz;
  }
  const float wx = (!TWO_D && live) ? a.wx[ix] : 1.f;
  const bool lxm = TWO_D || (ix >= g.lx0 && ix < g.lx1);
  const bool needL = valid && slot >= 1 && (sl == 0 || zs == 0);
  const bool needR = valid && slot + 1 < a.S && (sl == spw - 1 || zs == a.ZS - 1);
  const int erz = a.rz - iz0;
  const bool rec_zx = live && erz >= 0 && erz < 4 && ix >= a.rx0 && ix < a.rx0 + a.nrx;
  const bool in_zx = ix >= a.nbx && ix < a.nbx + a.nx1;
  const int nrec = a.nrx * a.nry;

  const int y0 = by * a.ych;
  const int y1 = min(g.ny, y0 + a.ych);
  float4 *rA = ring, *rB = ring + NS * nth, *rV = ring + 2 * NS * nth;
  // plane y's copies: A at y+2 (the queue's leading plane), B and vv at y
  auto issue = [&](int y) {
    if (y < y1) {
      const int k = (y & (NS - 1)) * nth + t;
      const long long o = base + sy * y;
      cp16ca(rA + k, A + o + 2 * sy, valid);
      cp16(rB + k, B + o, valid);
      cp16(rV + k, a.vv + o, valid);
    }
    cp_commit();
  };
  float4 q0 = zero4, q1 = zero4, q2 = zero4, q3 = zero4;
  if (valid) {
    q0 = __ldg(reinterpret_cast<const float4 *>(A + base + sy * (y0 - 2)));
    q1 = __ldg(reinterpret_cast<const float4 *>(A + base + sy * (y0 - 1)));
    q2 = __ldg(reinterpret_cast<const float4 *>(A + base + sy * y0));
    q3 = __ldg(reinterpret_cast<const float4 *>(A + base + sy * (y0 + 1)));
  }
#pragma unroll
  for (int j = 0; j < D; j++) issue(y0 + j);
  const unsigned full = 0xffffffffu;
  for (int y = y0; y < y1; y++) {
    issue(y + D);
    cp_wait<D>();
    const long long o = base + sy * y;
    const int k = (y & (NS - 1)) * nth + t;
    const float4 q4 = rA[k];
    const float4 pv = rB[k];
    const float4 vv4 = rV[k];
    float4 xm1, xp1, xm2, xp2;
    if (!TWO_D) {
      xm1 = xp1 = xm2 = xp2 = zero4;
      if (valid) {
        xm1 = __ldg(reinterpret_cast<const float4 *>(A + o - sx));
        xp1 = __ldg(reinterpret_cast<const float4 *>(A + o + sx));
        xm2 = __ldg(reinterpret_cast<const float4 *>(A + o - 2 * sx));
        xp2 = __ldg(reinterpret_cast<const float4 *>(A + o + 2 * sx));
      }
    }
    float Lz = __shfl_up_sync(full, q2.z, G), Lw = __shfl_up_sync(full, q2.w, G);
    float Rx = __shfl_down_sync(full, q2.x, G), Ry = __shfl_down_sync(full, q2.y, G);
    if (needL) {
      const float4 h = __ldg(reinterpret_cast<const float4 *>(A + o - 4));
      Lz = h.z;
      Lw = h.w;
    }
    if (needR) {
      const float4 h = __ldg(reinterpret_cast<const float4 *>(A + o + 4));
      Rx = h.x;
      Ry = h.y;
    }
    const float wy = __ldg(a.wy + y);
    const bool lyok = y >= g.ly0 && y < g.ly1;
    const bool rec_here = rec_zx && y >= a.ry0 && y < a.ry0 + a.nry;
    const int r_idx = rec_here ? (y - a.ry0) * a.nrx + (ix - a.rx0) : 0;
    bool inj = false;
    float dval = 0.f;
    if (TRI && rec_here) {
      inj = a.gid == nullptr ? gi == 0 : a.gid[r_idx] == gi;
      if (inj) dval = a.tri_dat[(size_t)a.it * nrec + r_idx];
    }
    bool src_plane = false;
    if (!TRI)
      for (int s = 0; s < a.ns; s++) src_plane |= (y >= a.sy[s] - 1 && y <= a.sy[s] + 1);
    // prev = taper(u_{k-1} as stored); x1.0 outside the faces is exact
    const f2 k1 = pk2(a.one, a.one);
    float4 lap = lap_quad<!TWO_D>(a, k1, q2, q1, q3, q0, q4, xm1, xp1, xm2, xp2, Lz, Lw, Rx, Ry);
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (!(lzm[e] && lxm && lyok)) set_el(lap, e, 0.f);
    float4 res = update_quad<!TWO_D>(k1, q2, pv, lap, vv4, wz, wx, wy);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float vve = el(vv4, e);
      float v = el(res, e);
      if (TRI) {
        if (inj && e == erz) v = fadd(v, fmul(vve, dval));
      } else if (src_plane) {
        const int iz = iz0 + e;
        for (int s = 0; s < a.ns; s++) {
          const int dz = iz - a.sz[s], dxs = TWO_D ? 0 : ix - a.sx[s], dys = y - a.sy[s];
          if (dz >= -1 && dz <= 1 && dxs >= -1 && dxs <= 1 && dys >= -1 && dys <= 1) {
            const float den = (float)(abs(dxs) + abs(dys) + abs(dz) + 1);
            v = fadd(v, fdiv(fmul(vve, a.rick[(size_t)s * a.nt + a.it]), den));
          }
        }
      }
      set_el(res, e, v);
    }
    res = taper_quad<!TWO_D>(res, wz, wx, wy);
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (!keep[e]) set_el(res, e, 0.f);
    if (live) *reinterpret_cast<float4 *>(B + o) = res;
    if (!TRI && rec_here && a.rec && gi == 0) a.rec[(size_t)a.it * nrec + r_idx] = el(res, erz);
    if (SNAP) {
      const bool interior = live && in_zx && y >= a.nby && y < a.nby + a.ny1;
      if (a.wfd && gi == 0 && interior) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          if (iz >= a.nbz && iz < a.nbz + a.nz1)
            a.wfd[((size_t)(y - a.nby) * a.nx1 + (ix - a.nbx)) * a.nz1 + (iz - a.nbz)] =
                el(res, e);
        }
      }
      if (TRI && a.img != nullptr) {
        // prod_g u_g^2 in group order; the groups of a slot sit in lanes sl*G + gg
        float4 prod = make_float4(1.f, 1.f, 1.f, 1.f);
        for (int gg = 0; gg < G; gg++) {
          const int src = sl * G + gg;
          float4 u;
          u.x = __shfl_sync(full, res.x, src);
          u.y = __shfl_sync(full, res.y, src);
          u.z = __shfl_sync(full, res.z, src);
          u.w = __shfl_sync(full, res.w, src);
          prod.x = fmul(fmul(prod.x, u.x), u.x);
          prod.y = fmul(fmul(prod.y, u.y), u.y);
          prod.z = fmul(fmul(prod.z, u.z), u.z);
          prod.w = fmul(fmul(prod.w, u.w), u.w);
        }
        if (gi == 0 && interior) {
          float4 im = *reinterpret_cast<const float4 *>(a.img + o);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int iz = iz0 + e;
            if (iz >= a.nbz && iz < a.nbz + a.nz1) set_el(im, e, fadd(el(im, e), el(prod, e)));
          }
          *reinterpret_cast<float4 *>(a.img + o) = im;
        }
      }
    }
    q0 = q1;
    q1 = q2;
    q2 = q3;
    q3 = q4;
  }
  cp_wait_all();
}

template <bool TWO_D, bool TRI, bool SNAP>
__global__ void __launch_bounds__(MARCH_MAXT) march_kernel(const StepArgs a) {
  extern __shared__ float4 ring[];
  march_body<TWO_D, TRI, SNAP>(a, blockIdx.x, blockIdx.y, ring);
}

// Cluster-resident 2-D propagation for grids that fit in the distributed
// shared memory of one thread-block cluster: ONE launch runs every time step.
// CTA r of the cluster owns columns [r*w, r*w + w) of the kernel y axis (the
// model's x) with all z; its shared memory holds, per group, the current and
// the next/previous field of those columns plus two halo columns on each
// side, and vv.  A step updates the owned cells in place over the previous
// field (each cell reads its own previous value only), writes the two edge
// columns also into the neighbours' halo columns (distributed shared memory
// stores), and ends with one cluster barrier; the next step reads the halos
// locally.  Domain edges keep zero halos, as the global layout does.  The
// arithmetic per cell is march_body's, term by term, so results are
// bit-identical to the step-per-launch path.
constexpr int RES_NTH = 512;   // threads per CTA
constexpr int RES_MAXIPT = 8;  // items (float4 of z cells) per thread, at most

struct ResArgs {
  StepArgs s;    // it, wfd and img are set per step inside the kernel
  int w;         // owned columns per CTA
  int nsl;       // live z float4 slots per column (slot 0 is the zero halo)
  int LZ;        // floats per shared-memory column
  int jsnap;
  float *wfd0;   // snapshot base [ntsnap][interior] or null
  size_t nvel;   // floats per snapshot
  float *img0;   // TRI image accumulator (field layout) or null
};

__device__ __forceinline__ float4 *dsmem_map(float4 *p, unsigned rank) {
  // address of the same shared-memory offset in CTA `rank` of the cluster
  unsigned long long r;
  asm volatile("mapa.u64 %0, %1, %2;\n" : "=l"(r) : "l"(p), "r"(rank));
  return reinterpret_cast<float4 *>(r);
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\n"
               "barrier.cluster.wait.acquire;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned n;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(n));
  return n;
}

template <bool TRI, int IPT>
__global__ void __launch_bounds__(RES_NTH) resident_kernel(const __grid_constant__ ResArgs r) {
  extern __shared__ float4 res_sm[];
  const StepArgs &a = r.s;
  const Geo &g = a.g;
  const int G = TRI ? a.ngroups : 1;
  const unsigned rank = cluster_rank(), nrank = cluster_size();
  const int w = r.w, W4 = w + 4, LZ4 = r.LZ / 4;  // columns incl. halos; float4 per column
  const int arr4 = W4 * LZ4;                       // float4 per array
  const int y0 = (int)rank * w;
  float4 *vvs = res_sm + 2 * G * arr4;
  // taper factors: z for every row (1 beyond nz), y for the owned columns
  float4 *swz4 = vvs + arr4;
  float *swz = reinterpret_cast<float *>(swz4);
  float *swy = swz + r.LZ;
  for (int i = threadIdx.x; i < r.LZ; i += blockDim.x)
    swz[i] = (i >= HZ && i - HZ < g.nz) ? a.wz[i - HZ] : 1.f;
  for (int i = threadIdx.x; i < w; i += blockDim.x) swy[i] = y0 + i < g.ny ? a.wy[y0 + i] : 1.f;
  // zero the fields and halos, load vv of the owned columns
  for (int i = threadIdx.x; i < 2 * G * arr4; i += blockDim.x)
    res_sm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < arr4; i += blockDim.x) {
    const int c = i / LZ4, sl = i - c * LZ4;
    const int y = y0 + c - 2;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c >= 2 && c < w + 2 && y < g.ny && sl >= 1 && 4 * sl - HZ < g.nz)
      v = *reinterpret_cast<const float4 *>(a.vv + foff(g, 4 * sl - HZ, 0, y));
    vvs[i] = v;
  }
  // this thread's items (fixed for the whole run): shared-memory offset, and
  // flag bits 0 live, 1-4 Laplacian rows, 5-8 kept rows, 9 Laplacian
  // column, 10 receiver row, 11 source column, 12 interior column, 13/14 edge
  // column copied to the left / right neighbour
  const int items = w * r.nsl;
  int po4[IPT], pc[IPT];
  unsigned pf[IPT];
  float4 pwz[IPT];
  float pwy[IPT];
#pragma unroll
  for (int j = 0; j < IPT; j++) {
    const int item = threadIdx.x + j * RES_NTH;
    const int c = item / r.nsl;
    const int slot = item - c * r.nsl + 1;
    const int y = y0 + c;
    const int iz0 = 4 * slot - HZ;
    unsigned f = 0;
    if (item < items && y < g.ny) {
      f = 1u;
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int iz = iz0 + e;
        if (iz >= g.lz0 && iz < g.lz1) f |= 2u << e;
        if (iz < g.nz) f |= 32u << e;
      }
      if (y >= g.ly0 && y < g.ly1) f |= 1u << 9;
      const int erz = a.rz - iz0;
      if (erz >= 0 && erz < 4 && a.rx0 == 0 && a.nrx >= 1 && y >= a.ry0 && y < a.ry0 + a.nry)
        f |= 1u << 10;
      bool sp = false;
      if (!TRI)
        for (int sidx = 0; sidx < a.ns; sidx++) sp |= (y >= a.sy[sidx] - 1 && y <= a.sy[sidx] + 1);
      if (sp) f |= 1u << 11;
      if (y >= a.nby && y < a.nby + a.ny1 && 0 >= a.nbx && 0 < a.nbx + a.nx1) f |= 1u << 12;
      if (c < 2 && rank > 0) f |= 1u << 13;
      if (c >= w - 2 && rank + 1 < nrank) f |= 1u << 14;
    }
    po4[j] = (c + 2) * LZ4 + slot;
    pc[j] = c;
    pf[j] = f;
  }
  __syncthreads();  // the taper tables
#pragma unroll
  for (int j = 0; j < IPT; j++) {
    const bool live = pf[j] & 1u;
    const int slot = po4[j] - (pc[j] + 2) * LZ4;
    pwz[j] = live ? swz4[slot] : make_float4(1.f, 1.f, 1.f, 1.f);
    pwy[j] = live ? swy[pc[j]] : 1.f;
  }
  cluster_sync_all();  // every CTA's arrays are zeroed before any halo store
  const int nrec = a.nrx * a.nry;
  for (int k = 0; k < a.nt; k++) {
    const int it = TRI ? a.nt - 1 - k : k;
    const bool snap = r.jsnap > 0 && it % r.jsnap == 0;
    float *wfd = (snap && r.wfd0) ? r.wfd0 + (size_t)(it / r.jsnap) * r.nvel : nullptr;
    float *img = (TRI && snap) ? r.img0 : nullptr;
    const int par = k & 1;  // array 2g+par is the current field of group g
#pragma unroll
    for (int j = 0; j < IPT; j++) {
      const unsigned f = pf[j];
      if (!(f & 1u)) continue;
      const int o4 = po4[j], c = pc[j];
      const int slot = o4 - (c + 2) * LZ4;
      const int y = y0 + c;
      const int iz0 = 4 * slot - HZ;
      const float wz[4] = {pwz[j].x, pwz[j].y, pwz[j].z, pwz[j].w};
      const float wy = pwy[j];
      const bool lyok = f & (1u << 9);
      const bool rec_here = f & (1u << 10);
      const bool src_plane = f & (1u << 11);
      const int erz = a.rz - iz0;
      const int r_idx = rec_here ? (y - a.ry0) * a.nrx : 0;
      const float4 vv4 = vvs[o4];
      float4 prod = make_float4(1.f, 1.f, 1.f, 1.f);
      float4 res0 = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int gi = 0; gi < G; gi++) {
        const float4 *__restrict__ cur = res_sm + (2 * gi + par) * arr4;
        float4 *__restrict__ nxt = res_sm + (2 * gi + 1 - par) * arr4;
        const float4 q0 = cur[o4 - 2 * LZ4], q1 = cur[o4 - LZ4], q2 = cur[o4];
        const float4 q3 = cur[o4 + LZ4], q4 = cur[o4 + 2 * LZ4];
        const float4 L = cur[o4 - 1], R = cur[o4 + 1];
        const float Lz = L.z, Lw = L.w, Rx = R.x, Ry = R.y;
        const float4 pv = nxt[o4];
        bool inj = false;
        float dval = 0.f;
        if (TRI && rec_here) {
          inj = a.gid == nullptr ? gi == 0 : a.gid[r_idx] == gi;
          if (inj) dval = a.tri_dat[(size_t)it * nrec + r_idx];
        }
        const f2 k1 = pk2(a.one, a.one);
        float4 lap = lap_quad<false>(a, k1, q2, q1, q3, q0, q4, q2, q2, q2, q2, Lz, Lw, Rx, Ry);
#pragma unroll
        for (int e = 0; e < 4; e++)
          if (!((f & (2u << e)) && lyok)) set_el(lap, e, 0.f);
        float4 res = update_quad<false>(k1, q2, pv, lap, vv4, wz, 1.f, wy);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const float vve = el(vv4, e);
          float v = el(res, e);
          if (TRI) {
            if (inj && e == erz) v = fadd(v, fmul(vve, dval));
          } else if (src_plane) {
            const int iz = iz0 + e;
            for (int sidx = 0; sidx < a.ns; sidx++) {
              const int dz = iz - a.sz[sidx], dys = y - a.sy[sidx];
              if (dz >= -1 && dz <= 1 && dys >= -1 && dys <= 1) {
                const float den = (float)(abs(dys) + abs(dz) + 1);
                v = fadd(v, fdiv(fmul(vve, a.rick[(size_t)sidx * a.nt + it]), den));
              }
            }
          }
          set_el(res, e, v);
        }
        res = taper_quad<false>(res, wz, 1.f, wy);
#pragma unroll
        for (int e = 0; e < 4; e++)
          if (!(f & (32u << e))) set_el(res, e, 0.f);
        nxt[o4] = res;
        // the neighbours' halo copies of the two edge columns
        if (f & (1u << 13)) *dsmem_map(nxt + o4 + w * LZ4, rank - 1) = res;
        if (f & (1u << 14)) *dsmem_map(nxt + o4 - w * LZ4, rank + 1) = res;
        if (gi == 0) res0 = res;
        if (TRI) {
          prod.x = fmul(fmul(prod.x, res.x), res.x);
          prod.y = fmul(fmul(prod.y, res.y), res.y);
          prod.z = fmul(fmul(prod.z, res.z), res.z);
          prod.w = fmul(fmul(prod.w, res.w), res.w);
        }
      }
      if (!TRI && rec_here && a.rec) a.rec[(size_t)it * nrec + r_idx] = el(res0, erz);
      const bool interior = f & (1u << 12);
      if (wfd && interior) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          if (iz >= a.nbz && iz < a.nbz + a.nz1)
            wfd[((size_t)(y - a.nby) * a.nx1 + (0 - a.nbx)) * a.nz1 + (iz - a.nbz)] = el(res0, e);
        }
      }
      if (TRI && img && interior) {
        float4 *ip = reinterpret_cast<float4 *>(img + foff(g, iz0, 0, y));
        float4 im = *ip;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          if (iz >= a.nbz && iz < a.nbz + a.nz1) set_el(im, e, fadd(el(im, e), el(prod, e)));
        }
        *ip = im;
      }
    }
    cluster_sync_all();
  }
}

// Batched 2-D forward modelling of shots of uneven size and length: one
// launch per time step covers the tiles of every shot still running.  Item
// i = (shot, tile) with tile = z chunk + nzc * y chunk; items are ordered by
// decreasing shot length so that the launch at step `it` takes a prefix.
// The shot's arguments are copied into shared memory; A and B of a shot swap
// roles with the parity of the step.
__global__ void __launch_bounds__(MARCH_MAXT) batch_kernel(const StepArgs *args, const int2 *items,
                                                           int it) {
  extern __shared__ float4 ring[];
  __shared__ StepArgs sa;
  const int2 item = items[blockIdx.x];
  const int *src = reinterpret_cast<const int *>(args + item.x);
  int *dst = reinterpret_cast<int *>(&sa);
  for (int i = threadIdx.x; i < (int)(sizeof(StepArgs) / sizeof(int)); i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    sa.it = it;
    if (it & 1) {
      float *t = sa.nxt[0];
      sa.nxt[0] = const_cast<float *>(sa.cur[0]);
      sa.cur[0] = t;
    }
  }
  __syncthreads();
  march_body<true, false, false>(sa, item.y % sa.nzc, item.y / sa.nzc, ring);
}

// Warp-tile kernels (3-D): each warp owns an 8-slot x 4*NC-column patch of
// one group's field and marches it along y; a lane owns one float4 of z
// cells in NC columns (xl, xl + 4, ...).  Per plane the warp stages its
// patch with a 1-slot z halo and 2-column x halo (10 x (4 NC + 4) float4) in
// a private ring in shared memory, so an A value is fetched from L2
// (4 NC + 4) * 10 / (32 NC) times instead of once per neighbour use; the
// lanes read their z and x neighbours there after a warp-level wait (no CTA
// barrier).  The ring holds planes y .. y+2 plus TILE_NS - 3 in flight; the
// lead plane's centre (y+2) feeds a register queue of y neighbours.  Each
// lane's B and vv cells ride in the same ring slot as the A patch of their
// plane (TILE_NS - 1 planes ahead of their use).  Two ways to fill the ring:
//   tile_kernel      (NC = 1) every lane issues 16-byte cp.async copies (its
//                    share of the patch plus its B and vv cells);
//   tile_kernel_tma  one lane issues three TMA tile loads per plane (the A
//                    box, the 8 x 4 NC float4 B and vv boxes), completed on
//                    the slot's mbarrier; the tensor maps cover this GPU's
//                    own field buffers only (no multicast).
// Groups of a TRI launch are separate warps of the CTA; the TRI image of an
// imaging step is formed afterwards by image_kernel.
constexpr int TILE_ZW = 8, TILE_XW = 4;  // warp patch per column set: z slots x x columns
constexpr int TILE_TZ = TILE_ZW + 2;     // z slots with halo
constexpr int TILE_NS = 5;               // ring planes per warp
constexpr int TILE_MAXT = 512;
constexpr int TILE_MAXNC = 2;            // columns per lane
__host__ __device__ constexpr int tile_tx(int nc) { return TILE_XW * nc + 4; }  // A-box columns
__host__ __device__ constexpr int tile_tp(int nc) { return TILE_TZ * tile_tx(nc); }  // A-box float4
__host__ __device__ constexpr int tile_slot(int nc) { return tile_tp(nc) + 64 * nc; }  // + B, vv
__host__ __device__ constexpr int tile_ws(int nc) { return TILE_NS * tile_slot(nc); }  // per warp

// Per-lane constants of the warp-tile kernels.
template <int NC>
struct TileLane {
  int lane, gi, zl, xl, slot, iz0, s0, c0, erz;
  int ix[NC];
  bool valid[NC], live[NC], lxm[NC], rec_zx[NC], in_zx[NC];
  long long base[NC];  // field offset of each column's float4 in plane 0 (or a safe one)
  float wz4[4], wx[NC], wzx[NC][4];
  bool lzm[4], keep[4];
  bool warp_plain, warp_taper_zx, warp_edge_zx, warp_rec;
};

// GROUP_GRID: the CTA holds one group's warps and blockIdx.x = group + G *
// tile; otherwise the CTA holds the G group warps of one tile (warp = group
// + G * warp-in-group).
template <int NC, bool GROUP_GRID>
__device__ __forceinline__ void tile_lane_setup(const StepArgs &a, TileLane<NC> &L) {
  const Geo &g = a.g;
  const unsigned full = 0xffffffffu;
  const int t = threadIdx.x, w = t >> 5;
  L.lane = t & 31;
  const int G = a.ngroups;
  L.gi = GROUP_GRID ? (int)(blockIdx.x % G) : w % G;
  const int wt = GROUP_GRID ? w : w / G;
  const int tile = GROUP_GRID ? (int)(blockIdx.x / G) : (int)blockIdx.x;
  const int wzi = wt % a.WZ, wxi = wt / a.WZ;
  L.zl = L.lane % TILE_ZW;
  L.xl = L.lane / TILE_ZW;
  L.s0 = (tile % a.nzc) * (a.WZ * TILE_ZW) + wzi * TILE_ZW;  // warp's first slot
  L.c0 = (tile / a.nzc) * (a.WX * TILE_XW * NC) + wxi * TILE_XW * NC;
  L.slot = L.s0 + L.zl;
  L.iz0 = 4 * L.slot - HZ;
  const long long safe = g.sx * g.hx + g.sy * g.hy;  // slot 0, column 0: in range for every plane
  bool lane_taper = false, lane_plain = true, lane_edge = false, any_rec = false;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = L.iz0 + e;
    L.lzm[e] = iz >= g.lz0 && iz < g.lz1;
    L.keep[e] = iz < g.nz;
  }
  const bool zlive = L.slot < a.S && L.slot >= 1 && L.iz0 < g.nz;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = L.iz0 + e;
    L.wz4[e] = (zlive && iz < g.nz) ? a.wz[iz] : 1.f;
  }
  L.erz = a.rz - L.iz0;
#pragma unroll
  for (int j = 0; j < NC; j++) {
    const int ix = L.c0 + L.xl + TILE_XW * j;
    L.ix[j] = ix;
    L.valid[j] = L.slot < a.S && ix < g.nx;
    L.live[j] = L.valid[j] && zlive;
    L.base[j] = L.valid[j] ? 4LL * L.slot + g.sx * (ix + g.hx) + g.sy * g.hy : safe;
    L.wx[j] = L.live[j] ? a.wx[ix] : 1.f;
    L.lxm[j] = ix >= g.lx0 && ix < g.lx1;
    bool plain = L.lxm[j], taper = L.wx[j] != 1.f, edge = false;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      plain &= L.lzm[e] && L.keep[e];
      taper |= L.wz4[e] != 1.f;
      edge |= L.wz4[e] != 1.f && L.wx[j] != 1.f;
      L.wzx[j][e] = fmul(L.wz4[e], L.wx[j]);
    }
    lane_plain &= !L.live[j] || plain;
    lane_taper |= L.live[j] && taper;
    lane_edge |= L.live[j] && edge;
    L.rec_zx[j] = L.live[j] && L.erz >= 0 && L.erz < 4 && ix >= a.rx0 && ix < a.rx0 + a.nrx;
    any_rec |= L.rec_zx[j];
    L.in_zx[j] = ix >= a.nbx && ix < a.nbx + a.nx1;
  }
  // warp-uniform: every live cell free of masks; any cell tapered in z or x;
  // any z-x edge cell (tapered along both z and x: the factors one by one;
  // elsewhere wz * wx has at most one factor != 1 and is exact)
  L.warp_plain = __all_sync(full, lane_plain);
  L.warp_taper_zx = __any_sync(full, lane_taper);
  L.warp_edge_zx = __any_sync(full, lane_edge);
  L.warp_rec = __any_sync(full, any_rec);
}

// One plane y of a warp-tile kernel for the lane's NC float4: the 4th-order
// Laplacian (z neighbours and x neighbours from the staged A patch pc, y
// neighbours from the queue q), the leapfrog update against pv = u_{k-1} as
// stored, injection, the taper and the store, in the reference's float order.
// Warp-uniform paths, exact because every skipped factor is exactly 1:
// 0 no taper and no mask; 1 y taper only (x wy); 2 z / x taper only, no z-x
// edge (x wz*wx); 3 everything face by face (masks, sources, z-x edges).
// Returns the path taken.
template <bool TRI, bool SNAP, int NC>
__device__ __forceinline__ int tile_plane(const StepArgs &a, const TileLane<NC> &L, int y,
                                          float wy, const float4 (&q0)[NC],
                                          const float4 (&q1)[NC], const float4 (&q2)[NC],
                                          const float4 (&q3)[NC], const float4 (&q4)[NC],
                                          const float4 *pc, const float4 *pbv, float *const (&pB)[NC]) {
  const Geo &g = a.g;
  constexpr int TZ = TILE_TZ;
  const int erz = L.erz, gi = L.gi;
  const bool lyok = y >= g.ly0 && y < g.ly1;
  const f2 kc0 = pk2(a.c0, a.c0), kc1 = pk2(a.c1, a.c1), kc2 = pk2(a.c2, a.c2);
  const f2 kk0 = pk2(a.k0, a.k0), kidx = pk2(a.idx, a.idx), kidy = pk2(a.idy, a.idy);
  const f2 kidz = pk2(a.idz, a.idz), k1 = pk2(a.one, a.one);
  const int nrec = a.nrx * a.nry;
  bool src_plane = false;
  if (!TRI)
    for (int s = 0; s < a.ns; s++) src_plane |= (y >= a.sy[s] - 1 && y <= a.sy[s] + 1);
  // receivers of this plane: forward recording, time-reversal injection
  bool rec_here[NC], inj[NC];
  int r_idx[NC];
  float dval[NC];
  bool inj_warp = false;
#pragma unroll
  for (int j = 0; j < NC; j++) {
    rec_here[j] = inj[j] = false;
    r_idx[j] = 0;
    dval[j] = 0.f;
  }
  if (L.warp_rec) {  // warp-uniform: only warps holding the receiver row
    bool any = false;
#pragma unroll
    for (int j = 0; j < NC; j++) {
      const int ix = L.ix[j];
      rec_here[j] = L.rec_zx[j] && y >= a.ry0 && y < a.ry0 + a.nry;
      r_idx[j] = rec_here[j] ? (y - a.ry0) * a.nrx + (ix - a.rx0) : 0;
      if (TRI && rec_here[j]) {
        inj[j] = a.gid == nullptr ? gi == 0 : a.gid[r_idx[j]] == gi;
        if (inj[j]) dval[j] = a.tri_dat[(size_t)a.it * nrec + r_idx[j]];
      }
      any |= inj[j];
    }
    if (TRI) inj_warp = __any_sync(0xffffffffu, any);
  }
  // injecting warps take the face-by-face path, which adds the trace after
  // the update and before the taper
  const bool clean = L.warp_plain && lyok && !src_plane && !inj_warp;
  const int path = !clean ? 3
                   : (!L.warp_taper_zx ? (wy == 1.f ? 0 : 1)
                                       : (wy == 1.f && !L.warp_edge_zx ? 2 : 3));
#pragma unroll
  for (int j = 0; j < NC; j++) {
    const int ix = L.ix[j];
    const int ci = (L.xl + TILE_XW * j + 2) * TZ + L.zl + 1;  // centre in the A patch
    const float4 xm1 = pc[ci - TZ], xp1 = pc[ci + TZ];
    const float4 xm2 = pc[ci - 2 * TZ], xp2 = pc[ci + 2 * TZ];
    const float2 Lf = reinterpret_cast<const float2 *>(pc + ci - 1)[1];  // (z, w)
    const float2 Rf = reinterpret_cast<const float2 *>(pc + ci + 1)[0];  // (x, y)
    const float4 pv = pbv[L.lane + 32 * j];
    const float4 vv4 = pbv[32 * NC + L.lane + 32 * j];
    // Laplacian sums in the reference's order, two cells per f32x2 op: cells
    // (0, 1) and (2, 3) of the quad; the z +-1 neighbours are the quad
    // shifted by one cell, so their pairs are repacked
    const float4 &c4 = q2[j];
    const f2 cv[2] = {lo2(c4), hi2(c4)};
    const f2 zpa = pk2(Lf.y, c4.x), zpb = pk2(c4.y, c4.z), zpc = pk2(c4.w, Rf.x);
    const f2 s_y1[2] = {add2(lo2(q1[j]), lo2(q3[j])), add2(hi2(q1[j]), hi2(q3[j]))};
    const f2 s_y2[2] = {add2(lo2(q0[j]), lo2(q4[j])), add2(hi2(q0[j]), hi2(q4[j]))};
    const f2 s_x1[2] = {add2(lo2(xm1), lo2(xp1)), add2(hi2(xm1), hi2(xp1))};
    const f2 s_x2[2] = {add2(lo2(xm2), lo2(xp2)), add2(hi2(xm2), hi2(xp2))};
    const f2 s_z1[2] = {add2(zpa, zpb), add2(zpb, zpc)};
    const f2 s_z2[2] = {add2(pk2(Lf.x, Lf.y), hi2(c4)), add2(lo2(c4), pk2(Rf.x, Rf.y))};
    f2 lp2[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      f2 tt = mul2(mul2(mul2(kc0, cv[h]), kk0), k1);
      tt = add2(tt, mul2(mul2(mul2(kc1, s_y1[h]), kidy), k1));
      tt = add2(tt, mul2(mul2(mul2(kc2, s_y2[h]), kidy), k1));
      tt = add2(tt, mul2(mul2(mul2(kc1, s_x1[h]), kidx), k1));
      tt = add2(tt, mul2(mul2(mul2(kc2, s_x2[h]), kidx), k1));
      tt = add2(tt, mul2(mul2(mul2(kc1, s_z1[h]), kidz), k1));
      tt = add2(tt, mul2(mul2(mul2(kc2, s_z2[h]), kidz), k1));
      lp2[h] = tt;
    }
    const f2 pvp[2] = {lo2(pv), hi2(pv)}, vvp[2] = {lo2(vv4), hi2(vv4)};
    float4 res;
    if (path == 0) {
      f2 r[2];
#pragma unroll
      for (int h = 0; h < 2; h++)
        r[h] = add2(add2(cv[h], sub2(cv[h], pvp[h])), mul2(mul2(lp2[h], vvp[h]), k1));
      res = join2(r[0], r[1]);
    } else if (path == 1 || path == 2) {
      const f2 f[2] = {path == 1 ? pk2(wy, wy) : pk2(L.wzx[j][0], L.wzx[j][1]),
                       path == 1 ? pk2(wy, wy) : pk2(L.wzx[j][2], L.wzx[j][3])};
      f2 r[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        f2 v = add2(cv[h], sub2(cv[h], mul2(mul2(pvp[h], f[h]), k1)));
        v = add2(v, mul2(mul2(lp2[h], vvp[h]), k1));
        r[h] = mul2(v, f[h]);
      }
      res = join2(r[0], r[1]);
    } else {
      const float4 lp = join2(lp2[0], lp2[1]);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const float cv = el(q2[j], e);
        const float lap = (L.lzm[e] && L.lxm[j] && lyok) ? el(lp, e) : 0.f;
        // prev = taper(u_{k-1} as stored), face by face
        float p = fmul(el(pv, e), L.wz4[e]);
        p = fmul(p, L.wx[j]);
        p = fmul(p, wy);
        const float vve = el(vv4, e);
        float v = fadd(cv, fsub(cv, p));
        v = fadd(v, fmul(lap, vve));
        // time reversal injects after the update and before the taper
        if (TRI && inj_warp && inj[j] && e == erz) v = fadd(v, fmul(vve, dval[j]));
        if (!TRI && src_plane) {
          const int iz = L.iz0 + e;
          for (int s = 0; s < a.ns; s++) {
            const int dz = iz - a.sz[s], dxs = ix - a.sx[s], dys = y - a.sy[s];
            if (dz >= -1 && dz <= 1 && dxs >= -1 && dxs <= 1 && dys >= -1 && dys <= 1) {
              const float den = (float)(abs(dxs) + abs(dys) + abs(dz) + 1);
              v = fadd(v, fdiv(fmul(vve, a.rick[(size_t)s * a.nt + a.it]), den));
            }
          }
        }
        set_el(res, e, v);
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        float v = fmul(el(res, e), L.wz4[e]);
        v = fmul(v, L.wx[j]);
        v = fmul(v, wy);
        set_el(res, e, L.keep[e] ? v : 0.f);
      }
    }
    if (L.live[j]) *reinterpret_cast<float4 *>(pB[j]) = res;
    if (!TRI && L.warp_rec && rec_here[j] && a.rec && gi == 0)
      a.rec[(size_t)a.it * nrec + r_idx[j]] = el(res, erz);
    if (SNAP) {
      const bool interior = L.live[j] && L.in_zx[j] && y >= a.nby && y < a.nby + a.ny1;
      if (a.wfd && gi == 0 && interior) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = L.iz0 + e;
          if (iz >= a.nbz && iz < a.nbz + a.nz1)
            a.wfd[((size_t)(y - a.nby) * a.nx1 + (ix - a.nbx)) * a.nz1 + (iz - a.nbz)] =
                el(res, e);
        }
      }
    }
  }
  return path;
}

// Per-warp path counts (16 bits per path; a launch gives a warp at most
// ych < 65536 planes), kept only when a.stats is set and flushed at the end:
// [0..3] TRI paths 0..3, [4..7] forward paths 0..3.
template <bool TRI>
__device__ __forceinline__ void flush_path_counts(const StepArgs &a, int lane,
                                                  unsigned long long pcount) {
  if (a.stats != nullptr && lane == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const unsigned long long c = (pcount >> (16 * k)) & 0xffffull;
      if (c) atomicAdd(a.stats + (TRI ? k : 4 + k), c);
    }
  }
}

// cp.async ring of the warp-tile kernel (CTA = the G group warps of WZ x WX
// tiles, as with the TMA ring).  !SPLIT: one ring of TILE_NS slots, each the
// A patch of a plane with this warp's B and vv cells of that plane (copied
// four planes before their use).  SPLIT: an A ring of TILE_NS patches and a
// separate ring of TILE_BV_NS planes of B and vv, copied two planes before
// their use: less shared memory per warp (more resident warps) for a few
// more instructions per plane.
constexpr int TILE_BV_NS = 3;
__host__ __device__ constexpr int tile_cp_ws(int nc, bool split) {  // float4 per warp
  return !split ? TILE_NS * tile_slot(nc) : TILE_NS * tile_tp(nc) + TILE_BV_NS * 64 * nc;
}

template <bool TRI, bool SNAP, int NC, bool SPLIT>
__global__ void __launch_bounds__(TILE_MAXT) tile_kernel(const StepArgs a) {
  extern __shared__ float4 tsm[];
  constexpr int NS = TILE_NS, D = NS - 3, TP = tile_tp(NC), BVS = 64 * NC;
  constexpr int ASTEP = SPLIT ? TP : tile_slot(NC);  // float4 between A slots
  constexpr int CPL = (TP + 31) / 32;                // A-patch copies per lane per plane
  static_assert(NS == 5, "the y loop is unrolled by the queue length 5");
  const Geo &g = a.g;
  TileLane<NC> L;
  tile_lane_setup<NC, false>(a, L);
  const int lane = L.lane, w = threadIdx.x >> 5;
  const float *A = a.cur[0];
  float *B = a.nxt[0];
#pragma unroll
  for (int k = 1; k < MAXG; k++)
    if (L.gi == k) {
      A = a.cur[k];
      B = a.nxt[k];
    }
  const long long sx = g.sx, sy = g.sy;
  const long long safe = sx * g.hx + sy * g.hy;
  float4 *ring = tsm + (size_t)w * tile_cp_ws(NC, SPLIT);  // A slots (B / vv too when !SPLIT)
  float4 *bvring = ring + NS * TP;                  // SPLIT: TILE_BV_NS planes of [B, vv]
  const int y0 = blockIdx.y * a.ych;
  const int y1 = min(g.ny, y0 + a.ych);

  // this lane's share of the A-patch copy: element j = lane + 32k of the
  // (TILE_TZ x tile_tx(NC)) patch, tz fastest; pointers at the next plane
  const float *cpp[CPL];
  bool c_ok[CPL];
#pragma unroll
  for (int k = 0; k < CPL; k++) {
    const int j = lane + 32 * k;
    const int tz = j % TILE_TZ, tx = j / TILE_TZ;
    const int sl = L.s0 - 1 + tz, col = L.c0 - 2 + tx;
    c_ok[k] = j < TP && sl >= 0 && sl < a.S && col >= -g.hx && col < g.nx + g.hx;
    cpp[k] = A + (c_ok[k] ? 4LL * sl + sx * (col + g.hx) + sy * g.hy : safe) + sy * y0;
  }
  // this lane's B and vv cells, pointers at the next plane
  const float *cB[NC], *cV[NC];
#pragma unroll
  for (int j = 0; j < NC; j++) {
    cB[j] = B + L.base[j] + sy * y0;
    cV[j] = a.vv + L.base[j] + sy * y0;
  }
  int next_a = y0, next_bv = y0;
  auto issue_a = [&](int rs) {  // A patch of plane next_a into A slot rs
    if (next_a <= y1 + 1) {
      float4 *dst = ring + rs * ASTEP;
#pragma unroll
      for (int k = 0; k < CPL; k++) {
        const int j = lane + 32 * k;
        if (j < TP) cp16(dst + j, cpp[k], c_ok[k]);
        cpp[k] += sy;
      }
    }
    next_a++;
  };
  auto issue_bv = [&](float4 *dst) {  // B and vv of plane next_bv into dst
    if (next_bv < y1) {
#pragma unroll
      for (int j = 0; j < NC; j++) {
        cp16(dst + lane + 32 * j, cB[j], L.valid[j]);
        cp16(dst + 32 * NC + lane + 32 * j, cV[j], L.valid[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < NC; j++) {
      cB[j] += sy;
      cV[j] += sy;
    }
    next_bv++;
  };

  const bool counting = a.stats != nullptr;
  unsigned long long pcount = 0;
  // queue: plane y-2+k sits in q[(y - y0 + k) % 5]
  float4 q[5][NC];
  float *pB[NC];
#pragma unroll
  for (int j = 0; j < NC; j++) {
    q[4][j] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float *pA = A + L.base[j];
    pB[j] = B + L.base[j] + sy * y0;
    q[0][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 - 2)));
    q[1][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 - 1)));
    q[2][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * y0));
    q[3][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 + 1)));
  }
  float wyn = y0 < y1 ? __ldg(a.wy + y0) : 1.f;
  int bvs = 0;  // SPLIT: B/vv slot of plane y
  if constexpr (!SPLIT) {
    // one commit group per plane (A patch and B / vv of that plane); at plane
    // y the group of plane y + 2 must be complete, so D = 2 may stay in flight
#pragma unroll
    for (int j = 0; j < 2 + D; j++) {
      issue_a(j);
      issue_bv(ring + j * ASTEP + TP);
      cp_commit();
    }
  } else {
    // commit groups: {A y0..y0+2, B/vv y0..y0+1}, {A y0+3}, then per plane y
    // {A y+4, B/vv y+2}; at plane y the group of plane y-2 (or the first two)
    // holds A y+2 and B/vv y, so D = 2 groups may stay in flight
    issue_a(0);
    issue_a(1);
    issue_a(2);
    issue_bv(bvring);
    issue_bv(bvring + BVS);
    cp_commit();
    issue_a(3);
    cp_commit();
  }

  for (int yb = y0; yb < y1; yb += NS) {
#pragma unroll
    for (int u = 0; u < NS; u++) {
      const int y = yb + u;
      if (y < y1) {
        const float4 *pbv;
        issue_a((u + 4) % NS);  // into the slot plane y - 1 left
        if constexpr (!SPLIT) {
          issue_bv(ring + ((u + 4) % NS) * ASTEP + TP);
          pbv = ring + u * ASTEP + TP;
        } else {
          issue_bv(bvring + (bvs == 0 ? 2 : bvs - 1) * BVS);  // (bvs + 2) % 3: plane y - 1's
          pbv = bvring + bvs * BVS;
        }
        cp_commit();
        cp_wait<D>();
        __syncwarp();
        const float4 *slot = ring + u * ASTEP;
        const float4 *lead = ring + ((u + 2) % NS) * ASTEP;
#pragma unroll
        for (int j = 0; j < NC; j++)
          q[(u + 4) % NS][j] = lead[(L.xl + TILE_XW * j + 2) * TILE_TZ + L.zl + 1];
        const float wy = wyn;
        if (y + 1 < y1) wyn = __ldg(a.wy + y + 1);
        const int path = tile_plane<TRI, SNAP, NC>(a, L, y, wy, q[u], q[(u + 1) % NS],
                                                   q[(u + 2) % NS], q[(u + 3) % NS],
                                                   q[(u + 4) % NS], slot, pbv, pB);
        if (counting) pcount += 1ull << (16 * path);
#pragma unroll
        for (int j = 0; j < NC; j++) pB[j] += sy;
        if constexpr (SPLIT) bvs = bvs == 2 ? 0 : bvs + 1;
        __syncwarp();  // the ring slots refilled next iteration were read above
      }
    }
  }
  cp_wait_all();
  flush_path_counts<TRI>(a, lane, pcount);
}

// ---- TMA ring -----------------------------------------------------------
// Tensor maps of one step launch (3-D field layout, float32, zero fill out of
// bounds): the A box (40 z floats x (4 NC + 4) columns x 1 plane) of each
// group's current field, the B box (32 x 4 NC x 1) of each group's previous
// field and of vv.  Dimensions {lz, nx + 2 hx, ny + 2 hy} in array
// coordinates.
struct TileMaps {
  CUtensorMap a[MAXG];
  CUtensorMap b[MAXG];
  CUtensorMap v;
};
constexpr unsigned long long TILE_WAIT_NS = 2000000000ull;  // a wait gives up after 2 s

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
// One try_wait on the given phase parity; the thread may be suspended in the
// hardware for up to about a millisecond while the phase is incomplete.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *b, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(phase), "r"(1000000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Wait for the given phase of an mbarrier, bounded in time: false when it
// gave up (TILE_WAIT_NS).
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned phase) {
  if (mbar_try_wait(b, phase)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(b, phase))
    if (global_ns() - t0 > TILE_WAIT_NS) return false;
  return true;
}
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *m, int c0, int c1, int c2,
                                          unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
      "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

template <bool TRI, bool SNAP, int NC>
__global__ void __launch_bounds__(TILE_MAXT)
    tile_kernel_tma(const StepArgs a, const __grid_constant__ TileMaps maps) {
  extern __shared__ __align__(128) float4 tsm_tma[];
  constexpr int NS = TILE_NS, D = NS - 3, TP = tile_tp(NC), SLOT = tile_slot(NC);
  constexpr unsigned A_BYTES = TP * 16, BV_BYTES = 32 * NC * 16;
  static_assert(NS == 5, "the y loop is unrolled by the queue length 5");
  static_assert((SLOT * 16) % 128 == 0 && (TP * 16) % 128 == 0 && (32 * NC * 16) % 128 == 0,
                "TMA destinations stay 128-byte aligned");
  const Geo &g = a.g;
  TileLane<NC> L;
  tile_lane_setup<NC, false>(a, L);
  const int lane = L.lane, w = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  float *B = a.nxt[0];
#pragma unroll
  for (int k = 1; k < MAXG; k++)
    if (L.gi == k) B = a.nxt[k];
  const float *A = a.cur[0];
#pragma unroll
  for (int k = 1; k < MAXG; k++)
    if (L.gi == k) A = a.cur[k];
  const long long sy = g.sy;
  float4 *ring = tsm_tma + (size_t)w * tile_ws(NC);  // NS slots of [A patch, B, vv]
  unsigned long long *bars =
      reinterpret_cast<unsigned long long *>(tsm_tma + (size_t)nwarps * tile_ws(NC)) + w * NS;
  const int y0 = blockIdx.y * a.ych;
  const int y1 = min(g.ny, y0 + a.ych);
  const CUtensorMap *mA = &maps.a[L.gi], *mB = &maps.b[L.gi], *mV = &maps.v;
  // box origins in array coordinates (z floats, x columns, y planes)
  const int az = 4 * (L.s0 - 1), ax = L.c0 - 2 + g.hx, bz = 4 * L.s0, bx = L.c0 + g.hx;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; s++) mbar_init(bars + s, 1);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncwarp();
  int next_plane = y0;
  // lane 0 loads plane next_plane into ring slot rs: the A box, and the B and
  // vv boxes when next_plane is updated; planes past y1 + 1 are not needed
  auto issue = [&](int rs) {
    if (lane == 0 && next_plane <= y1 + 1) {
      float4 *dst = ring + rs * SLOT;
      const bool upd = next_plane < y1;
      // the slot was last read by the whole warp (ordered by the __syncwarp
      // that precedes this call); order those reads before the async writes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_expect_tx(bars + rs, A_BYTES + (upd ? 2 * BV_BYTES : 0));
      const int py = next_plane + g.hy;
      tma_load3(dst, mA, az, ax, py, bars + rs);
      if (upd) {
        tma_load3(dst + TP, mB, bz, bx, py, bars + rs);
        tma_load3(dst + TP + 32 * NC, mV, bz, bx, py, bars + rs);
      }
    }
    next_plane++;
  };
  int waited = y0 - 1;  // last plane whose slot this lane has waited for
  bool ok = true;
  // wait for plane p (ring slot (p - y0) % NS, phase ((p - y0) / NS) & 1)
  auto wait_plane = [&](int p) {
    if (ok) {
      const int k = p - y0;
      ok = mbar_wait(bars + k % NS, (unsigned)((k / NS) & 1));
      if (ok) waited = p;
    }
  };

  const bool counting = a.stats != nullptr;
  unsigned long long pcount = 0;
  // queue: plane y-2+k sits in q[(y - y0 + k) % 5]
  float4 q[5][NC];
  float *pB[NC];
#pragma unroll
  for (int j = 0; j < NC; j++) {
    q[4][j] = make_float4(0.f, 0.f, 0.f, 0.f);
    const float *pA = A + L.base[j];
    pB[j] = B + L.base[j] + sy * y0;
    q[0][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 - 2)));
    q[1][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 - 1)));
    q[2][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * y0));
    q[3][j] = __ldg(reinterpret_cast<const float4 *>(pA + sy * (y0 + 1)));
  }
  float wyn = y0 < y1 ? __ldg(a.wy + y0) : 1.f;
#pragma unroll
  for (int j = 0; j < 2 + D; j++) issue(j);
  wait_plane(y0);
  wait_plane(y0 + 1);
  ok = __all_sync(0xffffffffu, ok);

  for (int yb = y0; yb < y1 && ok; yb += NS) {
#pragma unroll
    for (int u = 0; u < NS; u++) {
      const int y = yb + u;
      if (y < y1 && ok) {
        issue((u + 2 + D) % NS);  // plane y + 2 + D into the slot plane y - 1 left
        wait_plane(y + 2);
        if (!__all_sync(0xffffffffu, ok)) {
          ok = false;
          break;
        }
        const float4 *slot = ring + u * SLOT;
        const float4 *lead = ring + ((u + 2) % NS) * SLOT;
#pragma unroll
        for (int j = 0; j < NC; j++)
          q[(u + 4) % NS][j] = lead[(L.xl + TILE_XW * j + 2) * TILE_TZ + L.zl + 1];
        const float wy = wyn;
        if (y + 1 < y1) wyn = __ldg(a.wy + y + 1);
        const int path = tile_plane<TRI, SNAP, NC>(a, L, y, wy, q[u], q[(u + 1) % NS],
                                                   q[(u + 2) % NS], q[(u + 3) % NS],
                                                   q[(u + 4) % NS], slot, slot + TP, pB);
        if (counting) pcount += 1ull << (16 * path);
#pragma unroll
        for (int j = 0; j < NC; j++) pB[j] += sy;
        __syncwarp();  // the ring slot refilled next iteration was read above
      }
    }
  }
  if (!ok) {
    // a wait gave up: report it, then let the loads still in flight land in
    // this CTA's shared memory (bounded again) before the warp exits
    if (lane == 0 && a.err) atomicOr(a.err, 1);
    ok = true;
    for (int p = waited + 1; p < next_plane && p <= y1 + 1 && ok; p++) wait_plane(p);
  }
  flush_path_counts<TRI>(a, lane, pcount);
}

// TRI image of one imaging step: img += prod_g u_g^2 over the interior cells
// (the demos' image, test_third_tri.py:71-77, in group order), on the field
// layout, one float4 of z cells per thread.  Used after warp-tile steps.
struct ImgArgs {
  Geo g;
  const float *u[MAXG];
  int G;
  float *img;
  int nbz, nbx, nby, nz1, nx1, ny1;
  int s0, ns4;  // float4 slots covering the interior z range
};

__global__ void image_kernel(const ImgArgs a) {
  const long long n = (long long)a.ns4 * a.nx1 * a.ny1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int sl = a.s0 + (int)(i % a.ns4);
    const long long r = i / a.ns4;
    const int ix = (int)(r % a.nx1) + a.nbx, iy = (int)(r / a.nx1) + a.nby;
    const long long o = 4LL * sl + a.g.sx * (ix + a.g.hx) + a.g.sy * (iy + a.g.hy);
    float4 prod = make_float4(1.f, 1.f, 1.f, 1.f);
#pragma unroll
    for (int k = 0; k < MAXG; k++) {
      if (k < a.G) {
        const float4 u = __ldg(reinterpret_cast<const float4 *>(a.u[k] + o));
        prod.x = fmul(fmul(prod.x, u.x), u.x);
        prod.y = fmul(fmul(prod.y, u.y), u.y);
        prod.z = fmul(fmul(prod.z, u.z), u.z);
        prod.w = fmul(fmul(prod.w, u.w), u.w);
      }
    }
    float4 im = *reinterpret_cast<const float4 *>(a.img + o);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int iz = 4 * sl - HZ + e;
      if (iz >= a.nbz && iz < a.nbz + a.nz1) set_el(im, e, fadd(el(im, e), el(prod, e)));
    }
    *reinterpret_cast<float4 *>(a.img + o) = im;
  }
}

// vv = ((v*v)*dt)*dt on the expanded grid with edge replication of the
// interior velocity (vel_expand, wave_abc.c:14-125; wave_fdm.c:173-175).
// Kernel axes; (nbz,nbx,nby) and (nz1,nx1,ny1) describe the interior.
__global__ void expand_vv_kernel(Geo g, const float *vel, int nz1, int nx1, int ny1, int nbz,
                                 int nbx, int nby, float dt, float *vv) {
  const long long n = (long long)g.nz * g.nx * g.ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % g.nz);
    const int ix = int((i / g.nz) % g.nx);
    const int iy = int(i / ((long long)g.nz * g.nx));
    const int jz = min(max(iz - nbz, 0), nz1 - 1);
    const int jx = min(max(ix - nbx, 0), nx1 - 1);
    const int jy = min(max(iy - nby, 0), ny1 - 1);
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

// interior cells of a field-layout array -> [ny1][nx1][nz1] (kernel axes)
__global__ void extract_kernel(Geo g, const float *f, int nbz, int nbx, int nby, int nz1, int nx1,
                               int ny1, float *out) {
  const long long n = (long long)nz1 * nx1 * ny1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % nz1);
    const int ix = int((i / nz1) % nx1);
    const int iy = int(i / ((long long)nz1 * nx1));
    out[i] = f[foff(g, iz + nbz, ix + nbx, iy + nby)];
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

// ------------------------------------------------------------------ host --

struct Plan {
  int dim;
  int nz1, nx1, ny1, nb;
  // interior placement in kernel axes
  int kbz, kbx, kby, knz1, knx1, kny1;
  Geo g;
  int nz2, nx2, ny2;  // the reference's padded sizes (model axes)
  int ych;
  dim3 grid;
  size_t smem;
  void *fn, *fn_snap;  // plain steps / snapshot and imaging steps
  bool tile;           // warp-tile kernel: TRI images by image_kernel
  bool tma;            // warp-tile kernel with the TMA ring (takes TileMaps)
  int nc;              // warp-tile kernel: columns per lane
  int threads;
  int S, ZS, KX, nzc, WPC, WZ, WX;
};

template <bool TWO_D, bool TRI, bool SNAP>
static void *march_ptr() {
  void *f = (void *)march_kernel<TWO_D, TRI, SNAP>;
  static bool once = [f] {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         3 * MARCH_NS * MARCH_MAXT * (int)sizeof(float4));
    return true;
  }();
  (void)once;
  return f;
}

static void *march_fn(bool tri, bool snap) {  // 2-D runs
  if (tri) return snap ? march_ptr<true, true, true>() : march_ptr<true, true, false>();
  return snap ? march_ptr<true, false, true>() : march_ptr<true, false, false>();
}

// Tile override for measurements: PW_AFD_TILE_G<G>="a,b" fixes the first two
// tile parameters of the planner for G groups.
static void tile_override(int G, int &fa, int &fb) {
  fa = fb = 0;
  char name[32];
  snprintf(name, sizeof name, "PW_AFD_TILE_G%d", G);
  if (const char *e = getenv(name)) sscanf(e, "%d,%d", &fa, &fb);
}

// Tile of the march kernel: WPC warps per z chunk of ZS = WPC * (32/G) slots,
// KX columns per CTA, ych planes per CTA.  Score = useful thread-planes /
// thread-plane capacity spent (idle lanes, dead slots, partial waves, the
// 2-plane prologue of each y chunk), times a latency factor below 24 resident
// warps per SM and a penalty for x-neighbour loads served by other CTAs.
static int plan_march(bool tri, int G, int nsm, Plan &p) {
  const Geo &g = p.g;
  const bool two_d = p.dim == 2;
  void *fn = march_fn(tri, false);
  const int S = g.lz / 4;
  const int spw = 32 / G;
  const int live_slots = ceil_div(g.nz, 4);
  const double useful = (double)G * live_slots * g.nx * g.ny;
  int fw, fk;
  tile_override(G, fw, fk);
  double best = -1;
  int bw = 0, bk = 0, by = 0;
  for (int WPC = 1; WPC <= ceil_div(S, spw); WPC++) {
    if (fw && WPC != fw) continue;
    const int ZS = WPC * spw;
    const int nzc = ceil_div(S, ZS);
    if (WPC > 1 && ceil_div(S, (WPC - 1) * spw) == nzc) continue;  // same chunks, fewer lanes
    for (int KX = 1; KX <= (two_d ? 1 : 64); KX++) {
      const int threads = 32 * WPC * KX;
      if (threads > MARCH_MAXT) break;
      if (fk && KX != fk) continue;
      const size_t smem = (size_t)3 * MARCH_NS * threads * sizeof(float4);
      int occ = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        occ = 0;
      }
      if (occ <= 0) continue;
      const long long slots = (long long)nsm * occ;
      const long long tiles = (long long)nzc * ceil_div(g.nx, KX);
      const double warps = (double)occ * threads / 32;
      const double lat = std::min(1.0, warps / 24.0);
      const double outside = two_d ? 0.0 : (KX == 1 ? 1.0 : 6.0 / (4.0 * KX));
      const double xh = 1.0 / (1.0 + 0.3 * outside);
      for (int ych = std::max(4, ceil_div(g.ny, 65535)); ych <= g.ny + 3; ych++) {
        const int yc = std::min(ych, g.ny);
        const long long ctas = tiles * ceil_div(g.ny, yc);
        const long long waves = (ctas + slots - 1) / slots;
        const double cap = (double)waves * slots * threads * (yc + 2);
        const double score = useful / cap * lat * xh;
        if (score > best + 1e-9) {
          best = score;
          bw = WPC;
          bk = KX;
          by = yc;
        }
        if (yc == g.ny) break;
      }
    }
  }
  PW_CHECK(best > 0, PW_ERR_SHAPE, "no launchable tile for the step kernel");
  p.fn = fn;
  p.fn_snap = march_fn(tri, true);
  p.S = S;
  p.WPC = bw;
  p.ZS = bw * spw;
  p.nzc = ceil_div(S, p.ZS);
  p.KX = bk;
  p.ych = by;
  p.threads = 32 * bw * bk;
  p.smem = (size_t)3 * MARCH_NS * p.threads * sizeof(float4);
  p.grid = dim3((unsigned)(p.nzc * ceil_div(g.nx, bk)), (unsigned)ceil_div(g.ny, by), 1);
  if (getenv("PW_AFD_VERBOSE"))
    fprintf(stderr,
            "afd march plan: G=%d S=%d nzc=%d ZS=%d WPC=%d KX=%d ych=%d threads=%d grid=%ux%u "
            "score=%.3f\n",
            G, S, p.nzc, p.ZS, bw, bk, by, p.threads, p.grid.x, p.grid.y, best);
  return PW_OK;
}

// split B / vv ring of the cp.async kernel (3 slots of B and vv beside the
// 5-slot A ring, less shared memory per warp, so more warps resident): the
// default; PW_AFD_SPLIT=0 selects one 5-slot ring of [A, B, vv] at one
// column per lane
static bool tile_split(int nc) {
  if (nc > 1) return true;
  const char *e = getenv("PW_AFD_SPLIT");
  return !(e && e[0] == '0');
}

static size_t tile_smem(int threads, bool tma, int nc) {
  const size_t nw = (size_t)threads / 32;
  if (!tma) return nw * tile_cp_ws(nc, tile_split(nc)) * sizeof(float4);
  return nw * tile_ws(nc) * sizeof(float4) + nw * TILE_NS * sizeof(unsigned long long);
}

template <bool TRI, bool SNAP, bool TMA, int NC, bool SPLIT = (NC > 1)>
static void *tile_ptr() {
  void *f = TMA ? (void *)tile_kernel_tma<TRI, SNAP, NC>
                : (void *)tile_kernel<TRI, SNAP, NC, SPLIT>;
  static bool once = [f] {
    // as much as a block may opt into (the planner only picks launchable tiles)
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         std::min((int)tile_smem(TILE_MAXT, TMA, NC), maxsm));
    cudaGetLastError();
    return true;
  }();
  (void)once;
  return f;
}

template <bool TRI, bool SNAP>
static void *tile_fn_t(bool tma, int nc) {
  if (!tma) {
    if (nc == 2) return tile_ptr<TRI, SNAP, false, 2>();
    return tile_split(1) ? tile_ptr<TRI, SNAP, false, 1, true>() : tile_ptr<TRI, SNAP, false, 1>();
  }
  return nc == 2 ? tile_ptr<TRI, SNAP, true, 2>() : tile_ptr<TRI, SNAP, true, 1>();
}
static void *tile_fn(bool tri, bool snap, bool tma, int nc) {
  if (tri) return snap ? tile_fn_t<true, true>(tma, nc) : tile_fn_t<true, false>(tma, nc);
  return snap ? tile_fn_t<false, true>(tma, nc) : tile_fn_t<false, false>(tma, nc);
}

// Ring filling of the 3-D warp-tile kernels: per-lane cp.async copies
// (default) or TMA tile loads (PW_AFD_TMA=1); both give identical results.
static bool tile_use_tma() {
  const char *e = getenv("PW_AFD_TMA");
  return e && e[0] == '1';
}

// Tile of the 3-D warp-tile kernel: warps of 8 slots x 4 NC columns (NC
// columns per lane: 1 or 2), ych planes; a CTA holds the G group warps of
// WZ x WX tiles.
// Score = useful thread-planes / capacity spent (idle lanes, dead slots,
// partial waves, the 2-plane prologue of each y chunk) times a latency
// factor below 24 resident warps per SM.  One column per lane unless
// PW_AFD_NC=2: on the 261^3 TRI step two columns issued 6% fewer
// instructions but ran 12% slower (12 instead of 16 resident warps);
// PW_AFD_TILE_G<G>="WZ,WX" fixes the warp layout.
static int plan_tile(bool tri, int G, int nsm, bool tma, Plan &p) {
  const Geo &g = p.g;
  const int S = g.lz / 4;
  const int live_slots = ceil_div(g.nz, 4);
  int fw, fk;
  tile_override(G, fw, fk);
  int fnc = 1;
  if (const char *e = getenv("PW_AFD_NC")) fnc = std::max(1, std::min(TILE_MAXNC, atoi(e)));
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  double best = -1;
  int bz = 0, bx = 0, by = 0, bnc = 1;
  const int gpc = G;  // groups per CTA
  for (int nc = 1; nc <= TILE_MAXNC; nc++) {
    if (fnc && nc != fnc) continue;
    void *fn = tile_fn(tri, false, tma, nc);
    const double useful = (double)G * live_slots * g.nx * g.ny / nc;  // lane-planes
    for (int WZ = 1; WZ <= ceil_div(S, TILE_ZW); WZ++) {
      if (fw && WZ != fw) continue;
      const int nzc = ceil_div(S, WZ * TILE_ZW);
      if (WZ > 1 && ceil_div(S, (WZ - 1) * TILE_ZW) == nzc) continue;
      for (int WX = 1; gpc * WZ * WX * 32 <= TILE_MAXT; WX++) {
        if (fk && WX != fk) continue;
        const int threads = gpc * WZ * WX * 32;
        const size_t smem = tile_smem(threads, tma, nc);
        if (smem > (size_t)maxsm) continue;
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess) {
          cudaGetLastError();
          occ = 0;
        }
        if (occ <= 0) continue;
        const long long slots = (long long)nsm * occ;
        const long long tiles = (long long)nzc * ceil_div(g.nx, WX * TILE_XW * nc) * (G / gpc);
        const double warps = (double)occ * threads / 32;
        const double lat = std::min(1.0, warps / 24.0);
        for (int ych = std::max(4, ceil_div(g.ny, 65535)); ych <= g.ny + 3; ych++) {
          const int yc = std::min(ych, g.ny);
          const long long ctas = tiles * ceil_div(g.ny, yc);
          const long long waves = (ctas + slots - 1) / slots;
          const double cap = (double)waves * slots * threads * (yc + 2);
          const double score = useful / cap * lat;
          // forward runs (one group): among equal scores the larger CTA, which
          // measured faster (201^3: 4 warps 112.8 us per step, 1 warp 121.8)
          const bool wider = G == 1 && nc == bnc && score > best - 1e-9 && threads > 32 * bz * bx;
          if (score > best + 1e-9 || wider) {
            best = std::max(best, score);
            bz = WZ;
            bx = WX;
            by = yc;
            bnc = nc;
          }
          if (yc == g.ny) break;
        }
      }
    }
  }
  PW_CHECK(best > 0, PW_ERR_SHAPE, "no launchable tile for the step kernel");
  p.fn = tile_fn(tri, false, tma, bnc);
  p.fn_snap = tile_fn(tri, true, tma, bnc);
  p.tile = true;
  p.tma = tma;
  p.nc = bnc;
  p.S = S;
  p.WZ = bz;
  p.WX = bx;
  p.nzc = ceil_div(S, bz * TILE_ZW);
  p.ych = by;
  p.threads = gpc * bz * bx * 32;
  p.smem = tile_smem(p.threads, tma, bnc);
  p.grid = dim3((unsigned)(p.nzc * ceil_div(g.nx, bx * TILE_XW * bnc) * (G / gpc)),
                (unsigned)ceil_div(g.ny, by), 1);
  if (getenv("PW_AFD_VERBOSE"))
    fprintf(stderr,
            "afd tile plan: G=%d S=%d nzc=%d WZ=%d WX=%d NC=%d ych=%d threads=%d grid=%ux%u "
            "score=%.3f ring=%s\n",
            G, S, p.nzc, bz, bx, bnc, by, p.threads, p.grid.x, p.grid.y, best,
            tma ? "tma" : (tile_split(bnc) ? "cp.async+split" : "cp.async"));
  return PW_OK;
}

static int make_plan(const pw_afd_args *a, bool tri, int G, Plan &p, bool allow_tma = true) {
  PW_CHECK(a->dim == 2 || a->dim == 3, PW_ERR_SHAPE, "dim must be 2 or 3 (got %d)", a->dim);
  PW_CHECK(a->nz >= 1 && a->nx >= 1 && a->ny >= 1 && a->nt >= 1 && a->nbt >= 0, PW_ERR_SHAPE,
           "sizes must be positive (nz=%d nx=%d ny=%d nt=%d nbt=%d)", a->nz, a->nx, a->ny, a->nt,
           a->nbt);
  PW_CHECK(a->dim == 3 || a->ny == 1, PW_ERR_SHAPE, "2-D runs need ny = 1 (got %d)", a->ny);
  const bool two_d = a->dim == 2;
  p.dim = a->dim;
  p.nz1 = a->nz;
  p.nx1 = a->nx;
  p.ny1 = a->ny;
  p.nb = a->nbt;
  const int enz = p.nz1 + 2 * p.nb, enx = p.nx1 + 2 * p.nb, eny = two_d ? 1 : p.ny1 + 2 * p.nb;
  p.nz2 = pad_first(enz);
  p.nx2 = next_fast(enx);
  p.ny2 = two_d ? 1 : next_fast(eny);
  // abc_apply's opposite faces are disjoint whenever the padded grid holds both
  PW_CHECK(p.nz2 >= 2 * p.nb && p.nx2 >= 2 * p.nb && (two_d || p.ny2 >= 2 * p.nb), PW_ERR_SHAPE,
           "taper faces overlap");
  Geo &g = p.g;
  g.nz = enz;
  g.lz = (int)round_up(HZ + round_up(enz, 4) + 4, 32);
  g.lz0 = 2;
  g.lz1 = std::min(enz, p.nz2 - 2);
  if (two_d) {
    g.nx = 1; g.hx = 0; g.sx = g.lz;
    g.ny = enx; g.hy = 2; g.sy = g.lz;
    g.lx0 = 0; g.lx1 = 1;
    g.ly0 = 2; g.ly1 = std::min(enx, p.nx2 - 2);
    p.kbz = p.nb; p.kbx = 0; p.kby = p.nb;
    p.knz1 = p.nz1; p.knx1 = 1; p.kny1 = p.nx1;
  } else {
    g.nx = enx; g.hx = 2; g.sx = g.lz;
    g.ny = eny; g.hy = 2; g.sy = (long long)g.lz * (enx + 4);
    g.lx0 = 2; g.lx1 = std::min(enx, p.nx2 - 2);
    g.ly0 = 2; g.ly1 = std::min(eny, p.ny2 - 2);
    p.kbz = p.nb; p.kbx = p.nb; p.kby = p.nb;
    p.knz1 = p.nz1; p.knx1 = p.nx1; p.kny1 = p.ny1;
  }
  g.py = g.ny + 2 * g.hy;

  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  p.S = p.ZS = p.KX = p.nzc = p.WPC = p.WZ = p.WX = 0;
  p.tile = p.tma = false;
  p.nc = 1;
  if (two_d) PW_TRY(plan_march(tri, G, nsm, p));  // 2-D: no x neighbours to stage
  else PW_TRY(plan_tile(tri, G, nsm, allow_tma && tile_use_tma(), p));
  return PW_OK;
}

// Taper factor per cell along one model axis: the top/left face weight
// w[i] for i < nb, the bottom/right face weight, which abc_apply indexes from
// the padded end n2-1-i (wave_abc.c:234,260,286), or 1.
static void taper_axis(int n, int n2, int nb, const std::vector<float> &w, std::vector<float> &f) {
  f.assign(n, 1.f);
  for (int i = 0; i < nb && i < n; i++) f[i] = w[i];
  for (int i = 0; i < nb; i++) {
    const int cell = n2 - 1 - i;
    if (cell >= 0 && cell < n) f[cell] = w[i];
  }
}

static int check_cfl(const pw_afd_args *a, float vmax) {
  if (a->flags & PW_NO_CFL_CHECK) return PW_OK;
  // 4th-order leapfrog: v dt / h <= 0.612 (2-D) / 0.5 (3-D) (measured limits)
  const float h = std::min(a->dz, std::min(a->dx, a->dim == 3 ? a->dy : a->dx));
  const float lim = a->dim == 3 ? 0.5f : 0.612f;
  const float cfl = vmax * a->dt / h;
  PW_CHECK(cfl <= lim, PW_ERR_CFL, "unstable: vmax*dt/h = %g exceeds %g", cfl, lim);
  return PW_OK;
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
  return check_cfl(a, vmax);
}

// Shared driver of pw_afd / pw_tri_image.
// Cluster shape for resident_kernel: the largest cluster (16, 8, 4 or 2
// CTAs, one per SM) whose column bands of at least 2 columns fit in shared
// memory and that the device can schedule.  Returns false when the grid is
// too large (the step-per-launch path then runs).
struct ResPlan {
  int C, w, nsl, LZ, threads;
  size_t smem;
  void *fn;
};

template <bool TRI>
static void *resident_fn_t(int ipt) {
  switch (ipt) {
    case 1: return (void *)resident_kernel<TRI, 1>;
    case 2: return (void *)resident_kernel<TRI, 2>;
    case 3: return (void *)resident_kernel<TRI, 3>;
    case 4: return (void *)resident_kernel<TRI, 4>;
    case 5: case 6: return (void *)resident_kernel<TRI, 6>;
    default: return (void *)resident_kernel<TRI, 8>;
  }
}
static void *resident_fn(bool tri, int ipt) {
  return tri ? resident_fn_t<true>(ipt) : resident_fn_t<false>(ipt);
}

static bool plan_resident(const Geo &g, int G, bool tri, ResPlan &rp) {
  const char *env = getenv("PW_AFD_RESIDENT");
  if (env && env[0] == '0') return false;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  rp.nsl = (g.nz + HZ + 3) / 4 - 1;
  rp.LZ = 4 * (rp.nsl + 2);
  rp.threads = RES_NTH;
  const int narr = 2 * (tri ? G : 1) + 1;
  for (int C : {16, 8, 4, 2}) {
    const int w = (g.ny + C - 1) / C;
    if (w < 2) continue;
    const int ipt = (w * rp.nsl + RES_NTH - 1) / RES_NTH;
    if (ipt > RES_MAXIPT) break;  // smaller clusters only need more
    rp.fn = resident_fn(tri, ipt);
    const size_t smem = ((size_t)narr * (w + 4) * rp.LZ + rp.LZ + w) * sizeof(float);
    if (smem > (size_t)maxsm) break;  // smaller clusters only need more
    // the kernel's shared-memory limit only grows (it is per kernel, and a
    // cached smaller value must not shadow a larger one set since); the
    // cluster occupancy query runs once per (kernel, shared memory, cluster)
    static std::mutex mu;
    static std::map<std::pair<int, void *>, size_t> attr_max;
    static std::map<std::tuple<int, void *, size_t, int>, bool> seen;
    bool ok = true;
    {
      std::lock_guard<std::mutex> lock(mu);
      size_t &am = attr_max[std::make_pair(dev, rp.fn)];
      if (smem > am) {
        ok = cudaFuncSetAttribute(rp.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
             cudaSuccess;
        if (ok) am = smem;
      }
      if (ok && C > 8)
        ok = cudaFuncSetAttribute(rp.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
             cudaSuccess;
      const auto key = std::make_tuple(dev, rp.fn, smem, C);
      const auto hit = seen.find(key);
      if (ok && hit != seen.end()) {
        ok = hit->second;
      } else if (ok) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(rp.threads);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        ok = cudaOccupancyMaxActiveClusters(&nclusters, rp.fn, &cfg) == cudaSuccess &&
             nclusters >= 1;
        seen[key] = ok;
      }
      cudaGetLastError();
    }
    if (!ok) continue;
    rp.C = C;
    rp.w = w;
    rp.smem = smem;
    return true;
  }
  return false;
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// Tensor map of one field-layout array of this GPU (z floats x columns incl.
// halo x planes incl. halo) with a box of bz floats x bx columns x 1 plane.
static int field_map(const Geo &g, const float *base, int bz, int bx, CUtensorMap *m) {
  auto enc = encode_fn();
  PW_CHECK(enc != nullptr, PW_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dim[3] = {(cuuint64_t)g.lz, (cuuint64_t)(g.nx + 2 * g.hx), (cuuint64_t)g.py};
  const cuuint64_t stride[2] = {(cuuint64_t)g.sx * 4, (cuuint64_t)g.sy * 4};
  const cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)bx, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dim,
                         stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PW_CHECK(r == CUDA_SUCCESS, PW_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return PW_OK;
}

// The two step launches' tensor maps: parity 0 reads buf0 as the current
// field and buf1 as the previous one, parity 1 the other way round.
static int tile_maps(const Geo &g, int G, int nc, float *const *buf0, float *const *buf1,
                     const float *vv, TileMaps m[2]) {
  for (int par = 0; par < 2; par++) {
    memset(&m[par], 0, sizeof(TileMaps));
    for (int i = 0; i < G; i++) {
      PW_TRY(field_map(g, par ? buf1[i] : buf0[i], 4 * TILE_TZ, tile_tx(nc), &m[par].a[i]));
      PW_TRY(field_map(g, par ? buf0[i] : buf1[i], 4 * TILE_ZW, TILE_XW * nc, &m[par].b[i]));
    }
    PW_TRY(field_map(g, vv, 4 * TILE_ZW, TILE_XW * nc, &m[par].v));
  }
  return PW_OK;
}

static int run(const pw_afd_args *a, int G, const int *group, const float *vel, const float *src,
               const float *wavelet, float *dat, float *wfd, float *img_out, int normalize,
               cudaStream_t st) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const bool tri = a->tri != 0 || img_out != nullptr;
  PW_CHECK(G >= 1 && G <= MAXG, PW_ERR_SHAPE, "ngroups must be in [1,%d] (got %d)", MAXG, G);
  Plan p;
  PW_TRY(make_plan(a, tri, G, p));
  const Geo &g = p.g;
  const bool two_d = p.dim == 2;
  PW_CHECK(a->jsnap >= 0, PW_ERR_VALUE, "jsnap must be >= 0");
  PW_CHECK(a->gz >= 0 && a->gz < a->nz, PW_ERR_SHAPE, "receiver depth gz=%d outside [0,%d)", a->gz,
           a->nz);
  PW_CHECK(!img_out || a->jsnap > 0, PW_ERR_VALUE, "TRI imaging needs jsnap > 0");
  const int nt = a->nt;
  int ntsnap = 0;
  if (a->jsnap > 0)
    for (int it = 0; it < nt; it++)
      if (it % a->jsnap == 0) ntsnap++;
  const size_t nvel = (size_t)p.nz1 * p.nx1 * p.ny1;
  const size_t nrec = (size_t)p.nx1 * p.ny1;
  const size_t nfield = (size_t)g.sy * g.py + 64;

  // sources and wavelets (host)
  int ns = 0;
  std::vector<int> ksz, ksx, ksy;
  std::vector<float> rick;
  if (!tri) {
    ns = a->ns;
    PW_CHECK(ns >= 0 && ns <= MAXSRC, PW_ERR_SHAPE, "ns must be in [0,%d] (got %d)", MAXSRC, ns);
    const int rows = two_d ? 5 : 6;
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
      const int spy = two_d ? 0 : (int)s[ns + i];
      const int spz = (int)s[(two_d ? 1 : 2) * ns + i];
      const float f0 = s[(rows - 3) * ns + i], t0 = s[(rows - 2) * ns + i], A = s[(rows - 1) * ns + i];
      PW_CHECK(spx >= 0 && spx < p.nx1 && spz >= 0 && spz < p.nz1 && spy >= 0 && spy < p.ny1,
               PW_ERR_SHAPE, "source %d at (z=%d,x=%d,y=%d) outside the model", i, spz, spx, spy);
      PW_CHECK(p.nb >= 1 || (spx > 0 && spx < p.nx1 - 1 && spz > 0 && spz < p.nz1 - 1 &&
                             (two_d || (spy > 0 && spy < p.ny1 - 1))),
               PW_ERR_SHAPE, "source %d stencil leaves the grid", i);
      ksz.push_back(spz + p.nb);
      if (two_d) {
        ksx.push_back(0);
        ksy.push_back(spx + p.nb);
      } else {
        ksx.push_back(spx + p.nb);
        ksy.push_back(spy + p.nb);
      }
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
  // taper tables in kernel axes
  std::vector<float> w(std::max(p.nb, 1));
  // abc_cal (wave_abc.c:141-143): float product, double exp, stored as float
  for (int ib = 0; ib < p.nb; ib++)
    w[ib] = (float)exp(-a->ct * a->ct * (p.nb - 1 - ib) * (p.nb - 1 - ib));
  std::vector<float> wz, wx, wy;
  taper_axis(g.nz, p.nz2, p.nb, w, wz);
  if (two_d) {
    wx.assign(1, 1.f);
    taper_axis(g.ny, p.nx2, p.nb, w, wy);
  } else {
    taper_axis(g.nx, p.nx2, p.nb, w, wx);
    taper_axis(g.ny, p.ny2, p.nb, w, wy);
  }

  // workspace layout
  Carve cv;
  const size_t o_vv = cv.add(nfield * 4);
  size_t o_A[MAXG], o_B[MAXG];
  for (int i = 0; i < G; i++) {
    o_A[i] = cv.add(nfield * 4);
    o_B[i] = cv.add(nfield * 4);
  }
  const size_t ntab = wz.size() + wx.size() + wy.size();
  const size_t o_t = cv.add(ntab * 4);
  const size_t o_rick = cv.add(rick.size() * 4 + 4);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_trid = cv.add(tri ? (size_t)nt * nrec * 4 : 0);
  const size_t o_trin = cv.add((tri && host) ? (size_t)nt * nrec * 4 : 0);
  const size_t o_rec = cv.add(!tri && dat ? (size_t)nt * nrec * 4 : 0);
  const size_t o_dat = cv.add(!tri && dat && host ? (size_t)nt * nrec * 4 : 0);
  const size_t o_img = cv.add(img_out ? nfield * 4 : 0);
  const size_t o_imgx = cv.add(img_out && host ? nvel * 4 : 0);
  const bool use_gid = group != nullptr || G > 1;
  const size_t o_gid = cv.add(use_gid ? nrec * 4 : 0);
  const size_t o_wfd = cv.add(wfd && host ? (size_t)ntsnap * nvel * 4 : 0);
  const size_t o_mx = cv.add(16);
  // PW_AFD_VERBOSE: also count which paths the 3-D step kernels took
  const bool want_stats = p.tile && getenv("PW_AFD_VERBOSE") != nullptr;
  const size_t o_stats = cv.add(want_stats ? 8 * sizeof(unsigned long long) : 0);
  const size_t o_err = cv.add(p.tma ? 16 : 0);

  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  float *vv = at<float>(base, o_vv);
  float *A[MAXG], *B[MAXG];
  for (int i = 0; i < G; i++) {
    A[i] = at<float>(base, o_A[i]);
    B[i] = at<float>(base, o_B[i]);
  }
  float *tb = at<float>(base, o_t);
  float *d_wz = tb, *d_wx = d_wz + wz.size(), *d_wy = d_wx + wx.size();
  float *d_rick = at<float>(base, o_rick);
  const float *d_vel = host ? at<float>(base, o_vel) : vel;
  float *trid = at<float>(base, o_trid);
  float *rec = at<float>(base, o_rec);
  float *img = img_out ? at<float>(base, o_img) : nullptr;
  int *gid = use_gid ? at<int>(base, o_gid) : nullptr;
  unsigned int *mx = at<unsigned int>(base, o_mx);

  // inputs
  PW_CHECK(vel != nullptr, PW_ERR_VALUE, "velocity is null");
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  if (host) PW_TRY(to_device(at<float>(base, o_vel), vel, nvel * 4, true, st));
  PW_TRY(check_velocity(a, d_vel, nvel, mx, st));
  {
    std::vector<float> all;
    for (auto *v : {&wz, &wx, &wy}) all.insert(all.end(), v->begin(), v->end());
    PW_CUDA(cudaMemcpyAsync(tb, all.data(), all.size() * 4, cudaMemcpyHostToDevice, st));
  }
  if (!tri && ns > 0)
    PW_CUDA(cudaMemcpyAsync(d_rick, rick.data(), (size_t)ns * nt * 4, cudaMemcpyHostToDevice, st));
  expand_vv_kernel<<<1184, 256, 0, st>>>(g, d_vel, p.knz1, p.knx1, p.kny1, p.kbz, p.kbx, p.kby,
                                         a->dt, vv);
  PW_CUDA(cudaGetLastError());
  long long aux_launches = 2;
  if (tri) {
    PW_CHECK(src != nullptr, PW_ERR_VALUE, "TRI traces are null");
    const float *din = src;
    if (host) {
      float *tmp = at<float>(base, o_trin);
      PW_TRY(to_device(tmp, src, (size_t)nt * nrec * 4, true, st));
      din = tmp;
    }
    dim3 tb2(32, 8), tg(ceil_div(nt, 32), ceil_div((long long)nrec, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(din, trid, (long long)nrec, nt);
    PW_CUDA(cudaGetLastError());
    aux_launches++;
  }
  if (gid) {
    if (group) {
      PW_TRY(to_device(gid, group, nrec * 4, host, st));
    } else {
      // the demos' x-bands: dg = nx/G, columns >= G*dg unused
      std::vector<int> gh(nrec);
      const int dg = p.nx1 / G;
      for (int iy = 0; iy < p.ny1; iy++)
        for (int ix = 0; ix < p.nx1; ix++)
          gh[(size_t)iy * p.nx1 + ix] = dg > 0 && ix / dg < G ? ix / dg : -1;
      PW_CUDA(cudaMemcpyAsync(gid, gh.data(), nrec * 4, cudaMemcpyHostToDevice, st));
    }
  }

  // time loop
  StepArgs s{};
  s.g = g;
  s.ych = p.ych;
  s.ngroups = G;
  s.S = p.S;
  s.ZS = p.ZS;
  s.KX = p.KX;
  s.nzc = p.nzc;
  s.WPC = p.WPC;
  s.WZ = p.WZ;
  s.WX = p.WX;
  {
    const float c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;  // wave_fdm.c:15
    s.c0 = c0;
    s.c1 = c1;
    s.c2 = c2;
    const float idz = 1 / (a->dz * a->dz), idx = 1 / (a->dx * a->dx);
    s.idz = idz;
    if (two_d) {
      s.idy = idx;  // the model's x is the marched axis
      s.idx = 0.f;
      s.k0 = idx + idz;
    } else {
      const float idy = 1 / (a->dy * a->dy);
      s.idx = idx;
      s.idy = idy;
      s.k0 = (idy + idx) + idz;
    }
    s.one = 1.f;
  }
  s.vv = vv;
  s.wz = d_wz;
  s.wx = d_wx;
  s.wy = d_wy;
  s.nt = nt;
  s.ns = ns;
  for (int i = 0; i < ns; i++) {
    s.sz[i] = ksz[i];
    s.sx[i] = ksx[i];
    s.sy[i] = ksy[i];
  }
  s.rick = d_rick;
  s.rz = p.nb + a->gz;
  if (two_d) {
    s.rx0 = 0; s.nrx = 1; s.ry0 = p.nb; s.nry = p.nx1;
  } else {
    s.rx0 = p.nb; s.nrx = p.nx1; s.ry0 = p.nb; s.nry = p.ny1;
  }
  s.tri_dat = tri ? trid : nullptr;
  s.gid = gid;
  s.rec = (!tri && dat) ? rec : nullptr;
  s.nbz = p.kbz; s.nbx = p.kbx; s.nby = p.kby;
  s.nz1 = p.knz1; s.nx1 = p.knx1; s.ny1 = p.kny1;
  s.stats = want_stats ? at<unsigned long long>(base, o_stats) : nullptr;
  s.err = p.tma ? at<int>(base, o_err) : nullptr;
  TileMaps maps[2];
  if (p.tma) PW_TRY(tile_maps(g, G, p.nc, A, B, vv, maps));
  float *wfd_dev = wfd ? (host ? at<float>(base, o_wfd) : wfd) : nullptr;
  void *fn = p.fn;
  const int threads = p.threads;
  ImgArgs ia{};
  ia.g = g;
  ia.G = G;
  ia.img = img;
  ia.nbz = p.kbz; ia.nbx = p.kbx; ia.nby = p.kby;
  ia.nz1 = p.knz1; ia.nx1 = p.knx1; ia.ny1 = p.kny1;
  ia.s0 = (p.kbz + HZ) / 4;
  ia.ns4 = (p.kbz + p.knz1 - 1 + HZ) / 4 - ia.s0 + 1;
  long long img_launches = 0, step_launches = nt;
  ResPlan rp{};
  const bool resident = two_d && plan_resident(g, G, tri, rp);
  if (getenv("PW_AFD_VERBOSE") && resident)
    fprintf(stderr, "afd resident plan: cluster %d x %d threads, %d columns per CTA, %zu B smem\n",
            rp.C, rp.threads, rp.w, rp.smem);
  LoopTimer timer(st);
  timer.start();
  if (resident) {
    ResArgs ra{};
    ra.s = s;
    ra.w = rp.w;
    ra.nsl = rp.nsl;
    ra.LZ = rp.LZ;
    ra.jsnap = a->jsnap;
    ra.wfd0 = wfd_dev;
    ra.nvel = nvel;
    ra.img0 = img;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = rp.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(rp.C);
    cfg.blockDim = dim3(rp.threads);
    cfg.dynamicSmemBytes = rp.smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&ra};
    PW_CUDA(cudaLaunchKernelExC(&cfg, rp.fn, args));
    step_launches = 1;
  }
  for (int k = 0; k < nt && !resident; k++) {
    const int it = tri ? nt - 1 - k : k;
    s.it = it;
    for (int i = 0; i < G; i++) {
      s.cur[i] = A[i];
      s.nxt[i] = B[i];
    }
    const bool snap = a->jsnap > 0 && it % a->jsnap == 0;
    s.wfd = (snap && wfd_dev) ? wfd_dev + (size_t)(it / a->jsnap) * nvel : nullptr;
    const bool img_step = snap && img;
    s.img = (img_step && !p.tile) ? img : nullptr;
    void *args[] = {(void *)&s, (void *)&maps[k & 1]};
    void *f = (s.wfd || s.img) ? p.fn_snap : fn;
    PW_CUDA(cudaLaunchKernel(f, p.grid, dim3(threads), args, p.smem, st));
    if (img_step && p.tile) {
      for (int i = 0; i < G; i++) ia.u[i] = B[i];
      image_kernel<<<1184, 256, 0, st>>>(ia);
      img_launches++;
    }
    for (int i = 0; i < G; i++) std::swap(A[i], B[i]);
  }
  timer.stop();

  // outputs
  if (!tri && dat) {
    float *dst = host ? at<float>(base, o_dat) : dat;
    dim3 tb2(32, 8), tg(ceil_div((long long)nrec, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(rec, dst, nt, (long long)nrec);
    PW_CUDA(cudaGetLastError());
    aux_launches++;
    if (host) PW_TRY(to_host(dat, dst, (size_t)nt * nrec * 4, true, st));
  }
  if (wfd && host) PW_TRY(to_host(wfd, wfd_dev, (size_t)ntsnap * nvel * 4, true, st));
  if (img_out) {
    float *dst = host ? at<float>(base, o_imgx) : img_out;
    extract_kernel<<<1184, 256, 0, st>>>(g, img, p.kbz, p.kbx, p.kby, p.knz1, p.knx1, p.kny1, dst);
    PW_CUDA(cudaGetLastError());
    aux_launches++;
    if (normalize) {
      absmax_kernel<<<592, 256, 0, st>>>(dst, (long long)nvel, mx);
      scale_by_max_kernel<<<1184, 256, 0, st>>>(dst, (long long)nvel, mx);
      PW_CUDA(cudaGetLastError());
      aux_launches += 2;
    }
    if (host) PW_TRY(to_host(img_out, dst, nvel * 4, true, st));
  }
  int err_flag = 0;
  if (p.tma) PW_CUDA(cudaMemcpyAsync(&err_flag, s.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(step_launches, step_launches + aux_launches + img_launches);
  PW_CHECK(err_flag == 0, PW_ERR_TIMEOUT,
           "a 3-D step kernel gave up waiting for its TMA loads (results are invalid)");
  if (want_stats) {
    unsigned long long c[8];
    PW_CUDA(cudaMemcpy(c, s.stats, sizeof c, cudaMemcpyDeviceToHost));
    fprintf(stderr,
            "afd tile paths (warp-planes): tri_path0=%llu tri_path1=%llu tri_path2=%llu "
            "tri_path3=%llu fwd_path0=%llu fwd_path1=%llu fwd_path2=%llu fwd_path3=%llu\n",
            c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]);
  }
  return PW_OK;
}


// ------------------------------------------------- batched 2-D forward --
// pw_afd_batch: forward modelling of many 2-D shots of uneven size and nt in
// lockstep, one batch_kernel launch per time step over all running shots.

struct BatchShot {
  Plan p;
  int ns;
  std::vector<int> ksz, ksy;
  std::vector<float> rick, wz, wy;
  size_t nvel, nrec, nfield;
  size_t o_vv, o_A, o_B, o_t, o_rick, o_vel, o_rec, o_dat, o_mx;
};

// Host part of run()'s set-up for one forward 2-D shot: plan, sources,
// wavelets and taper tables, and its slices of the workspace.
static int batch_setup(const pw_afd_args *a, const float *src, const float *wavelet, bool host,
                       Carve &cv, BatchShot &b) {
  PW_CHECK(a->dim == 2, PW_ERR_SHAPE, "pw_afd_batch runs 2-D shots only (dim=%d)", a->dim);
  PW_CHECK(a->tri == 0, PW_ERR_VALUE, "pw_afd_batch runs forward modelling only (tri = 0)");
  PW_CHECK(a->jsnap == 0, PW_ERR_VALUE, "pw_afd_batch records traces only (jsnap = 0)");
  PW_CHECK(a->gz >= 0 && a->gz < a->nz, PW_ERR_SHAPE, "receiver depth gz=%d outside [0,%d)", a->gz,
           a->nz);
  Plan &p = b.p;
  PW_TRY(make_plan(a, false, 1, p));
  const Geo &g = p.g;
  const int nt = a->nt;
  b.ns = a->ns;
  PW_CHECK(b.ns >= 0 && b.ns <= MAXSRC, PW_ERR_SHAPE, "ns must be in [0,%d] (got %d)", MAXSRC,
           b.ns);
  std::vector<float> s((size_t)5 * b.ns);
  if (b.ns > 0) {
    PW_CHECK(src != nullptr, PW_ERR_VALUE, "source array is null");
    if (host) memcpy(s.data(), src, s.size() * sizeof(float));
    else PW_CUDA(cudaMemcpy(s.data(), src, s.size() * sizeof(float), cudaMemcpyDeviceToHost));
  }
  b.rick.assign((size_t)std::max(b.ns, 1) * nt, 0.f);
  for (int i = 0; i < b.ns; i++) {
    // afd.c:416-425: positions are truncated to int
    const int spx = (int)s[i], spz = (int)s[b.ns + i];
    const float f0 = s[2 * b.ns + i], t0 = s[3 * b.ns + i], A = s[4 * b.ns + i];
    PW_CHECK(spx >= 0 && spx < p.nx1 && spz >= 0 && spz < p.nz1, PW_ERR_SHAPE,
             "source %d at (z=%d,x=%d) outside the model", i, spz, spx);
    PW_CHECK(p.nb >= 1 || (spx > 0 && spx < p.nx1 - 1 && spz > 0 && spz < p.nz1 - 1),
             PW_ERR_SHAPE, "source %d stencil leaves the grid", i);
    b.ksz.push_back(spz + p.nb);
    b.ksy.push_back(spx + p.nb);
    if (wavelet == nullptr) {
      PW_CHECK(t0 >= 0.f && (int)(t0 / a->dt) < nt, PW_ERR_VALUE,
               "source %d onset t=%g outside [0, nt*dt)", i, t0);
      ricker_table(nt, a->dt, f0, t0, A, b.rick.data() + (size_t)i * nt);
    }
  }
  if (wavelet != nullptr && b.ns > 0) {
    if (host) memcpy(b.rick.data(), wavelet, (size_t)b.ns * nt * sizeof(float));
    else PW_CUDA(cudaMemcpy(b.rick.data(), wavelet, (size_t)b.ns * nt * sizeof(float),
                            cudaMemcpyDeviceToHost));
  }
  std::vector<float> w(std::max(p.nb, 1));
  // abc_cal (wave_abc.c:141-143): float product, double exp, stored as float
  for (int ib = 0; ib < p.nb; ib++)
    w[ib] = (float)exp(-a->ct * a->ct * (p.nb - 1 - ib) * (p.nb - 1 - ib));
  taper_axis(g.nz, p.nz2, p.nb, w, b.wz);
  taper_axis(g.ny, p.nx2, p.nb, w, b.wy);
  b.nvel = (size_t)p.nz1 * p.nx1;
  b.nrec = (size_t)p.nx1;
  b.nfield = (size_t)g.sy * g.py + 64;
  b.o_vv = cv.add(b.nfield * 4);
  b.o_A = cv.add(b.nfield * 4);
  b.o_B = cv.add(b.nfield * 4);
  b.o_t = cv.add((b.wz.size() + 1 + b.wy.size()) * 4);
  b.o_rick = cv.add(b.rick.size() * 4 + 4);
  b.o_vel = cv.add(host ? b.nvel * 4 : 0);
  b.o_rec = cv.add((size_t)nt * b.nrec * 4);
  b.o_dat = cv.add(host ? (size_t)nt * b.nrec * 4 : 0);
  b.o_mx = cv.add(16);
  return PW_OK;
}

// run()'s step arguments for one forward 2-D shot (tile fields set later)
static void batch_args(const pw_afd_args *a, const BatchShot &b, char *base, StepArgs &s) {
  const Plan &p = b.p;
  memset(&s, 0, sizeof s);
  s.g = p.g;
  s.ngroups = 1;
  const float c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;  // wave_fdm.c:15
  s.c0 = c0;
  s.c1 = c1;
  s.c2 = c2;
  const float idz = 1 / (a->dz * a->dz), idx = 1 / (a->dx * a->dx);
  s.idz = idz;
  s.idy = idx;  // the model's x is the marched axis
  s.idx = 0.f;
  s.k0 = idx + idz;
  s.one = 1.f;
  s.cur[0] = at<float>(base, b.o_A);
  s.nxt[0] = at<float>(base, b.o_B);
  s.vv = at<float>(base, b.o_vv);
  float *tb = at<float>(base, b.o_t);
  s.wz = tb;
  s.wx = tb + b.wz.size();
  s.wy = tb + b.wz.size() + 1;
  s.nt = a->nt;
  s.ns = b.ns;
  for (int i = 0; i < b.ns; i++) {
    s.sz[i] = b.ksz[i];
    s.sx[i] = 0;
    s.sy[i] = b.ksy[i];
  }
  s.rick = at<float>(base, b.o_rick);
  s.rz = p.nb + a->gz;
  s.rx0 = 0;
  s.nrx = 1;
  s.ry0 = p.nb;
  s.nry = p.nx1;
  s.rec = at<float>(base, b.o_rec);
  s.nbz = p.kbz;
  s.nbx = p.kbx;
  s.nby = p.kby;
  s.nz1 = p.knz1;
  s.nx1 = p.knx1;
  s.ny1 = p.kny1;
  s.S = p.g.lz / 4;
  s.KX = 1;
}

// A batch tile: WPC warps per z chunk (ZS = 32 * WPC slots), ych planes.
struct BatchTile {
  int wpc, ych;
};

// Sets the tile fields of every shot and builds the (shot, tile) items in
// decreasing shot length; cum[k] = items of the k longest shots.
static void batch_items(const BatchTile &t, const std::vector<int> &order,
                        std::vector<StepArgs> &args, std::vector<int2> &items,
                        std::vector<int> &cum) {
  items.clear();
  cum.assign(1, 0);
  for (int k : order) {
    StepArgs &s = args[k];
    s.WPC = t.wpc;
    s.ZS = 32 * t.wpc;
    s.nzc = ceil_div(s.S, s.ZS);
    s.ych = std::min(t.ych, s.g.ny);
    const int tiles = s.nzc * ceil_div(s.g.ny, s.ych);
    for (int i = 0; i < tiles; i++) items.push_back(make_int2(k, i));
    cum.push_back((int)items.size());
  }
}

static int run_batch(int nshot, const pw_afd_args *args, const float *const *vel,
                     const float *const *src, const float *const *wavelet, float *const *dat,
                     cudaStream_t st) {
  PW_CHECK(nshot >= 1 && nshot <= 65536, PW_ERR_SHAPE, "nshot must be in [1,65536] (got %d)",
           nshot);
  PW_CHECK(args && vel && src && dat, PW_ERR_VALUE, "null argument array");
  const bool host = (args[0].flags & PW_HOST_PTRS) != 0;
  std::vector<BatchShot> shots(nshot);
  Carve cv;
  int ntmax = 0;
  for (int k = 0; k < nshot; k++) {
    PW_CHECK(((args[k].flags & PW_HOST_PTRS) != 0) == host, PW_ERR_VALUE,
             "shot %d: every shot must use the same PW_HOST_PTRS flag", k);
    PW_CHECK(vel[k] && dat[k], PW_ERR_VALUE, "shot %d: velocity or trace pointer is null", k);
    const int rc = batch_setup(&args[k], src[k], wavelet ? wavelet[k] : nullptr, host, cv, shots[k]);
    if (rc != PW_OK) {
      set_error("shot %d: %s", k, std::string(pw_last_error()).c_str());
      return rc;
    }
    ntmax = std::max(ntmax, args[k].nt);
  }
  const size_t o_args = cv.add((size_t)nshot * sizeof(StepArgs));
  size_t max_items = 0;
  const BatchTile cands[] = {{1, 16}, {1, 32}, {2, 32}, {2, 64}, {4, 32}, {4, 64}};
  const int ncand = (int)(sizeof cands / sizeof cands[0]);
  for (const BatchTile &t : cands) {
    size_t n = 0;
    for (int k = 0; k < nshot; k++) {
      const Geo &g = shots[k].p.g;
      n += (size_t)ceil_div(g.lz / 4, 32 * t.wpc) * ceil_div(g.ny, std::min(t.ych, g.ny));
    }
    max_items = std::max(max_items, n);
  }
  PW_CHECK(max_items < (1u << 31), PW_ERR_SHAPE, "too many tiles");
  const size_t o_items = cv.add(max_items * sizeof(int2));

  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  std::vector<StepArgs> sargs(nshot);
  for (int k = 0; k < nshot; k++) {
    const BatchShot &b = shots[k];
    const pw_afd_args *a = &args[k];
    const Plan &p = b.p;
    const float *d_vel = vel[k];
    if (host) {
      PW_TRY(to_device(at<float>(base, b.o_vel), vel[k], b.nvel * 4, true, st));
      d_vel = at<float>(base, b.o_vel);
    }
    const int rc = check_velocity(a, d_vel, b.nvel, at<unsigned int>(base, b.o_mx), st);
    if (rc != PW_OK) {
      set_error("shot %d: %s", k, std::string(pw_last_error()).c_str());
      return rc;
    }
    std::vector<float> tab(b.wz);
    tab.push_back(1.f);
    tab.insert(tab.end(), b.wy.begin(), b.wy.end());
    PW_CUDA(cudaMemcpyAsync(at<float>(base, b.o_t), tab.data(), tab.size() * 4,
                            cudaMemcpyHostToDevice, st));
    if (b.ns > 0)
      PW_CUDA(cudaMemcpyAsync(at<float>(base, b.o_rick), b.rick.data(),
                              (size_t)b.ns * a->nt * 4, cudaMemcpyHostToDevice, st));
    expand_vv_kernel<<<1184, 256, 0, st>>>(p.g, d_vel, p.knz1, p.knx1, p.kny1, p.kbz, p.kbx,
                                           p.kby, a->dt, at<float>(base, b.o_vv));
    PW_CUDA(cudaGetLastError());
    batch_args(a, b, base, sargs[k]);
    PW_CUDA(cudaStreamSynchronize(st));  // tab and rick are host temporaries
  }
  // longest shots first: the launch at step it covers a prefix of the items
  std::vector<int> order(nshot);
  for (int k = 0; k < nshot; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return args[x].nt > args[y].nt; });
  std::vector<int> nt_sorted(nshot);
  for (int k = 0; k < nshot; k++) nt_sorted[k] = args[order[k]].nt;
  StepArgs *d_args = at<StepArgs>(base, o_args);
  int2 *d_items = at<int2>(base, o_items);
  std::vector<int2> items;
  std::vector<int> cum;
  {
    static bool attr = [] {
      cudaFuncSetAttribute((const void *)batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           3 * MARCH_NS * MARCH_MAXT * (int)sizeof(float4));
      return true;
    }();
    (void)attr;
  }
  auto use_tile = [&](const BatchTile &t) -> int {
    batch_items(t, order, sargs, items, cum);
    PW_CUDA(cudaMemcpyAsync(d_args, sargs.data(), sargs.size() * sizeof(StepArgs),
                            cudaMemcpyHostToDevice, st));
    PW_CUDA(cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(int2),
                            cudaMemcpyHostToDevice, st));
    PW_CUDA(cudaStreamSynchronize(st));  // host vectors are reused
    return PW_OK;
  };
  int tile_threads = 32;
  size_t tile_smem = 0;
  // running shots at step it: the first n with nt_sorted[n - 1] > it
  int running = nshot;
  auto step = [&](int it) -> int {
    while (running > 0 && nt_sorted[running - 1] <= it) running--;
    const int n = cum[running];
    if (n == 0) return PW_OK;
    batch_kernel<<<n, tile_threads, tile_smem, st>>>(d_args, d_items, it);
    PW_CUDA(cudaGetLastError());
    return PW_OK;
  };

  // Online tile tuning on the first real steps: every tile computes the same
  // values, so each candidate simply takes two steps, timed by events; the
  // fastest runs the rest.  Short runs keep the first candidate.
  const int tune_steps = 2;
  int best = 0;
  int it = 0;
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  if (ntmax >= 8 * ncand * tune_steps) {
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    PW_CUDA(cudaEventCreate(&e0));
    PW_CUDA(cudaEventCreate(&e1));
    int rc = PW_OK;
    for (int c = 0; c < ncand && rc == PW_OK; c++) {
      rc = use_tile(cands[c]);
      if (rc != PW_OK) break;
      tile_threads = 32 * cands[c].wpc;
      tile_smem = (size_t)3 * MARCH_NS * tile_threads * sizeof(float4);
      cudaEventRecord(e0, st);
      for (int j = 0; j < tune_steps && rc == PW_OK; j++, it++, launches++) rc = step(it);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      // per cell-update (later steps may have fewer running shots)
      double cells = 0;
      for (int k = 0; k < nshot; k++)
        if (args[k].nt > it - tune_steps) cells += (double)shots[k].p.g.nz * shots[k].p.g.ny;
      const float norm = cells > 0 ? (float)(ms / cells) : ms;
      if (norm < best_ms) {
        best_ms = norm;
        best = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PW_TRY(rc);
  }
  PW_TRY(use_tile(cands[best]));
  tile_threads = 32 * cands[best].wpc;
  tile_smem = (size_t)3 * MARCH_NS * tile_threads * sizeof(float4);
  if (getenv("PW_AFD_VERBOSE"))
    fprintf(stderr, "afd batch: %d shots, tile wpc=%d ych=%d, %zu items\n", nshot,
            cands[best].wpc, cands[best].ych, items.size());
  // the remaining steps replay as one CUDA graph (direct launches on the
  // legacy default stream, which cannot be captured)
  bool graphed = false;
  if (st != nullptr && it < ntmax) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      int rc = PW_OK;
      const int it0 = it;
      const int running0 = running;
      for (int j = it0; j < ntmax && rc == PW_OK; j++) rc = step(j);
      const cudaError_t ec = cudaStreamEndCapture(st, &graph);
      if (rc == PW_OK && ec == cudaSuccess &&
          cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess &&
          cudaGraphLaunch(exec, st) == cudaSuccess) {
        graphed = true;
        launches += ntmax - it0;
        it = ntmax;
      } else {
        running = running0;
      }
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
    } else {
      cudaGetLastError();
    }
  }
  if (!graphed)
    for (; it < ntmax; it++, launches++) PW_TRY(step(it));
  timer.stop();

  // traces [nt][nrec] -> [nrec][nt] per shot
  for (int k = 0; k < nshot; k++) {
    const BatchShot &b = shots[k];
    const int nt = args[k].nt;
    float *out = host ? at<float>(base, b.o_dat) : dat[k];
    dim3 tb2(32, 8), tg(ceil_div((long long)b.nrec, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(at<float>(base, b.o_rec), out, nt, (long long)b.nrec);
    PW_CUDA(cudaGetLastError());
    if (host) PW_TRY(to_host(dat[k], out, (size_t)nt * b.nrec * 4, true, st));
  }
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(launches, launches + 2LL * nshot);
  return PW_OK;
}

}  // namespace afd
}  // namespace pw

extern "C" int pw_afd(const pw_afd_args *a, const float *vel, const float *src,
                      const float *wavelet, float *dat, float *wfd, void *stream) {
  return pw::afd::run(a, 1, nullptr, vel, src, wavelet, dat, wfd, nullptr, 0,
                      (cudaStream_t)stream);
}

extern "C" int pw_afd_batch(int nshot, const pw_afd_args *args, const float *const *vel,
                            const float *const *src, const float *const *wavelet,
                            float *const *dat, void *stream) {
  return pw::afd::run_batch(nshot, args, vel, src, wavelet, dat, (cudaStream_t)stream);
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

// ------------------------------------------------------ no-alloc variant --
// pw_afd_noalloc: run()'s forward modelling with every scratch buffer carved
// from the fixed device array of noalloc_scratch.cu instead of the cached
// workspace, for callers that may not allocate device memory.  Same plan,
// step kernel and launch sequence as run(); device pointers only.

namespace pw {
int noalloc_scratch(char **ptr);  // noalloc_scratch.cu

namespace afd {

// Per-cell taper factors of one axis from the nb face weights w: taper_axis
// evaluated on the device.  Only copies of w are stored, so the table equals
// the host-built one bit for bit.
__global__ void taper_table_kernel(const float *w, int nb, int n, int n2, float *f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float v = 1.f;
    if (i < nb) v = w[i];
    const int j = n2 - 1 - i;  // bottom/right face, indexed from the padded end
    if (j >= 0 && j < nb) v = w[j];
    f[i] = v;
  }
}

constexpr int NOALLOC_MAXDEV = 64;

static int run_noalloc(const pw_afd_args *a, const float *vel, const float *src,
                       const float *wavelet, float *dat, float *wfd, cudaStream_t st) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  PW_CHECK((a->flags & PW_HOST_PTRS) == 0, PW_ERR_VALUE,
           "pw_afd_noalloc takes device pointers only (PW_HOST_PTRS is set)");
  PW_CHECK(a->tri == 0, PW_ERR_VALUE, "pw_afd_noalloc runs forward modelling only (tri = 0)");
  PW_CHECK(vel != nullptr, PW_ERR_VALUE, "velocity is null");
  Plan p;
  PW_TRY(make_plan(a, false, 1, p, false));
  const Geo &g = p.g;
  const bool two_d = p.dim == 2;
  PW_CHECK(a->jsnap >= 0, PW_ERR_VALUE, "jsnap must be >= 0");
  PW_CHECK(a->gz >= 0 && a->gz < a->nz, PW_ERR_SHAPE, "receiver depth gz=%d outside [0,%d)", a->gz,
           a->nz);
  const int nt = a->nt;
  const int ns = a->ns;
  PW_CHECK(ns >= 0 && ns <= MAXSRC, PW_ERR_SHAPE, "ns must be in [0,%d] (got %d)", MAXSRC, ns);
  PW_CHECK(ns == 0 || (src != nullptr && wavelet != nullptr), PW_ERR_VALUE,
           "pw_afd_noalloc needs the source array and the wavelet table [ns][nt] on the device");
  const size_t nvel = (size_t)p.nz1 * p.nx1 * p.ny1;
  const size_t nrec = (size_t)p.nx1 * p.ny1;
  const size_t nfield = (size_t)g.sy * g.py + 64;

  // scratch layout: run()'s buffers without the host staging ones
  Carve cv;
  const size_t o_vv = cv.add(nfield * 4);
  const size_t o_A = cv.add(nfield * 4);
  const size_t o_B = cv.add(nfield * 4);
  const size_t o_w = cv.add((size_t)p.nb * 4);
  const size_t o_t = cv.add((size_t)(g.nz + g.nx + g.ny) * 4);
  const size_t o_rec = cv.add(dat ? (size_t)nt * nrec * 4 : 0);
  const size_t o_mx = cv.add(16);
  const size_t need = cv.total();
  PW_CHECK(need <= (size_t)PW_NOALLOC_SCRATCH_BYTES, PW_ERR_SHAPE,
           "pw_afd_noalloc needs %zu bytes of scratch; its fixed device array holds %zu "
           "(pw_afd has no such limit)", need, (size_t)PW_NOALLOC_SCRATCH_BYTES);

  int dev = 0;
  PW_CUDA(cudaGetDevice(&dev));
  PW_CHECK(dev >= 0 && dev < NOALLOC_MAXDEV, PW_ERR_VALUE, "device %d out of range", dev);
  // one scratch array per device: a call holds the device's lock until its
  // stream has drained, so calls never overlap on the array
  static std::mutex locks[NOALLOC_MAXDEV];
  std::lock_guard<std::mutex> lock(locks[dev]);
  // Declared after the lock, so it runs first on every return: once work on
  // the array is queued, the lock is released only after `st` has drained,
  // on the error returns too (its status is ignored there; the error that
  // caused the return is the one reported).
  struct DrainOnExit {
    cudaStream_t st;
    bool armed = false;
    ~DrainOnExit() {
      if (armed) cudaStreamSynchronize(st);
    }
  } drain{st};
  char *base = nullptr;
  PW_TRY(noalloc_scratch(&base));
  float *vv = at<float>(base, o_vv);
  float *A = at<float>(base, o_A), *B = at<float>(base, o_B);
  float *d_w = at<float>(base, o_w);
  float *d_wz = at<float>(base, o_t), *d_wx = d_wz + g.nz, *d_wy = d_wx + g.nx;
  float *rec = at<float>(base, o_rec);
  unsigned int *mx = at<unsigned int>(base, o_mx);

  // wavefields, the padded velocity's halo and the trace buffer start at zero
  drain.armed = true;
  PW_CUDA(cudaMemsetAsync(base, 0, need, st));
  PW_TRY(check_velocity(a, vel, nvel, mx, st));

  // source positions, read back into a fixed host array
  int ksz[MAXSRC], ksx[MAXSRC], ksy[MAXSRC];
  if (ns > 0) {
    const int rows = two_d ? 5 : 6;
    float s[6 * MAXSRC];
    PW_CUDA(cudaMemcpyAsync(s, src, (size_t)rows * ns * sizeof(float), cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < ns; i++) {
      // afd.c:416-425 (2-D) / 136-147 (3-D): positions are truncated to int
      const int spx = (int)s[i];
      const int spy = two_d ? 0 : (int)s[ns + i];
      const int spz = (int)s[(two_d ? 1 : 2) * ns + i];
      PW_CHECK(spx >= 0 && spx < p.nx1 && spz >= 0 && spz < p.nz1 && spy >= 0 && spy < p.ny1,
               PW_ERR_SHAPE, "source %d at (z=%d,x=%d,y=%d) outside the model", i, spz, spx, spy);
      PW_CHECK(p.nb >= 1 || (spx > 0 && spx < p.nx1 - 1 && spz > 0 && spz < p.nz1 - 1 &&
                             (two_d || (spy > 0 && spy < p.ny1 - 1))),
               PW_ERR_SHAPE, "source %d stencil leaves the grid", i);
      ksz[i] = spz + p.nb;
      ksx[i] = two_d ? 0 : spx + p.nb;
      ksy[i] = two_d ? spx + p.nb : spy + p.nb;
    }
  }

  // face weights abc_cal (wave_abc.c:141-143), staged through a fixed host
  // buffer chunk by chunk, then expanded to per-cell tables on the device
  {
    float wb[256];
    for (int i0 = 0; i0 < p.nb; i0 += 256) {
      const int m = std::min(256, p.nb - i0);
      for (int k = 0; k < m; k++) {
        const int ib = i0 + k;
        wb[k] = (float)exp(-a->ct * a->ct * (p.nb - 1 - ib) * (p.nb - 1 - ib));
      }
      PW_CUDA(cudaMemcpyAsync(d_w + i0, wb, (size_t)m * 4, cudaMemcpyHostToDevice, st));
      PW_CUDA(cudaStreamSynchronize(st));
    }
  }
  taper_table_kernel<<<ceil_div(g.nz, 256), 256, 0, st>>>(d_w, p.nb, g.nz, p.nz2, d_wz);
  if (two_d) {
    taper_table_kernel<<<1, 32, 0, st>>>(d_w, 0, 1, 1, d_wx);  // dummy axis: factor 1
    taper_table_kernel<<<ceil_div(g.ny, 256), 256, 0, st>>>(d_w, p.nb, g.ny, p.nx2, d_wy);
  } else {
    taper_table_kernel<<<ceil_div(g.nx, 256), 256, 0, st>>>(d_w, p.nb, g.nx, p.nx2, d_wx);
    taper_table_kernel<<<ceil_div(g.ny, 256), 256, 0, st>>>(d_w, p.nb, g.ny, p.ny2, d_wy);
  }
  PW_CUDA(cudaGetLastError());
  expand_vv_kernel<<<1184, 256, 0, st>>>(g, vel, p.knz1, p.knx1, p.kny1, p.kbz, p.kbx, p.kby,
                                         a->dt, vv);
  PW_CUDA(cudaGetLastError());

  // time loop: run()'s step arguments with one group
  StepArgs s{};
  s.g = g;
  s.ych = p.ych;
  s.ngroups = 1;
  s.S = p.S;
  s.ZS = p.ZS;
  s.KX = p.KX;
  s.nzc = p.nzc;
  s.WPC = p.WPC;
  s.WZ = p.WZ;
  s.WX = p.WX;
  {
    const float c0 = -30. / 12., c1 = +16. / 12., c2 = -1. / 12.;  // wave_fdm.c:15
    s.c0 = c0;
    s.c1 = c1;
    s.c2 = c2;
    const float idz = 1 / (a->dz * a->dz), idx = 1 / (a->dx * a->dx);
    s.idz = idz;
    if (two_d) {
      s.idy = idx;
      s.idx = 0.f;
      s.k0 = idx + idz;
    } else {
      const float idy = 1 / (a->dy * a->dy);
      s.idx = idx;
      s.idy = idy;
      s.k0 = (idy + idx) + idz;
    }
    s.one = 1.f;
  }
  s.vv = vv;
  s.wz = d_wz;
  s.wx = d_wx;
  s.wy = d_wy;
  s.nt = nt;
  s.ns = ns;
  for (int i = 0; i < ns; i++) {
    s.sz[i] = ksz[i];
    s.sx[i] = ksx[i];
    s.sy[i] = ksy[i];
  }
  s.rick = wavelet;
  s.rz = p.nb + a->gz;
  if (two_d) {
    s.rx0 = 0; s.nrx = 1; s.ry0 = p.nb; s.nry = p.nx1;
  } else {
    s.rx0 = p.nb; s.nrx = p.nx1; s.ry0 = p.nb; s.nry = p.ny1;
  }
  s.tri_dat = nullptr;
  s.gid = nullptr;
  s.rec = dat ? rec : nullptr;
  s.nbz = p.kbz; s.nbx = p.kbx; s.nby = p.kby;
  s.nz1 = p.knz1; s.nx1 = p.knx1; s.ny1 = p.kny1;
  s.img = nullptr;
  void *fn = p.fn;
  const int threads = p.threads;
  for (int it = 0; it < nt; it++) {
    s.it = it;
    s.cur[0] = A;
    s.nxt[0] = B;
    const bool snap = a->jsnap > 0 && it % a->jsnap == 0;
    s.wfd = (snap && wfd) ? wfd + (size_t)(it / a->jsnap) * nvel : nullptr;
    void *args[] = {(void *)&s};
    void *f = s.wfd ? p.fn_snap : fn;
    PW_CUDA(cudaLaunchKernel(f, p.grid, dim3(threads), args, p.smem, st));
    std::swap(A, B);
  }
  if (dat) {
    dim3 tb2(32, 8), tg(ceil_div((long long)nrec, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb2, 0, st>>>(rec, dat, nt, (long long)nrec);
    PW_CUDA(cudaGetLastError());
  }
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

}  // namespace afd
}  // namespace pw

extern "C" int pw_afd_noalloc(const pw_afd_args *a, const float *vel, const float *src,
                              const float *wavelet, float *dat, float *wfd, void *stream) {
  return pw::afd::run_noalloc(a, vel, src, wavelet, dat, wfd, (cudaStream_t)stream);
}
