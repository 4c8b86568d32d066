// pfwi passive mode 4 (lstric) on the GPU: the time-reversal modelling
// operator of pywave/src/wave_triutil.c:48-180 (timerev_init / timerev_lop,
// sponge pfwiabc_* :264-316) and the least-squares source inversion of
// wave_fwi.c:121-175 / wave_fwigradient.c:454-520, which is np_solver
// (wave_bigsolver.c:1170-1430, model weight 1, no starting model) stepping
// np_cgstep (wave_cgstep.c:16-67) with that operator.
//
// Two-field form of the three rotated fields.  Per modelling step the
// reference records row rz+nb of u1, sets u2 = Lap(u1) + 2 u1 - u0 on the
// cells [4, pad-4) of both axes, rotates (u0, u1) <- (u1, u2), adds the
// source times vv on the interior and multiplies u0 and u1 by the sponge.
// Per adjoint step it multiplies u1 and u0 by the sponge, images u1 vv,
// sets u2 = LapT(u1) + 2 u1 - u0, rotates and adds the data row.  Writing A
// for u1 as the stencil reads it and B for the field whose sponged value is
// the step's u0, both directions become
//     A' = sponge(L(A) + 2 A - sponge(B) + injection),   B' = A,
// where each cell's new A' reads only its own B.  So A' overwrites B in place
// and the two buffers swap roles every step, with the same products and sums
// in the reference's order (explicitly rounded, never contracted): the
// fields are bit-identical to the reference's.  The reference's step never
// writes the 4-cell rim outside [4, pad-4); with nb >= 4 no source, data
// row or receiver reaches the rim either, so it stays zero (the entry
// points require nb >= 4 and a data row inside [4, pad-4)).
//
// Kernels.  A padded column holds nq = ceil(nzp/4) float4 "quads" of z
// cells, zero beyond nzp.  One thread updates one quad per step.
//   resident_kernel: one thread-block cluster (up to 16 CTAs, one per SM)
//     holds a shot's two fields and vv in distributed shared memory, CTA r
//     owning a band of w padded columns plus 4 halo columns on each side;
//     ONE launch runs every time step, the band's 4 edge columns are also
//     stored into the neighbours' halos, one cluster barrier per step.  The
//     next step's source samples (modelling) or data samples (adjoint) are
//     loaded into registers one step ahead.  Several shots run as separate
//     clusters of the same launch.
//   step_kernel: the same per-quad arithmetic on fields in global memory,
//     one launch per step, for grids too large for a cluster.
#include "pw_common.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

namespace pw {
namespace tr {

constexpr int RNTH = 512;   // resident_kernel: threads per CTA
constexpr int RMAXIPT = 8;  // resident_kernel: quads per thread, at most
constexpr int SNTH = 256;   // step_kernel: threads per block
constexpr int DOTB = 296;   // reduction blocks (2 per SM)
constexpr int DOTT = 256;   // reduction threads per block

struct Args {
  int nzp, nxp, nq;  // padded sizes; z quads per padded column
  int nz, nx, nt, nb, depth;
  float sx, sz;      // 1/dx^2, 1/dz^2 as the reference rounds them
  float c0, c1, c2, c3, c4;
  float one;         // 1.0f at run time: keeps packed products unfused (pk2 helpers)
  const float4 *vv;  // [nxp][nq] quads of vvpad = (v v) dt^2, zero beyond nzp
  const float4 *wz;  // [nq] z sponge factors (1 inside, and beyond nzp)
  const float *wx;   // [nxp] x sponge factors
  float *mod;        // source / image [shot][nt][nx][nz]
  float *dat;        // data [shot][nx][nt]
  size_t mod_stride, dat_stride;  // floats per shot
  int w;             // resident_kernel: padded columns per CTA
  const float4 *X;   // step_kernel: A of every shot, [shot][nxp][nq]
  float4 *Y;         // step_kernel: B, overwritten with A'
  size_t fstride;    // step_kernel: float4 per shot field
  int it;            // step_kernel: time index of this step
};

__device__ __forceinline__ float qel(const float4 &v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void qset(float4 &v, int e, float x) {
  if (e == 0) v.x = x;
  else if (e == 1) v.y = x;
  else if (e == 2) v.z = x;
  else v.w = x;
}
// cell j (-4..7) of the z window made of the quads below, at and above
__device__ __forceinline__ float zwin(const float4 &lo, const float4 &c, const float4 &hi, int j) {
  return j < 0 ? qel(lo, j + 4) : (j < 4 ? qel(c, j) : qel(hi, j - 4));
}

// Static description of one quad (column ix, quad k): bit 0 live (has a
// stencil cell), bits 1-4 stencil cell e, bits 5-8 interior (source /
// image) cell e, bit 9 the quad holds the data row of an interior column
// (element depth - 4k).
__device__ __forceinline__ unsigned quad_flags(const Args &a, int ix, int k) {
  unsigned f = 0;
  if (ix < 4 || ix >= a.nxp - 4) return 0;
  const bool xin = ix >= a.nb && ix < a.nb + a.nx;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = 4 * k + e;
    if (iz >= 4 && iz < a.nzp - 4) f |= 2u << e;
    if (xin && iz >= a.nb && iz < a.nb + a.nz) f |= 32u << e;
  }
  if (!(f & 0x1Eu)) return 0;  // the interior and the data row lie inside the stencil's cells
  f |= 1u;
  const int er = a.depth - 4 * k;
  if (xin && er >= 0 && er < 4) f |= 1u << 9;
  return f;
}

// A' of the quad, two cells per f32x2 op (pk2 helpers).  The 8th-order sums
// of Lap (ADJ = false: plain samples, the sum times the centre's vv) or LapT
// (ADJ = true: every sample times its own vv) in the reference's order;
// ux[4] / vx[4] is the quad's own column, ux[4 +- d] the columns +-d, uzl /
// uzh (vzl / vzh) the quads below / above.  Every product that is added is
// multiplied by the runtime 1.0 first, and 2 u is formed as u + u.  Cells
// outside the stencil stay zero.  inj: modelling, the source samples of the
// interior cells (mod[it]); adjoint, element 0 the data sample of the data
// row.
template <bool ADJ>
__device__ __forceinline__ float4 quad_step(const Args &a, unsigned f, const float4 (&ux)[9],
                                            const float4 &uzl, const float4 &uzh,
                                            const float4 (&vx)[9], const float4 &vzl,
                                            const float4 &vzh, const float4 &B, const float4 &wz4,
                                            float wxv, const float4 &inj, int k) {
  const f2 k1 = pk2(a.one, a.one);
  const f2 kc[5] = {pk2(a.c0, a.c0), pk2(a.c1, a.c1), pk2(a.c2, a.c2), pk2(a.c3, a.c3),
                    pk2(a.c4, a.c4)};
  // z partners (+d, -d), d = 1..4, of each pair of cells: the quads shifted
  const float4 &c = ux[4], &L = uzl, &R = uzh;
  const f2 u_yz = pk2(c.y, c.z), u_wx = pk2(L.w, c.x), u_wR = pk2(c.w, R.x);
  const f2 zpu[2][4] = {{u_yz, hi2(c), u_wR, lo2(R)}, {u_wR, lo2(R), pk2(R.y, R.z), hi2(R)}};
  const f2 zmu[2][4] = {{u_wx, hi2(L), pk2(L.y, L.z), lo2(L)}, {u_yz, lo2(c), u_wx, hi2(L)}};
  f2 zpv[2][4], zmv[2][4];
  if (ADJ) {
    const float4 &cv = vx[4], &Lv = vzl, &Rv = vzh;
    const f2 v_yz = pk2(cv.y, cv.z), v_wx = pk2(Lv.w, cv.x), v_wR = pk2(cv.w, Rv.x);
    const f2 p0[4] = {v_yz, hi2(cv), v_wR, lo2(Rv)}, p1[4] = {v_wR, lo2(Rv), pk2(Rv.y, Rv.z), hi2(Rv)};
    const f2 m0[4] = {v_wx, hi2(Lv), pk2(Lv.y, Lv.z), lo2(Lv)}, m1[4] = {v_yz, lo2(cv), v_wx, hi2(Lv)};
#pragma unroll
    for (int d = 0; d < 4; d++) {
      zpv[0][d] = p0[d];
      zpv[1][d] = p1[d];
      zmv[0][d] = m0[d];
      zmv[1][d] = m1[d];
    }
  }
  const f2 sx = pk2(a.sx, a.sx), sz = pk2(a.sz, a.sz), wx2 = pk2(wxv, wxv);
  f2 n2[2];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    auto P = [h](const float4 &v) { return h ? hi2(v) : lo2(v); };
    // sample i of the x window and the z sample pair at +-d (times vv for LapT)
    auto tx = [&](int i) { return ADJ ? mul2(mul2(P(ux[i]), P(vx[i])), k1) : P(ux[i]); };
    auto tzp = [&](int d) { return ADJ ? mul2(mul2(zpu[h][d - 1], zpv[h][d - 1]), k1) : zpu[h][d - 1]; };
    auto tzm = [&](int d) { return ADJ ? mul2(mul2(zmu[h][d - 1], zmv[h][d - 1]), k1) : zmu[h][d - 1]; };
    const f2 t0 = ADJ ? mul2(mul2(P(ux[4]), P(vx[4])), k1) : P(ux[4]);
    f2 xs = mul2(mul2(kc[4], add2(tx(8), tx(0))), k1);
    xs = add2(xs, mul2(mul2(kc[3], add2(tx(7), tx(1))), k1));
    xs = add2(xs, mul2(mul2(kc[2], add2(tx(6), tx(2))), k1));
    xs = add2(xs, mul2(mul2(kc[1], add2(tx(5), tx(3))), k1));
    xs = add2(xs, mul2(mul2(kc[0], t0), k1));
    f2 zs = mul2(mul2(kc[4], add2(tzp(4), tzm(4))), k1);
    zs = add2(zs, mul2(mul2(kc[3], add2(tzp(3), tzm(3))), k1));
    zs = add2(zs, mul2(mul2(kc[2], add2(tzp(2), tzm(2))), k1));
    zs = add2(zs, mul2(mul2(kc[1], add2(tzp(1), tzm(1))), k1));
    zs = add2(zs, mul2(mul2(kc[0], t0), k1));
    f2 lap = add2(mul2(mul2(xs, sx), k1), mul2(mul2(zs, sz), k1));
    if (!ADJ) lap = mul2(mul2(lap, P(vx[4])), k1);
    const f2 u0 = mul2(mul2(mul2(P(B), P(wz4)), wx2), k1);
    n2[h] = sub2(add2(lap, add2(P(ux[4]), P(ux[4]))), u0);
  }
  float4 n = join2(n2[0], n2[1]);
#pragma unroll
  for (int e = 0; e < 4; e++) {
    float v = qel(n, e);
    if (!ADJ) {
      if (f & (32u << e)) v = fadd(v, fmul(qel(inj, e), qel(vx[4], e)));
    } else {
      if ((f & (1u << 9)) && e == a.depth - 4 * k) v = fadd(v, inj.x);
    }
    qset(n, e, v);
  }
  float4 r = join2(mul2(mul2(lo2(n), lo2(wz4)), wx2), mul2(mul2(hi2(n), hi2(wz4)), wx2));
#pragma unroll
  for (int e = 0; e < 4; e++)
    if (!(f & (2u << e))) qset(r, e, 0.f);
  return r;
}

// the next step's injected samples of one quad
template <bool ADJ>
__device__ __forceinline__ float4 load_inj(const Args &a, const float *mod, const float *dat,
                                           unsigned f, int ix, int k, int it) {
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  if (it < 0 || it >= a.nt) return v;
  if (!ADJ) {
    const long long row = ((long long)it * a.nx + (ix - a.nb)) * a.nz - a.nb + 4 * k;
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (f & (32u << e)) qset(v, e, __ldcs(mod + row + e));
  } else if (f & (1u << 9)) {
    v.x = __ldcs(dat + (size_t)(ix - a.nb) * a.nt + it);
  }
  return v;
}

// what a step writes besides the fields: modelling records the data row of
// A (before the step), the adjoint images A vv on the interior
template <bool ADJ>
__device__ __forceinline__ void quad_out(const Args &a, float *mod, float *dat, unsigned f,
                                         const float4 &A, const float4 &V, int ix, int k, int it) {
  if (!ADJ) {
    if (f & (1u << 9)) {
      const int e = a.depth - 4 * k;
      dat[(size_t)(ix - a.nb) * a.nt + it] = fadd(0.f, qel(A, e));
    }
  } else if (f & (0xFu << 5)) {
    const long long row = ((long long)it * a.nx + (ix - a.nb)) * a.nz - a.nb + 4 * k;
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (f & (32u << e)) __stcs(mod + row + e, fadd(0.f, fmul(qel(A, e), qel(V, e))));
  }
}

__device__ __forceinline__ unsigned cl_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cl_size() {
  unsigned n;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(n));
  return n;
}
__device__ __forceinline__ void cl_sync() {
  asm volatile("barrier.cluster.arrive.release;\nbarrier.cluster.wait.acquire;\n" ::: "memory");
}
__device__ __forceinline__ float4 *cl_map(float4 *p, unsigned rank) {
  unsigned long long r;
  asm volatile("mapa.u64 %0, %1, %2;\n" : "=l"(r) : "l"(p), "r"(rank));
  return reinterpret_cast<float4 *>(r);
}

template <bool ADJ, int IPT>
__global__ void __launch_bounds__(RNTH) resident_kernel(const __grid_constant__ Args a) {
  extern __shared__ float4 sm[];
  const unsigned rank = cl_rank(), ncta = cl_size();
  const int shot = blockIdx.x / ncta;
  const int w = a.w, nq = a.nq, arr = (w + 8) * nq;
  float4 *F0 = sm, *F1 = sm + arr, *Vs = sm + 2 * arr;
  float4 *wzs = sm + 3 * arr;                             // [nq]
  float *wxs = reinterpret_cast<float *>(wzs + nq);       // [w]
  const int x0 = (int)rank * w;
  float *mod = a.mod + (size_t)shot * a.mod_stride;
  float *dat = a.dat + (size_t)shot * a.dat_stride;
  for (int i = threadIdx.x; i < 2 * arr; i += RNTH) sm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < arr; i += RNTH) {
    const int c = i / nq, k = i - c * nq, ix = x0 + c - 4;
    Vs[i] = (ix >= 0 && ix < a.nxp) ? a.vv[(size_t)ix * nq + k] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int i = threadIdx.x; i < nq; i += RNTH) wzs[i] = a.wz[i];
  for (int i = threadIdx.x; i < w; i += RNTH) wxs[i] = x0 + i < a.nxp ? a.wx[x0 + i] : 1.f;
  // this thread's quads, packed: quad_flags bits 0-9, bit 10 / 11 the edge
  // column is also stored into the left / right neighbour's halo, band
  // column c in bits 12-21, z quad k in bits 22-31 (nq and w below 1024)
  unsigned pf[IPT];
#pragma unroll
  for (int j = 0; j < IPT; j++) {
    const int item = threadIdx.x + j * RNTH;
    const int c = item / nq, k = item - c * nq, ix = x0 + c;
    unsigned f = (item < w * nq && ix < a.nxp) ? quad_flags(a, ix, k) : 0u;
    if (f) {
      if (c < 4 && rank > 0) f |= 1u << 10;
      if (c >= w - 4 && rank + 1 < ncta) f |= 1u << 11;
      f |= ((unsigned)c << 12) | ((unsigned)k << 22);
    }
    pf[j] = f;
  }
  // the injected samples of the coming step, loaded one step ahead (each
  // quad's next samples are requested right after its update)
  float4 inj[IPT];
#pragma unroll
  for (int j = 0; j < IPT; j++)
    inj[j] = pf[j] ? load_inj<ADJ>(a, mod, dat, pf[j], x0 + (int)((pf[j] >> 12) & 1023u),
                                   (int)(pf[j] >> 22), ADJ ? a.nt - 1 : 0)
                   : make_float4(0.f, 0.f, 0.f, 0.f);
  cl_sync();  // every CTA's arrays are set before any halo store
  for (int s = 0; s < a.nt; s++) {
    const int it = ADJ ? a.nt - 1 - s : s;
    const float4 *cur = (s & 1) ? F1 : F0;
    float4 *nxt = (s & 1) ? F0 : F1;
#pragma unroll
    for (int j = 0; j < IPT; j++) {
      const unsigned f = pf[j];
      if (!f) continue;
      const int c = (int)((f >> 12) & 1023u), k = (int)(f >> 22), ix = x0 + c;
      const int o = (c + 4) * nq + k;
      float4 ux[9], vx[9];
#pragma unroll
      for (int d = 0; d < 9; d++) ux[d] = cur[o + (d - 4) * nq];
      const float4 uzl = cur[o - 1], uzh = cur[o + 1];
      float4 vzl = make_float4(0.f, 0.f, 0.f, 0.f), vzh = vzl;
      if (ADJ) {
#pragma unroll
        for (int d = 0; d < 9; d++) vx[d] = Vs[o + (d - 4) * nq];
        vzl = Vs[o - 1];
        vzh = Vs[o + 1];
      } else {
#pragma unroll
        for (int d = 0; d < 9; d++) vx[d] = vzl;
        vx[4] = Vs[o];
      }
      quad_out<ADJ>(a, mod, dat, f, ux[4], vx[4], ix, k, it);
      const float4 r = quad_step<ADJ>(a, f, ux, uzl, uzh, vx, vzl, vzh, nxt[o], wzs[k], wxs[c],
                                      inj[j], k);
      inj[j] = load_inj<ADJ>(a, mod, dat, f, ix, k, ADJ ? it - 1 : it + 1);
      nxt[o] = r;
      if (f & (1u << 10)) *cl_map(nxt + o + w * nq, rank - 1) = r;
      if (f & (1u << 11)) *cl_map(nxt + o - w * nq, rank + 1) = r;
    }
    cl_sync();
  }
}

template <bool ADJ>
__global__ void __launch_bounds__(SNTH) step_kernel(const Args a) {
  const int shot = blockIdx.y;
  const long long item = (long long)blockIdx.x * SNTH + threadIdx.x;
  const int nq = a.nq;
  const int ix = (int)(item / nq), k = (int)(item - (long long)ix * nq);
  if (ix >= a.nxp) return;
  const unsigned f = quad_flags(a, ix, k);
  if (!f) return;
  const float4 *__restrict__ X = a.X + (size_t)shot * a.fstride;
  float4 *__restrict__ Y = a.Y + (size_t)shot * a.fstride;
  const float4 *__restrict__ V = a.vv;
  float *mod = a.mod + (size_t)shot * a.mod_stride;
  float *dat = a.dat + (size_t)shot * a.dat_stride;
  const size_t o = (size_t)ix * nq + k;
  float4 ux[9], vx[9];
#pragma unroll
  for (int d = 0; d < 9; d++) ux[d] = __ldg(X + o + (long long)(d - 4) * nq);
  const float4 uzl = __ldg(X + o - 1), uzh = __ldg(X + o + 1);
  float4 vzl = make_float4(0.f, 0.f, 0.f, 0.f), vzh = vzl;
  if (ADJ) {
#pragma unroll
    for (int d = 0; d < 9; d++) vx[d] = __ldg(V + o + (long long)(d - 4) * nq);
    vzl = __ldg(V + o - 1);
    vzh = __ldg(V + o + 1);
  } else {
#pragma unroll
    for (int d = 0; d < 9; d++) vx[d] = vzl;
    vx[4] = __ldg(V + o);
  }
  const float4 inj = load_inj<ADJ>(a, mod, dat, f, ix, k, a.it);
  quad_out<ADJ>(a, mod, dat, f, ux[4], vx[4], ix, k, a.it);
  Y[o] = quad_step<ADJ>(a, f, ux, uzl, uzh, vx, vzl, vzh, Y[o], a.wz[k], a.wx[ix], inj, k);
}

// vvpad = (v v) dt^2 on the padded grid, the interior replicated onto every
// face (timerev_init, wave_triutil.c:63-78); vel [nx][nz]
__global__ void pad_vv_kernel(const float *__restrict__ vel, int nz, int nx, int nb, int nzp,
                              int nxp, int nq, float dt2, float *__restrict__ vv) {
  const size_t n = (size_t)nxp * nq * 4;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i / (4 * (size_t)nq)), iz = (int)(i - (size_t)ix * 4 * nq);
    float v = 0.f;
    if (iz < nzp) {
      const int jx = min(max(ix - nb, 0), nx - 1), jz = min(max(iz - nb, 0), nz - 1);
      const float u = vel[(size_t)jx * nz + jz];
      v = fmul(fmul(u, u), dt2);
    }
    vv[i] = v;
  }
}

// ---------------------------------------------------------- CG kernels --
// Deterministic FP64 sums: every thread adds a fixed strided subset, blocks
// reduce in a fixed tree, the final kernel adds the block sums in block
// order.  Products of two floats are exact in double.

// data side: gg.gg, Ss.Ss, gg.Ss, gg.rr, Ss.rr, rr.rr
__global__ void __launch_bounds__(DOTT) dots_kernel(const float *__restrict__ gg,
                                                    const float *__restrict__ Ss,
                                                    const float *__restrict__ rr, size_t n,
                                                    double *__restrict__ part) {
  __shared__ double sh[6][DOTT];
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = (size_t)blockIdx.x * DOTT + threadIdx.x; i < n; i += (size_t)DOTB * DOTT) {
    const double g = gg[i], S = Ss[i], r = rr[i];
    s[0] = __dadd_rn(s[0], __dmul_rn(g, g));
    s[1] = __dadd_rn(s[1], __dmul_rn(S, S));
    s[2] = __dadd_rn(s[2], __dmul_rn(g, S));
    s[3] = __dadd_rn(s[3], __dmul_rn(g, r));
    s[4] = __dadd_rn(s[4], __dmul_rn(S, r));
    s[5] = __dadd_rn(s[5], __dmul_rn(r, r));
  }
#pragma unroll
  for (int q = 0; q < 6; q++) sh[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int h = DOTT / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < 6; q++) sh[q][threadIdx.x] = __dadd_rn(sh[q][threadIdx.x], sh[q][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x < 6) part[(size_t)blockIdx.x * 8 + threadIdx.x] = sh[threadIdx.x][0];
}

// model side: g.g into slot 6
__global__ void __launch_bounds__(DOTT) sumsq_kernel(const float *__restrict__ g, size_t n,
                                                     double *__restrict__ part) {
  __shared__ double sh[DOTT];
  double s = 0;
  for (size_t i = (size_t)blockIdx.x * DOTT + threadIdx.x; i < n; i += (size_t)DOTB * DOTT) {
    const double v = g[i];
    s = __dadd_rn(s, __dmul_rn(v, v));
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = DOTT / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)blockIdx.x * 8 + 6] = sh[0];
}

__global__ void dots_final_kernel(const double *__restrict__ part, double *__restrict__ out) {
  const int q = threadIdx.x;
  if (q >= 7) return;
  double s = 0;
  for (int b = 0; b < DOTB; b++) s = __dadd_rn(s, part[(size_t)b * 8 + q]);
  out[q] = s;
}

// np_cgstep's update of one side (wave_cgstep.c:58-66): S = beta S +
// alfa g (sscal, then saxpy), x += S; forget starts S from zero
__global__ void cg_update_kernel(float *__restrict__ S, float *__restrict__ x,
                                 const float *__restrict__ g, size_t n, float alfa, float beta,
                                 int forget) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float s = forget ? 0.f : S[i];
    s = fmul(s, beta);
    s = fadd(s, fmul(alfa, g[i]));
    S[i] = s;
    x[i] = fadd(x[i], s);
  }
}

__global__ void negate_kernel(const float *__restrict__ d, float *__restrict__ r, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    r[i] = -d[i];
}

// ----------------------------------------------------------------- host --
struct Plan {
  int nzp, nxp, nq, depth;
  bool resident;
  int C, w, ipt;
  size_t smem;
  void *fn;
};

template <bool ADJ>
static void *resident_fn(int ipt) {
  switch (ipt) {
    case 1: return (void *)resident_kernel<ADJ, 1>;
    case 2: return (void *)resident_kernel<ADJ, 2>;
    case 3: return (void *)resident_kernel<ADJ, 3>;
    case 4: return (void *)resident_kernel<ADJ, 4>;
    case 5: case 6: return (void *)resident_kernel<ADJ, 6>;
    default: return (void *)resident_kernel<ADJ, 8>;
  }
}

static int check_args(const pw_fwi_args *a, bool need_shots) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null argument struct");
  PW_CHECK(a->nz >= 1 && a->nx >= 1 && a->nt >= 1, PW_ERR_SHAPE,
           "nz, nx, nt must be positive (got %d, %d, %d)", a->nz, a->nx, a->nt);
  PW_CHECK(!need_shots || a->ns >= 1, PW_ERR_SHAPE, "ns must be positive (got %d)", a->ns);
  PW_CHECK(a->nb >= 4, PW_ERR_SHAPE,
           "lstri needs a sponge of at least 4 cells (nb = %d): the stencil's rim must stay "
           "free of sources and receivers", a->nb);
  const int nzp = a->nz + 2 * a->nb, depth = a->rz + a->nb;
  PW_CHECK(depth >= 4 && depth < nzp - 4, PW_ERR_SHAPE,
           "receiver depth rz = %d puts the data row outside the stencil's rows", a->rz);
  PW_CHECK(a->dz > 0.f && a->dx > 0.f && std::isfinite(a->dz) && std::isfinite(a->dx),
           PW_ERR_VALUE, "dz and dx must be positive");
  PW_CHECK((a->nz + 2LL * a->nb + 4) * (a->nx + 2LL * a->nb) < (1LL << 31), PW_ERR_SHAPE,
           "padded grid too large");
  return PW_OK;
}

// Resident plan: the largest cluster (16, 8, 4, 2 CTAs, one per SM) whose
// bands of at least 4 columns fit in shared memory and that the device can
// schedule; otherwise (or with PW_LSTRI_RESIDENT=0) the step-per-launch path.
// The adjoint (LapT reads 9 more vv quads per quad) takes the step path
// where its resident form would need a 16-CTA cluster: on the passive
// demos' grid (250 x 454 padded, nt 3001) one adjoint application runs
// 12.4 ms step by step against 15.2 ms resident, while the modelling stays
// resident (11.7 against 12.4 ms).  PW_LSTRI_RESIDENT=1 keeps every
// operator resident where it fits.
static void make_plan(const pw_fwi_args *a, bool adj, Plan &p) {
  p.nzp = a->nz + 2 * a->nb;
  p.nxp = a->nx + 2 * a->nb;
  p.nq = (p.nzp + 3) / 4;
  p.depth = a->rz + a->nb;
  p.resident = false;
  const char *env = getenv("PW_LSTRI_RESIDENT");
  if (env && env[0] == '0') return;
  const bool force = env && env[0] == '1';
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  for (int C : {16, 8, 4, 2}) {
    const int w = (p.nxp + C - 1) / C;
    if (w < 4) continue;
    const int ipt = (w * p.nq + RNTH - 1) / RNTH;
    if (ipt > RMAXIPT) break;
    if (w >= 1024 || p.nq >= 1024) break;  // packed quad descriptors
    const size_t smem = ((size_t)3 * (w + 8) * p.nq + p.nq) * sizeof(float4) + (size_t)w * 4;
    if (smem > (size_t)maxsm) break;
    void *fn = adj ? resident_fn<true>(ipt) : resident_fn<false>(ipt);
    static std::mutex mu;
    static std::map<std::pair<int, void *>, size_t> attr_max;
    static std::map<std::tuple<int, void *, size_t, int>, bool> seen;
    bool ok = true;
    {
      std::lock_guard<std::mutex> lock(mu);
      size_t &am = attr_max[std::make_pair(dev, fn)];
      if (smem > am) {
        ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
             cudaSuccess;
        if (ok) am = smem;
      }
      if (ok && C > 8)
        ok = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
             cudaSuccess;
      const auto key = std::make_tuple(dev, fn, smem, C);
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
        cfg.blockDim = dim3(RNTH);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        ok = cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters >= 1;
        seen[key] = ok;
      }
      cudaGetLastError();
    }
    if (!ok) continue;
    if (adj && C == 16 && !force) return;
    p.resident = true;
    p.C = C;
    p.w = w;
    p.ipt = ipt;
    p.smem = smem;
    p.fn = fn;
    return;
  }
}

// the reference's constants and sponge (tri2d_make, pfwiabc_cal): 1/dx^2,
// 1/dz^2 and the 8th-order coefficients rounded to float, decay[ib] =
// exp(-c*c*(nb-1-ib)^2) with the exponent in float and exp in double
static void base_args(const pw_fwi_args *a, const Plan &p, Args &g, std::vector<float> &wz,
                      std::vector<float> &wx) {
  g = Args{};
  g.nzp = p.nzp;
  g.nxp = p.nxp;
  g.nq = p.nq;
  g.nz = a->nz;
  g.nx = a->nx;
  g.nt = a->nt;
  g.nb = a->nb;
  g.depth = p.depth;
  volatile float dx = a->dx, dz = a->dz;
  g.sx = 1.0f / (dx * dx);
  g.sz = 1.0f / (dz * dz);
  volatile float n205 = -205.0f, n1 = -1.0f, p8 = 8.0f;
  g.c0 = n205 / 72.0f;
  g.c1 = p8 / 5.0f;
  g.c2 = n1 / 5.0f;
  g.c3 = p8 / 315.0f;
  g.c4 = n1 / 560.0f;
  g.one = 1.f;
  std::vector<float> decay(a->nb);
  for (int ib = 0; ib < a->nb; ib++) {
    const float c = a->coef;
    const float e = -c * c * (float)(a->nb - 1 - ib) * (float)(a->nb - 1 - ib);
    decay[ib] = (float)std::exp((double)e);
  }
  wz.assign((size_t)4 * p.nq, 1.f);
  for (int iz = 0; iz < a->nb; iz++) {
    wz[iz] = decay[iz];
    wz[p.nzp - 1 - iz] = decay[iz];
  }
  wx.assign(p.nxp, 1.f);
  for (int ix = 0; ix < a->nb; ix++) {
    wx[ix] = decay[ix];
    wx[p.nxp - 1 - ix] = decay[ix];
  }
}

// Device tables of one call, carved from the workspace.
struct Tables {
  size_t o_vv, o_wz, o_wx, o_vel;
};
static void carve_tables(const pw_fwi_args *a, const Plan &p, bool host, Carve &cv, Tables &t) {
  t.o_vv = cv.add((size_t)p.nxp * p.nq * sizeof(float4));
  t.o_wz = cv.add((size_t)p.nq * sizeof(float4));
  t.o_wx = cv.add((size_t)p.nxp * sizeof(float));
  t.o_vel = cv.add(host ? (size_t)a->nz * a->nx * 4 : 0);
}
static int upload_tables(const pw_fwi_args *a, const Plan &p, const Tables &t, char *base,
                         const float *vel, bool host, cudaStream_t st, Args &g) {
  std::vector<float> wz, wx;
  base_args(a, p, g, wz, wx);
  const float *d_vel = vel;
  if (host) {
    PW_TRY(to_device(base + t.o_vel, vel, (size_t)a->nz * a->nx * 4, true, st));
    d_vel = at<float>(base, t.o_vel);
  }
  PW_CUDA(cudaMemcpyAsync(base + t.o_wz, wz.data(), wz.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + t.o_wx, wx.data(), wx.size() * 4, cudaMemcpyHostToDevice, st));
  volatile float dt = a->dt;
  const float dt2 = dt * dt;
  pad_vv_kernel<<<592, 256, 0, st>>>(d_vel, a->nz, a->nx, a->nb, p.nzp, p.nxp, p.nq, dt2,
                                     at<float>(base, t.o_vv));
  PW_CUDA(cudaGetLastError());
  // the host vectors must outlive the asynchronous copies
  PW_CUDA(cudaStreamSynchronize(st));
  g.vv = at<float4>(base, t.o_vv);
  g.wz = at<float4>(base, t.o_wz);
  g.wx = at<float>(base, t.o_wx);
  return PW_OK;
}

// One application of the operator to nshots shots (mod / dat strides in
// Args).  fields: 2 * nshots fields for the step path (unused when
// resident).  Returns the number of kernel launches through `launches`.
static int run_op(const Plan &p, Args g, bool adj, int nshots, float4 *fields, cudaStream_t st,
                  long long &launches) {
  if (p.resident) {
    g.w = p.w;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = p.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(p.C * nshots));
    cfg.blockDim = dim3(RNTH);
    cfg.dynamicSmemBytes = p.smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&g};
    PW_CUDA(cudaLaunchKernelExC(&cfg, p.fn, args));
    launches += 1;
    return PW_OK;
  }
  g.fstride = (size_t)p.nxp * p.nq;
  float4 *F0 = fields, *F1 = fields + (size_t)nshots * g.fstride;
  PW_CUDA(cudaMemsetAsync(fields, 0, (size_t)2 * nshots * g.fstride * sizeof(float4), st));
  const dim3 grid((unsigned)ceil_div((long long)p.nxp * p.nq, SNTH), (unsigned)nshots);
  for (int s = 0; s < g.nt; s++) {
    g.it = adj ? g.nt - 1 - s : s;
    g.X = (s & 1) ? F1 : F0;
    g.Y = (s & 1) ? F0 : F1;
    if (adj) step_kernel<true><<<grid, SNTH, 0, st>>>(g);
    else step_kernel<false><<<grid, SNTH, 0, st>>>(g);
    PW_CUDA(cudaGetLastError());
    launches += 1;
  }
  return PW_OK;
}

static void print_plan(const char *what, const Plan &p, int nshots) {
  if (!getenv("PW_LSTRI_VERBOSE")) return;
  if (p.resident)
    fprintf(stderr, "lstri %s plan: resident cluster %d x %d threads, %d columns per CTA, "
            "%zu B smem, %d shot(s) per launch, padded %d x %d\n",
            what, p.C, RNTH, p.w, p.smem, nshots, p.nzp, p.nxp);
  else
    fprintf(stderr, "lstri %s plan: step per launch, padded %d x %d, %d shot(s)\n", what, p.nzp,
            p.nxp, nshots);
}

}  // namespace tr
}  // namespace pw

using namespace pw;
using namespace pw::tr;

// timerev_lop (wave_triutil.c:86-180) with add = false, one shot:
// adj = 0 maps mod [nt][nx][nz] to dat [nx][nt]; adj = 1 maps dat to mod.
extern "C" int pw_timerev(const pw_fwi_args *a, int adj, const float *vel, float *mod, float *dat,
                          void *stream) {
  PW_TRY(check_args(a, false));
  PW_CHECK(vel && mod && dat, PW_ERR_VALUE, "null array");
  cudaStream_t st = (cudaStream_t)stream;
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  Plan p;
  make_plan(a, adj != 0, p);
  print_plan(adj ? "adjoint" : "modelling", p, 1);
  const size_t nm = (size_t)a->nz * a->nx * a->nt, nd = (size_t)a->nx * a->nt;
  Carve cv;
  Tables t;
  carve_tables(a, p, host, cv, t);
  const size_t o_f = cv.add(p.resident ? 0 : (size_t)2 * p.nxp * p.nq * sizeof(float4));
  const size_t o_m = cv.add(host ? nm * 4 : 0);
  const size_t o_d = cv.add(host ? nd * 4 : 0);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  Args g;
  PW_TRY(upload_tables(a, p, t, base, vel, host, st, g));
  float *dm = host ? at<float>(base, o_m) : mod;
  float *dd = host ? at<float>(base, o_d) : dat;
  if (host) {
    if (adj) PW_TRY(to_device(dd, dat, nd * 4, true, st));
    else PW_TRY(to_device(dm, mod, nm * 4, true, st));
  }
  g.mod = dm;
  g.dat = dd;
  long long launches = 0;
  LoopTimer timer(st);
  timer.start();
  PW_TRY(run_op(p, g, adj != 0, 1, at<float4>(base, o_f), st, launches));
  timer.stop();
  if (host) {
    if (adj) PW_TRY(to_host(mod, dm, nm * 4, true, st));
    else PW_TRY(to_host(dat, dd, nd * 4, true, st));
  }
  timer.finish(launches, launches + 1);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

// lstric with inv = 0 (pfwi.c:1031-1444, wave_fwi.c:121-175): data
// [ns][nx][nt] of every shot's source field src [ns][nt][nx][nz]; all shots
// in one launch on the resident path.
extern "C" int pw_lstri_forward(const pw_fwi_args *a, const float *vel, const float *src,
                                float *data, void *stream) {
  PW_TRY(check_args(a, true));
  PW_CHECK(vel && src && data, PW_ERR_VALUE, "null array");
  cudaStream_t st = (cudaStream_t)stream;
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  Plan p;
  make_plan(a, false, p);
  const int ns = a->ns;
  print_plan("modelling", p, ns);
  const size_t nm = (size_t)a->nz * a->nx * a->nt, nd = (size_t)a->nx * a->nt;
  Carve cv;
  Tables t;
  carve_tables(a, p, host, cv, t);
  const size_t o_f = cv.add(p.resident ? 0 : (size_t)2 * ns * p.nxp * p.nq * sizeof(float4));
  const size_t o_m = cv.add(host ? nm * ns * 4 : 0);
  const size_t o_d = cv.add(host ? nd * ns * 4 : 0);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  Args g;
  PW_TRY(upload_tables(a, p, t, base, vel, host, st, g));
  float *dm = host ? at<float>(base, o_m) : const_cast<float *>(src);
  float *dd = host ? at<float>(base, o_d) : data;
  if (host) PW_TRY(to_device(dm, src, nm * ns * 4, true, st));
  g.mod = dm;
  g.dat = dd;
  g.mod_stride = nm;
  g.dat_stride = nd;
  long long launches = 0;
  LoopTimer timer(st);
  timer.start();
  PW_TRY(run_op(p, g, false, ns, at<float4>(base, o_f), st, launches));
  timer.stop();
  if (host) PW_TRY(to_host(data, dd, nd * ns * 4, true, st));
  timer.finish(launches, launches + 1);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

// lstric with inv = 1 (pfwi.c:1031-1444, wave_fwi.c:121-175,
// wave_fwigradient.c:454-520): per shot, np_solver (wave_bigsolver.c:1170)
// with np_cgstep (wave_cgstep.c:16) for niter iterations from a zero model,
// src [ns][nt][nx][nz] from data [ns][nx][nt].  The CG step vectors persist
// from shot to shot within the call and start from zero at its first step,
// as the reference's static S, Ss do (never released by lstric).  FP64 dots
// are summed in a fixed block order (the reference sums sequentially); the
// stopping test (ratio of float sums of squares below 1e-12 in the
// reference) uses the same FP64 sums.
extern "C" int pw_lstri_invert(const pw_fwi_args *a, const float *vel, const float *data,
                               float *src, void *stream) {
  PW_TRY(check_args(a, true));
  PW_CHECK(vel && src && data, PW_ERR_VALUE, "null array");
  PW_CHECK(a->niter >= 0, PW_ERR_VALUE, "niter must be non-negative (got %d)", a->niter);
  cudaStream_t st = (cudaStream_t)stream;
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  Plan pa, pf;
  make_plan(a, true, pa);
  make_plan(a, false, pf);
  print_plan("adjoint", pa, 1);
  print_plan("modelling", pf, 1);
  const int ns = a->ns;
  const size_t nm = (size_t)a->nz * a->nx * a->nt, nd = (size_t)a->nx * a->nt;
  Carve cv;
  Tables t;
  carve_tables(a, pa, host, cv, t);
  const bool fields = !(pa.resident && pf.resident);
  const size_t o_f = cv.add(fields ? (size_t)2 * pa.nxp * pa.nq * sizeof(float4) : 0);
  const size_t o_x = cv.add(host ? nm * 4 : 0);
  const size_t o_g = cv.add(nm * 4);
  const size_t o_S = cv.add(nm * 4);
  const size_t o_dat = cv.add(host ? nd * 4 : 0);
  const size_t o_rr = cv.add(nd * 4);
  const size_t o_gg = cv.add(nd * 4);
  const size_t o_Ss = cv.add(nd * 4);
  const size_t o_part = cv.add((size_t)DOTB * 8 * sizeof(double));
  const size_t o_dots = cv.add(8 * sizeof(double));
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  Args g;
  PW_TRY(upload_tables(a, pa, t, base, vel, host, st, g));
  float *gv = at<float>(base, o_g), *S = at<float>(base, o_S);
  float *rr = at<float>(base, o_rr), *gg = at<float>(base, o_gg), *Ss = at<float>(base, o_Ss);
  double *part = at<double>(base, o_part), *dots = at<double>(base, o_dots);
  float4 *fl = at<float4>(base, o_f);
  PW_CUDA(cudaMemsetAsync(S, 0, nm * 4, st));
  PW_CUDA(cudaMemsetAsync(Ss, 0, nd * 4, st));
  const double EPS = (double)1.e-12f, TOL = (double)1.e-12f;
  bool first_step = true;  // np_cgstep's "Allocated" flag
  long long launches = 0;
  double h[8];
  auto reduce = [&](bool model) -> int {
    dots_kernel<<<DOTB, DOTT, 0, st>>>(gg, Ss, rr, nd, part);
    if (model) sumsq_kernel<<<DOTB, DOTT, 0, st>>>(gv, nm, part);
    dots_final_kernel<<<1, 32, 0, st>>>(part, dots);
    PW_CUDA(cudaGetLastError());
    launches += model ? 3 : 2;
    PW_CUDA(cudaMemcpyAsync(h, dots, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
    return PW_OK;
  };
  LoopTimer timer(st);
  timer.start();
  for (int is = 0; is < ns; is++) {
    float *x = host ? at<float>(base, o_x) : src + (size_t)is * nm;
    const float *dat = host ? at<float>(base, o_dat) : data + (size_t)is * nd;
    if (host) PW_TRY(to_device(at<float>(base, o_dat), data + (size_t)is * nd, nd * 4, true, st));
    negate_kernel<<<592, 256, 0, st>>>(dat, rr, nd);
    PW_CUDA(cudaGetLastError());
    PW_CUDA(cudaMemsetAsync(x, 0, nm * 4, st));
    PW_CUDA(cudaMemsetAsync(gg, 0, nd * 4, st));
    PW_TRY(reduce(false));
    const double dpr0 = h[5];
    double dpg0 = 1.0;
    for (int iter = 0; iter < a->niter; iter++) {
      Args ga = g;
      ga.mod = gv;
      ga.dat = rr;
      PW_TRY(run_op(pa, ga, true, 1, fl, st, launches));
      Args gf = g;
      gf.mod = gv;
      gf.dat = gg;
      PW_TRY(run_op(pf, gf, false, 1, fl, st, launches));
      PW_TRY(reduce(true));
      const double gdg = h[0], sds = h[1], gds = h[2], gdr = -h[3], sdr = -h[4];
      double dpr, dpg;
      if (iter == 0) {
        dpg0 = h[6];
        dpr = 1.0;
        dpg = 1.0;
      } else {
        dpr = h[5] / dpr0;
        dpg = h[6] / dpg0;
      }
      if (dpr < TOL || dpg < TOL) break;
      // np_cgstep
      const bool forget = first_step;
      first_step = false;
      double alfa, beta;
      if (forget) {
        beta = 0.0;
        alfa = gdg;
        if (alfa <= 0.) {
          PW_CUDA(cudaMemsetAsync(S, 0, nm * 4, st));
          PW_CUDA(cudaMemsetAsync(Ss, 0, nd * 4, st));
          continue;
        }
        alfa = gdr / alfa;
      } else {
        if (gdg == 0. || sds == 0.) continue;
        double determ = 1.0 - (gds / gdg) * (gds / sds);
        if (determ > EPS) determ *= gdg * sds;
        else determ = gdg * sds * EPS;
        alfa = (sds * gdr - gds * sdr) / determ;
        beta = (-gds * gdr + gdg * sdr) / determ;
      }
      cg_update_kernel<<<1184, 256, 0, st>>>(S, x, gv, nm, (float)alfa, (float)beta, forget);
      cg_update_kernel<<<592, 256, 0, st>>>(Ss, rr, gg, nd, (float)alfa, (float)beta, forget);
      PW_CUDA(cudaGetLastError());
      launches += 2;
    }
    if (host) PW_TRY(to_host(src + (size_t)is * nm, x, nm * 4, true, st));
  }
  timer.stop();
  timer.finish(launches, launches);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}
