// pfwi acoustic path on sm_100a: forward modelling, FWI gradients (the
// reference's gradient_av imaging and the exact discrete adjoint with
// checkpointing), residual / FP64 misfit and gradient post-processing.
//
// Scheme (pywave/src/wave_fwimodeling.c:72-104, wave_fwigradient.c:132-241):
//   term = Lap8(a) (zero outside [4,pad-4)) + rr*w[it]
//   a_new = S((2a - S(b)) + (v*v*dt^2)*term),   S = sponge, b = previous a
// on the padded grid (nz+2nb) x (nx+2nb).  Same field layout, two-buffer
// scheme and cp.async plane pipeline as the afd kernel, with an 8th-order
// stencil: the model's x is the marched axis (9-deep register queue), z is
// tiled (float4 per thread, one float4 of halo on each side = 4 cells).
// All shots of a call advance together, one after another inside each CTA,
// sharing the v^2 dt^2 plane.
#include "pw_common.cuh"

#include <algorithm>
#include <cfloat>
#include <map>
#include <mutex>
#include <cmath>

namespace pw {
namespace pf {

constexpr int HZ = 4;        // z halo (cells) in front of iz = 0
constexpr int HX = 4;        // x halo (planes) in front of ix = 0
constexpr int MAXS = 64;     // shots per launch
constexpr int MAXSRCW = 16;  // source-map cells per shot

// Shot geometry resolved on the host (preparation, wave_fwiutil.c:44-71).
struct ShotGeo {
  int r0v, r02, nr2;          // receivers rx = r0v + ir*drv, ir < nr2, stored at trace r02 + ir
  int nsrc;                   // non-zero source-map cells
  int sx0, sx1, sz0, sz1;     // bounding box of those cells
  int scell[MAXSRCW];         // (ix << 16) | iz of each cell
  float sw[MAXSRCW];          // source-map weight rr
};

enum Mode { FWD = 0, ADJ_REF = 1, ADJ_EXACT = 2 };

// Division by a constant d > 0 with the method of Brisebarre, Muller and
// Raina ("Accelerating correctly rounded floating-point division when the
// divisor is known in advance", IEEE Trans. Computers 53(8), 2004):
//   zh = RN(1/d), zl = RN(1/d - zh),  q = RN(x*zh + RN(x*zl))  (one FMA).
// It returns the correctly rounded x/d for every x only for some d, so each
// divisor is checked on the GPU against __fdiv_rn for all 2^23 significands
// of x in one binade; scaling x by 2^k scales every step exactly while the
// intermediate values stay normal, which |x| in [xmin, xmax] ensures.
// Below xmin (the tiny values at the edge of a wavefield, subnormal ones
// included) div_small scales x by 2^89 into that range, divides, and scales
// back, which is exact unless the quotient is subnormal and the scaled
// quotient sits exactly on a tie of the subnormal grid; there the sign of
// the exact remainder xs - qs*d (one FMA) picks the side.  The setup checks
// it against __fdiv_rn for every float in (0, xmin) as well.
// Above xmax, for NaN or infinity, or when a check fails: __fdiv_rn.
struct DivC {
  float d, zh, zl, xmin, xmax;
  int ok;
  unsigned int umin, uspan, umax;  // bits of xmin; of xmax minus xmin; of xmax
  float sup, sdn, sgrid;           // 2^K, 2^-K, 2^(149-K) for div_small
};
constexpr int DIV_SMALL_K = 89;

struct PfArgs {
  int pnz, pnx;               // padded grid
  int lz;                     // leading dimension of the field layout
  int nb, nz, nx;             // sponge width, interior
  float c0, c1, c2, c3, c4;   // 8th-order coefficients (wave_fwiutil.c:17)
  float dx2, dz2;
  float one;                  // 1.0f at run time: keeps packed products unfused (pk2 helpers)
  DivC divx, divz;            // fast exact division by dx2 / dz2
  int nshots;
  const float *cur[MAXS];
  float *nxt[MAXS];
  const float *V;             // v*v*dt^2 (field layout)
  const float *bz, *bx;       // sponge factor per z / x cell (1 off the faces)
  int it, nt;
  const ShotGeo *geo;         // [nshots] (device)
  int rz, drv, nr;
  const float *wav;           // forward: wavelet [nt]
  const float *dsrc;          // forward, passive sources: field [shot][nt][nx][nz] added to the
                              // term of every interior cell (replaces the wavelet), or null
  long long dsrc_stride;      // floats between the shots' source fields
  float *rec;                 // forward: traces [shot][nt][nr] or null
  float *snap;                // forward: interior snapshot for this step [shot][nx][nz] or null
  long long snap_stride;      // floats between shots' snapshots
  float *tout;                // forward: term output [shot] (field layout) or null
  long long tout_stride;
  const float *res;           // adjoint: residual [shot][nt][nr]
  // ADJ_REF imaging: grad[ix][iz] += (w1-2w0+wm1)/wdt2 * phi * (-2/v^3) in double
  const float *wprev, *wcur, *wnext;  // snapshots wit-1, wit, wit+1 [shot][nx][nz]
  long long wstride;
  float wdt2;
  const float *m2v3;          // (float)(-2/(double)v^3) per interior cell [nx][nz]
  float *grad;                // [nx][nz] (ADJ_REF) or field layout (ADJ_EXACT: sum phi*term)
  long long gstride;          // floats between the shots' gradient slices (0: one accumulator)
  const float *tin;           // ADJ_EXACT: term of the forward step [shot] (field layout)
  long long tin_stride;
  int imaging;                // this step images
  long long fstride;          // field size (floats)
};

__device__ __forceinline__ float el(const float4 &v, int e) {
  return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_el(float4 &v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ long long pfoff(int lz, int iz, int ix) {
  return (long long)(iz + HZ) + (long long)lz * (ix + HX);
}

__device__ __forceinline__ void cp16(float4 *dst, const float *src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp4(float *dst, const float *src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// z terms of the 8th-order Laplacian for cell e of the float4 c, with L / R
// the float4s below and above (cells -4..-1, +4..+7).
__device__ __forceinline__ float znb(const float4 &L, const float4 &c, const float4 &R, int e, int d) {
  const int j = e + d;  // -4 .. 7
  if (j < 0) return el(L, j + 4);
  if (j > 3) return el(R, j - 4);
  return el(c, j);
}

__device__ __forceinline__ float div_bmr(float x, const DivC &c) {
  // copysignf keeps the sign of a zero quotient (d > 0)
  return copysignf(__fmaf_rn(x, c.zh, __fmul_rn(x, c.zl)), x);
}

__device__ __forceinline__ float div_small(float x, const DivC &c) {
  const float xs = __fmul_rn(x, c.sup);  // exact, inside [xmin, xmax]
  const float qs = __fmaf_rn(xs, c.zh, __fmul_rn(xs, c.zl));
  const float q = copysignf(__fmul_rn(qs, c.sdn), x);
  const float t = fabsf(__fmul_rn(qs, c.sgrid));  // |qs| in units of 2^-149 (exact)
  const float n = truncf(t);
  if (t - n == 0.5f) {
    const float r = __fmaf_rn(-qs, c.d, xs);  // exact remainder
    if (r != 0.f)
      return __uint_as_float((__float2uint_rz(n) + ((r > 0.f) == (x > 0.f) ? 1u : 0u)) |
                             (__float_as_uint(x) & 0x80000000u));
  }
  return q;
}

// div_bmr on a pair: the same fused product and the sign of x per lane
__device__ __forceinline__ f2 div_bmr2(f2 x, f2 zh, f2 zl) {
  const f2 q = fma2(x, zh, mul2(x, zl));
  return (q & 0x7fffffff7fffffffull) | (x & 0x8000000080000000ull);
}

// tx[e]/cx.d and tz[e]/cz.d for the 4 cells of a float4, correctly rounded.
// The lanes of `mask` vote once: every numerator zero or in [xmin, xmax]
// runs div_bmr (two values per op); every one below xmax runs div_small or
// div_bmr per value; otherwise __fdiv_rn (a per-value choice of all three
// would be if-converted into every sequence).  Any grouping of lanes is
// correct, as every lane's own vote is in its group.
__device__ __forceinline__ void div4x2(const float (&tx)[4], const float (&tz)[4],
                                       const DivC &cx, const DivC &cz, unsigned mask,
                                       float (&qx)[4], float (&qz)[4]) {
  // |x| in [xmin, xmax] or 0 for all four: the largest |x| bits at most
  // umax, and the smallest of |x| bits - 1 (a zero wraps to the top and
  // drops out) at least umin - 1; positive floats order as their bits
  unsigned mxx = 0u, mxz = 0u, mnx = ~0u, mnz = ~0u;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const unsigned ux = __float_as_uint(tx[e]) & 0x7fffffffu;
    const unsigned uz = __float_as_uint(tz[e]) & 0x7fffffffu;
    mxx = max(mxx, ux);
    mxz = max(mxz, uz);
    mnx = min(mnx, ux - 1u);
    mnz = min(mnz, uz - 1u);
  }
  const bool ok = cx.ok && cz.ok;
  const bool in = ok && mxx <= cx.umax && mxz <= cz.umax && mnx >= cx.umin - 1u &&
                  mnz >= cz.umin - 1u;
  if (__all_sync(mask, in)) {
    const f2 xh = pk2(cx.zh, cx.zh), xl = pk2(cx.zl, cx.zl);
    const f2 zh = pk2(cz.zh, cz.zh), zl = pk2(cz.zl, cz.zl);
    up2(div_bmr2(pk2(tx[0], tx[1]), xh, xl), qx[0], qx[1]);
    up2(div_bmr2(pk2(tx[2], tx[3]), xh, xl), qx[2], qx[3]);
    up2(div_bmr2(pk2(tz[0], tz[1]), zh, zl), qz[0], qz[1]);
    up2(div_bmr2(pk2(tz[2], tz[3]), zh, zl), qz[2], qz[3]);
  } else if (__all_sync(mask, ok && mxx <= cx.umax && mxz <= cz.umax)) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const bool sx = (__float_as_uint(tx[e]) & 0x7fffffffu) < cx.umin;
      const bool sz = (__float_as_uint(tz[e]) & 0x7fffffffu) < cz.umin;
      qx[e] = sx ? div_small(tx[e], cx) : div_bmr(tx[e], cx);
      qz[e] = sz ? div_small(tz[e], cz) : div_bmr(tz[e], cz);
    }
  } else {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      qx[e] = __fdiv_rn(tx[e], cx.d);
      qz[e] = __fdiv_rn(tz[e], cz.d);
    }
  }
}

// One pfwi step over a z column segment of ZW float4 marching along x.
template <int ZW, int P, int MODE, bool PAS = false>
__global__ void __launch_bounds__(ZW) pf_step_kernel(const PfArgs a, int xch) {
  constexpr int W = ZW + 2;   // curr plane (float4) incl. z halo
  constexpr int NC = P + 10;  // curr planes (x-4..x+4 live, P ahead, 1 slack)
  constexpr int NP = P + 2;
  extern __shared__ float4 sm[];
  float4 *s_cur = sm;
  float4 *s_prev = sm + NC * W;
  float4 *s_V = s_prev + NP * ZW;
  float4 *s_t = s_V + NP * ZW;  // ADJ_EXACT: forward term tile
  float4 *s_g = s_t + NP * ZW;  // ADJ_EXACT: this shot's gradient slice
  float4 *s_d = s_t;            // FWD with passive sources: the step's source field

  const int tid = threadIdx.x;
  const int s = blockIdx.x;  // shot of the batch: fastest, so the shots of one x chunk
                             // run together and share V through L2
  const int z4 = blockIdx.z * ZW + tid;
  const int iz0 = 4 * z4;
  const int x0 = blockIdx.y * xch;
  const int x1 = min(a.pnx, x0 + xch);
  const int nplanes = x1 - x0;
  const int lz = a.lz;
  const bool live = iz0 < a.pnz;
  const long long o_c = pfoff(lz, iz0, 0);
  const int ci = tid + 1;
  const int hz4 = tid == 0 ? blockIdx.z * ZW - 1 : blockIdx.z * ZW + ZW;  // halo float4 (threads 0, 1)
  const bool has_h = tid < 2;
  const int hslot = tid == 0 ? 0 : ZW + 1;
  const bool h_ok = has_h && hz4 >= -1 && hz4 * 4 < a.pnz;
  const long long h_off = h_ok ? pfoff(lz, hz4 * 4, 0) : 0;

  float bzf[4];
  bool lz_ok[4], zin[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = iz0 + e;
    bzf[e] = (live && iz < a.pnz) ? a.bz[iz] : 1.f;
    lz_ok[e] = iz >= 4 && iz < a.pnz - 4;
    zin[e] = iz < a.pnz;
  }
  const bool rec_row = a.rz >= iz0 && a.rz < iz0 + 4;

  float *const gs = a.grad + s * a.gstride;  // this shot's gradient accumulator
  {
    const float *cur = a.cur[s];
    float *nxt = a.nxt[s];
    const float *tin = MODE == ADJ_EXACT ? a.tin + s * a.tin_stride : nullptr;
    const ShotGeo &sg = a.geo[s];
    const int r0v = sg.r0v, r02 = sg.r02, nr2 = sg.nr2;
    const int sx0 = sg.sx0, sx1 = sg.sx1;
    const bool src_z = MODE == FWD && iz0 <= sg.sz1 && iz0 + 3 >= sg.sz0;
    auto issue_cur = [&](int k) {  // plane x = x0 - 4 + k
      const int x = x0 - 4 + k;
      const bool xok = x >= -HX && x < a.pnx + HX;
      float4 *dst = s_cur + (k % NC) * W;
      const long long ox = (long long)lz * x;
      cp16(dst + ci, cur + (live && xok ? o_c + ox : 0), live && xok);
      if (has_h) cp16(dst + hslot, cur + (h_ok && xok ? h_off + ox : 0), h_ok && xok);
    };
    auto issue_pv = [&](int j) {  // plane x = x0 + j
      const long long o = o_c + (long long)lz * (x0 + j);
      cp16(s_prev + (j % NP) * ZW + tid, live ? nxt + o : nxt, live);
      cp16(s_V + (j % NP) * ZW + tid, live ? a.V + o : a.V, live);
      if (MODE == ADJ_EXACT) {
        cp16(s_t + (j % NP) * ZW + tid, live ? tin + o : tin, live && a.imaging);
        cp16(s_g + (j % NP) * ZW + tid, live ? gs + o : gs, live && a.imaging);
      }
      if (MODE == FWD && PAS) {
        // the interior cells' source samples of plane x0 + j (zero elsewhere)
        const int x = x0 + j;
        const bool xin = live && x >= a.nb && x < a.nb + a.nx;
        const float *row = a.dsrc + s * a.dsrc_stride +
                           ((long long)a.it * a.nx + (xin ? x - a.nb : 0)) * a.nz;
        float *dst = reinterpret_cast<float *>(s_d + (j % NP) * ZW + tid);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          const bool ok = xin && iz >= a.nb && iz < a.nb + a.nz;
          cp4(dst + e, ok ? row + (iz - a.nb) : a.dsrc, ok);
        }
      }
    };
    for (int k = 0; k < 8; k++) issue_cur(k);
#pragma unroll
    for (int b = 0; b < P; b++) {
      if (b < nplanes) {
        issue_cur(b + 8);
        issue_pv(b);
      }
      cp_commit();
    }
    float4 q[9];
    for (int i = 0; i < nplanes; i++) {
      const int x = x0 + i;
      // ADJ_REF imaging operands of this plane, loaded before the stencil so
      // their latency hides behind it
      double rw[4];
      float rt[4], rg[4];
      const bool img = MODE == ADJ_REF && a.imaging && live && x >= a.nb && x < a.nb + a.nx;
      if (MODE == ADJ_REF) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          rw[e] = 0.;
          rt[e] = rg[e] = 0.f;
          if (img && iz >= a.nb && iz < a.nb + a.nz) {
            const size_t k = (size_t)(x - a.nb) * a.nz + (iz - a.nb);
            const size_t ks = s * a.wstride + k;
            // wave[wit+1] - 2.*wave[wit] + wave[wit-1] in double, left to right
            rw[e] = __dadd_rn(__dsub_rn((double)a.wnext[ks], __dmul_rn(2., (double)a.wcur[ks])),
                              (double)a.wprev[ks]);
            rt[e] = a.m2v3[k];
            rg[e] = gs[k];
          }
        }
      }
      if (i + P < nplanes) {
        issue_cur(i + P + 8);
        issue_pv(i + P);
      }
      cp_commit();
      cp_wait<P>();
      __syncthreads();
      if (i == 0) {
#pragma unroll
        for (int k = 0; k < 8; k++) q[k] = s_cur[k * W + ci];
      }
      q[8] = s_cur[((i + 8) % NC) * W + ci];
      const float4 *pl = s_cur + ((i + 4) % NC) * W;
      if (live) {
        const float4 c = q[4];
        const float4 L = pl[ci - 1], R = pl[ci + 1];
        const float4 pv = s_prev[(i % NP) * ZW + tid];
        const float4 V4 = s_V[(i % NP) * ZW + tid];
        const float4 dv = (MODE == FWD && PAS) ? s_d[(i % NP) * ZW + tid]
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
        const float bxf = a.bx[x];
        const bool lx_ok = x >= 4 && x < a.pnx - 4;
        const long long o = o_c + (long long)lz * x;
        // receivers read the field before the update (wave_fwimodeling.c:76-79)
        int rir = -1;
        if (rec_row) {
          const int d = x - r0v;
          if (d >= 0) {
            const int ir = a.drv == 1 ? d : (d % a.drv == 0 ? d / a.drv : -1);
            if (ir >= 0 && ir < nr2) rir = r02 + ir;
          }
        }
        const bool src_here = src_z && x >= sx0 && x <= sx1;
        if (MODE == FWD && rir >= 0 && a.rec)
          a.rec[((size_t)s * a.nt + a.it) * a.nr + rir] = el(c, a.rz - iz0);
        const bool interior = x >= a.nb && x < a.nb + a.nx;
        if (MODE == FWD && a.snap && interior) {
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int iz = iz0 + e;
            if (iz >= a.nb && iz < a.nb + a.nz)
              a.snap[s * a.snap_stride + (size_t)(x - a.nb) * a.nz + (iz - a.nb)] = el(c, e);
          }
        }
        float4 term4, res4;
        float txs[4], tzs[4], qx[4], qz[4];
        {
          // the x and z sums of the 8th-order Laplacian in the reference's
          // order, cells (0, 1) and (2, 3) of the float4 per f32x2 op; the
          // z neighbours at odd distances are the float4s shifted by one cell
          const f2 k1 = pk2(a.one, a.one);
          const f2 kc[5] = {pk2(a.c0, a.c0), pk2(a.c1, a.c1), pk2(a.c2, a.c2), pk2(a.c3, a.c3),
                            pk2(a.c4, a.c4)};
          const f2 cl = lo2(c), ch = hi2(c);
          const f2 s_wx = pk2(L.w, c.x), s_yz = pk2(c.y, c.z), s_wR = pk2(c.w, R.x);
          const f2 s_Lyz = pk2(L.y, L.z), s_Ryz = pk2(R.y, R.z);
          // z partners (+d, -d) of each pair, d = 1 .. 4
          const f2 zp[2][4] = {{s_yz, ch, s_wR, lo2(R)}, {s_wR, lo2(R), s_Ryz, hi2(R)}};
          const f2 zm[2][4] = {{s_wx, hi2(L), s_Lyz, lo2(L)}, {s_yz, cl, s_wx, hi2(L)}};
          f2 tx2[2], tz2[2];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const f2 cv2 = h ? ch : cl;
            f2 tx = mul2(mul2(kc[0], cv2), k1);
#pragma unroll
            for (int d = 1; d <= 4; d++) {
              const f2 xs = h ? add2(hi2(q[4 + d]), hi2(q[4 - d])) : add2(lo2(q[4 + d]), lo2(q[4 - d]));
              tx = add2(tx, mul2(mul2(kc[d], xs), k1));
            }
            f2 tz = mul2(mul2(kc[0], cv2), k1);
#pragma unroll
            for (int d = 1; d <= 4; d++)
              tz = add2(tz, mul2(mul2(kc[d], add2(zp[h][d - 1], zm[h][d - 1])), k1));
            tx2[h] = tx;
            tz2[h] = tz;
          }
          const float4 tx4 = join2(tx2[0], tx2[1]), tz4 = join2(tz2[0], tz2[1]);
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const bool lap = lz_ok[e] && lx_ok;  // skipped cells vote with zeros
            txs[e] = lap ? el(tx4, e) : 0.f;
            tzs[e] = lap ? el(tz4, e) : 0.f;
          }
        }
        div4x2(txs, tzs, a.divx, a.divz, __activemask(), qx, qz);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int iz = iz0 + e;
          float t = (lz_ok[e] && lx_ok) ? fadd(qx[e], qz[e]) : 0.f;
          if (MODE == FWD && PAS) {
            // gradient_pas_av (wave_fwigradient.c:732-737): the interior's source
            // sample; its update covers the stencil's cells only, so none is
            // added on the 4-cell rim
            if (lz_ok[e] && lx_ok && iz >= a.nb && iz < a.nb + a.nz && x >= a.nb &&
                x < a.nb + a.nx)
              t = fadd(t, el(dv, e));
          } else if (MODE == FWD) {
            if (src_here)
              for (int k = 0; k < sg.nsrc; k++)
                if (sg.scell[k] == ((x << 16) | iz)) t = fadd(t, fmul(sg.sw[k], a.wav[a.it]));
          } else if (rir >= 0 && iz == a.rz) {
            t = fadd(t, a.res[((size_t)s * a.nt + a.it) * a.nr + rir]);
          }
          set_el(term4, e, t);
        }
        {
          // b = S(a_{k-1} as stored): z faces then x faces (apply_sponge);
          // 2 c as c + c (the same bits, and no product to fuse into the
          // subtraction)
          const f2 k1 = pk2(a.one, a.one), bx2 = pk2(bxf, bxf);
          f2 r2[2];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const f2 bz2 = pk2(bzf[2 * h], bzf[2 * h + 1]);
            const f2 cv2 = h ? hi2(c) : lo2(c);
            const f2 p = mul2(mul2(bx2, mul2(bz2, h ? hi2(pv) : lo2(pv))), k1);
            const f2 vt = mul2(mul2(h ? hi2(V4) : lo2(V4), h ? hi2(term4) : lo2(term4)), k1);
            const f2 v = add2(sub2(add2(cv2, cv2), p), vt);
            r2[h] = mul2(bx2, mul2(bz2, v));
          }
          res4 = join2(r2[0], r2[1]);
#pragma unroll
          for (int e = 0; e < 4; e++)
            if (!zin[e]) set_el(res4, e, 0.f);
        }
        *reinterpret_cast<float4 *>(nxt + o) = res4;
        if (MODE == FWD && a.tout)
          *reinterpret_cast<float4 *>(a.tout + s * a.tout_stride + o) = term4;
        if (MODE == ADJ_EXACT && a.imaging) {
          // dJ/dV accumulates phi_n * term_n (divided by V at the end)
          const float4 tf = s_t[(i % NP) * ZW + tid];
          const float4 g4 = s_g[(i % NP) * ZW + tid];  // read P planes ahead (cp.async)
          const f2 k1 = pk2(a.one, a.one);
          const float4 gacc = join2(add2(lo2(g4), mul2(mul2(lo2(c), lo2(tf)), k1)),
                                    add2(hi2(g4), mul2(mul2(hi2(c), hi2(tf)), k1)));
          *reinterpret_cast<float4 *>(gs + o) = gacc;
        }
        if (MODE == ADJ_REF && img) {
          // gradient_av (wave_fwigradient.c:221-230): the C expression in
          // double, unfused, added to the float gradient
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const int iz = iz0 + e;
            if (iz >= a.nb && iz < a.nb + a.nz) {
              const size_t k = (size_t)(x - a.nb) * a.nz + (iz - a.nb);
              const double gsum = __dmul_rn(__dmul_rn(__ddiv_rn(rw[e], (double)a.wdt2),
                                                      (double)el(c, e)),
                                            (double)rt[e]);
              gs[k] = __double2float_rn(__dadd_rn((double)rg[e], gsum));
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) q[k] = q[k + 1];
    }
    cp_wait_all();
    __syncthreads();
  }
}


// FP64 misfit and residual, one thread per (shot, it, ir):
//   REFERENCE: r = dobs - d, J += 0.5 r^2 (unweighted), adjoint source r*w
//   EXACT:     r = d - dobs, J += 0.5 w r^2, adjoint source w*r
// d, dobs, res: [shot][nt][nr]; w: [nr][nt] (residual_weighting layout) or
// null (every weight 1).
__global__ void residual_kernel(const float *d, const float *dobs, const float *w, float *res,
                                int ns, int nt, int nr, int exact, double *misfit) {
  const long long n = (long long)ns * nt * nr;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ir = int(i % nr);
    const int it = int((i / nr) % nt);
    const float wt = w ? w[(size_t)ir * nt + it] : 1.f;
    if (exact) {
      const float r = fsub(d[i], dobs[i]);
      acc += 0.5 * (double)wt * (double)r * (double)r;
      res[i] = fmul(wt, r);
    } else {
      const float r = fsub(dobs[i], d[i]);
      acc += 0.5 * (double)r * (double)r;
      res[i] = fmul(r, wt);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) misfit[1 + blockIdx.x] = v;  // block sums, added in order below
  }
}

// misfit[0] += the block sums misfit[1 .. nblocks] in block order (the same
// bits on every run, whatever order the blocks ran in)
__global__ void misfit_sum_kernel(double *misfit, int nblocks) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = misfit[0];
    for (int b = 0; b < nblocks; b++) s += misfit[1 + b];
    misfit[0] = s;
  }
}
constexpr int RESID_BLOCKS = 592;

// A Butterworth filter as np_butter_init builds it (wave_butter.c:18-62):
// for odd nn one first-order section (den[nn/2]), and nn/2 second-order
// sections sharing the middle coefficient `mid`.
constexpr int BUTTER_MAXP = 16;
struct ButterCoef {
  int nn, low;
  float den[BUTTER_MAXP / 2 + 1][2];
  float mid;
};

// One causal sweep of np_butter_apply (wave_butter.c:64-102) over the n
// samples x[0], x[st], ..., in index order or (bwd) from the last sample to
// the first -- reverse, apply, reverse in one pass.  Sections run one after
// the other over the whole trace, each product and sum in the reference's
// order.
__device__ __forceinline__ void butter_sweep(const ButterCoef &b, float *x, long long st, int n,
                                             bool bwd) {
  const float d1 = b.mid;
  if (b.nn % 2) {
    const float d0 = b.den[b.nn / 2][0], d2 = b.den[b.nn / 2][1];
    float x0 = 0.f, x1, y1 = 0.f;
    for (int k = 0; k < n; k++) {
      const long long i = (long long)(bwd ? n - 1 - k : k) * st;
      x1 = x0;
      x0 = x[i];
      const float u = b.low ? fadd(x0, x1) : fsub(x0, x1);
      y1 = fmul(fsub(u, fmul(d2, y1)), d0);
      x[i] = y1;
    }
  }
  for (int j = 0; j < b.nn / 2; j++) {
    const float d0 = b.den[j][0], d2 = b.den[j][1];
    float x0 = 0.f, x1 = 0.f, x2, y1 = 0.f, y2 = 0.f;
    for (int k = 0; k < n; k++) {
      const long long i = (long long)(bwd ? n - 1 - k : k) * st;
      x2 = x1;
      x1 = x0;
      x0 = x[i];
      const float t = fmul(2.f, x1);
      const float u = b.low ? fadd(fadd(x0, t), x2) : fadd(fsub(x0, t), x2);
      const float y0 = fmul(fsub(fsub(u, fmul(d1, y1)), fmul(d2, y2)), d0);
      y2 = y1;
      y1 = y0;
      x[i] = y0;
    }
  }
}

// pw_butter_apply: one causal sweep per trace, traces x [ntr][n]
__global__ void butter_traces_kernel(const ButterCoef b, float *x, int n, int ntr) {
  const int tr = blockIdx.x * blockDim.x + threadIdx.x;
  if (tr < ntr) butter_sweep(b, x + (size_t)tr * n, 1, n, false);
}

// The multiscale residual filter of gradient_pas_av (wave_fwigradient.c:
// 767-784) on res [shot][nt][nr]: per trace the zero-phase high-pass (apply,
// reverse, apply, reverse), then the low-pass, then the residual weight
// w [nr][nt] (or 1).
__global__ void butter_residual_kernel(const ButterCoef lo, const ButterCoef hi, int use_lo,
                                       int use_hi, float *res, int ns, int nt, int nr,
                                       const float *w) {
  const int tr = blockIdx.x * blockDim.x + threadIdx.x;
  if (tr >= ns * nr) return;
  const int s = tr / nr, ir = tr - s * nr;
  float *x = res + (size_t)s * nt * nr + ir;
  if (use_lo) {
    butter_sweep(lo, x, nr, nt, false);
    butter_sweep(lo, x, nr, nt, true);
  }
  if (use_hi) {
    butter_sweep(hi, x, nr, nt, false);
    butter_sweep(hi, x, nr, nt, true);
  }
  if (w)
    for (int it = 0; it < nt; it++) x[(size_t)it * nr] = fmul(x[(size_t)it * nr], w[(size_t)ir * nt + it]);
}

// np_butter_init on the host, its float/double mix kept
static ButterCoef butter_coef(bool low, float cutoff, int nn) {
  const double pi = 3.14159265358979323846264338328;
  ButterCoef b{};
  b.nn = nn;
  b.low = low ? 1 : 0;
  const float arg = 2. * pi * cutoff;
  const float sinw = ::sinf(arg), cosw = ::cosf(arg);
  float fact;
  if (nn % 2) {
    if (low) {
      fact = (1. + cosw) / sinw;
      b.den[nn / 2][0] = 1. / (1. + fact);
      b.den[nn / 2][1] = 1. - fact;
    } else {
      fact = sinw / (1. + cosw);
      b.den[nn / 2][0] = 1. / (fact + 1.);
      b.den[nn / 2][1] = fact - 1.;
    }
  }
  fact = low ? ::sinf(0.5 * arg) : ::cosf(0.5 * arg);
  fact *= fact;
  for (int j = 0; j < nn / 2; j++) {
    const float ss = ::sinf(pi * (2 * j + 1) / (2 * nn)) * sinw;
    b.den[j][0] = fact / (1. + ss);
    b.den[j][1] = (1. - ss) / fact;
  }
  b.mid = -2. * cosw / fact;
  return b;
}

// total[i] += slice_0[i] + slice_1[i] + ... in shot order (deterministic)
__global__ void sum_slices_kernel(const float *slices, int nb, long long n, float *total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float v = total[i];
    for (int s = 0; s < nb; s++) v = fadd(v, slices[s * n + i]);
    total[i] = v;
  }
}

// V = (v*v)*dt2 on the padded grid (pad2d edge replication, wave_fwiutil.c:123-147)
__global__ void pad_V_kernel(const float *vel, int nz, int nx, int nb, int pnz, int pnx, int lz,
                             float dt2, float *V) {
  const long long n = (long long)pnz * pnx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % pnz), ix = int(i / pnz);
    const int jz = min(max(iz - nb, 0), nz - 1), jx = min(max(ix - nb, 0), nx - 1);
    const float v = vel[(size_t)jx * nz + jz];
    V[pfoff(lz, iz, ix)] = fmul(fmul(v, v), dt2);
  }
}

// [rows][cols] -> [cols][rows]
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

// Exact gradient: dJ/dv_pad = 2 * sum(phi*term) / v_pad, folded back through
// pad2d's edge replication onto the interior (one thread per interior cell,
// summing the padded cells that copy it, in a fixed order).
// (float)(-2./temp) with temp = v*v*v in float (wave_fwigradient.c:224-226),
// once per call instead of per cell and step
__global__ void m2v3_kernel(const float *vel, size_t n, float *out) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const float v = vel[k];
    out[k] = __double2float_rn(__ddiv_rn(-2., (double)__fmul_rn(__fmul_rn(v, v), v)));
  }
}

__global__ void fold_grad_kernel(const float *gacc, const float *vel, int nz, int nx, int nb,
                                 int pnz, int pnx, int lz, float *grad) {
  const long long n = (long long)nz * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int jz = int(i % nz), jx = int(i / nz);
    const int z_lo = jz == 0 ? 0 : jz + nb, z_hi = jz == nz - 1 ? pnz - 1 : jz + nb;
    const int x_lo = jx == 0 ? 0 : jx + nb, x_hi = jx == nx - 1 ? pnx - 1 : jx + nb;
    const double v = vel[i];
    double s = 0.0;
    for (int ix = x_lo; ix <= x_hi; ix++)
      for (int iz = z_lo; iz <= z_hi; iz++) s += (double)gacc[pfoff(lz, iz, ix)];
    grad[i] = (float)(2.0 * s / v);
  }
}

// ---------------------------------------------- post-processing kernels --
// One line of np_smooth2 (wave_triangle.c:177-238) per thread, in the
// reference's float order; tmp: per-thread scratch of n + 2*rect floats.
__device__ void smooth2_line(int nb, int n, float *x, long long o, long long d, float *tmp) {
  const int np = n + 2 * nb;
  const float wt = (float)(1.0 / (nb * nb));
  float t;
  for (int i = 0; i < np; i++) tmp[i] = 0.f;
  for (int i = 0; i < n; i++) tmp[i] = fadd(tmp[i], fmul(-wt, x[o + i * d]));
  const float w2 = (float)(2. * wt);
  for (int i = 0; i < n; i++) tmp[i + nb] = fadd(tmp[i + nb], fmul(w2, x[o + i * d]));
  for (int i = 0; i < n; i++) tmp[i + 2 * nb] = fadd(tmp[i + 2 * nb], fmul(-wt, x[o + i * d]));
  t = 0.f;
  for (int i = 0; i < np; i++) { t = fadd(t, tmp[i]); tmp[i] = t; }
  t = 0.f;
  for (int i = np - 1; i >= 0; i--) { t = fadd(t, tmp[i]); tmp[i] = t; }
  for (int i = 0; i < n; i++) x[o + i * d] = tmp[i + nb];
  for (int m = 0; m < nb; m++) {  // right extension: mirrored, then direct, ...
    const int b = m / n, i = m % n;
    const int dst = (b % 2 == 0) ? (n - 1 - i) : i;
    x[o + dst * d] = fadd(x[o + dst * d], tmp[nb + n + m]);
  }
  for (int m = 0; m < nb; m++) {  // left extension: direct, then mirrored, ...
    const int b = m / n, i = m % n;
    const int dst = (b % 2 == 0) ? i : (n - 1 - i);
    x[o + dst * d] = fadd(x[o + dst * d], tmp[nb - 1 - m]);
  }
}

__global__ void smooth_lines_kernel(float *x, int nlines, int n, long long line_step,
                                    long long elem_step, int rect, float *scratch) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlines) return;
  smooth2_line(rect, n, x, (long long)l * line_step, elem_step, scratch + (size_t)l * (n + 2 * rect));
}

__global__ void absmax_kernel(const float *x, long long n, unsigned int *out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(x[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void vel_check_kernel(const float *x, long long n, unsigned int *out) {
  float m = 0.f;
  unsigned bad = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    if (!(v > 0.f) || !isfinite(v)) bad = 1;
    else m = fmaxf(m, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, __float_as_uint(m));
    if (bad) atomicOr(out + 1, 1u);
  }
}

// waterz rows to zero and the scale factor (gradient_smooth2 tail,
// wave_fwiutil.c:323-334); scaling <= 0 means "derive 0.1/max|g| here"
__global__ void finish_kernel(float *g, int nz, int nx, int waterz, const unsigned int *mx,
                              float *scaling) {
  float sc = *scaling;
  if (sc <= 0.f) sc = (float)(0.1 / (double)__uint_as_float(*mx));
  const long long n = (long long)nz * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % nz);
    float v = g[i];
    if (waterz >= 0 ? iz < waterz : iz >= nz + waterz) v = 0.f;
    g[i] = fmul(v, sc);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && *scaling <= 0.f) *scaling = sc;
}

// ------------------------------------------------------------------ host --

// Restated source map: a unit spike at (sx, sz) smoothed with rect 2 along
// z then x (source_map, wave_fwiutil.c:149-177), on the host in float.
static void smooth_line_host(int nb, int n, float *x, long long o, long long d, std::vector<float> &tmp) {
  const int np = n + 2 * nb;
  tmp.assign(np, 0.f);
  const float wt = (float)(1.0 / (nb * nb));
  for (int i = 0; i < n; i++) tmp[i] += (-wt) * x[o + i * d];
  for (int i = 0; i < n; i++) tmp[i + nb] += ((float)(2. * wt)) * x[o + i * d];
  for (int i = 0; i < n; i++) tmp[i + 2 * nb] += (-wt) * x[o + i * d];
  float t = 0.f;
  for (int i = 0; i < np; i++) { t += tmp[i]; tmp[i] = t; }
  t = 0.f;
  for (int i = np - 1; i >= 0; i--) { t += tmp[i]; tmp[i] = t; }
  for (int i = 0; i < n; i++) x[o + i * d] = tmp[i + nb];
  for (int m = 0; m < nb; m++) {
    const int b = m / n, i = m % n;
    const int dst = (b % 2 == 0) ? (n - 1 - i) : i;
    x[o + dst * d] += tmp[nb + n + m];
  }
  for (int m = 0; m < nb; m++) {
    const int b = m / n, i = m % n;
    const int dst = (b % 2 == 0) ? i : (n - 1 - i);
    x[o + dst * d] += tmp[nb - 1 - m];
  }
}

static int source_map(int sx, int sz, int pnz, int pnx, ShotGeo &sg) {
  // the map is separable and local: smooth a small window around the spike
  const int r = 6;
  const int x_lo = std::max(0, sx - r), x_hi = std::min(pnx - 1, sx + r);
  const int z_lo = std::max(0, sz - r), z_hi = std::min(pnz - 1, sz + r);
  // the fold reflections need the full line when the spike is near an edge
  const bool full = x_lo == 0 || z_lo == 0 || x_hi == pnx - 1 || z_hi == pnz - 1;
  std::vector<float> m, tmp;
  int zs, xs, nzw, nxw;
  if (full) { zs = 0; xs = 0; nzw = pnz; nxw = pnx; }
  else { zs = z_lo; xs = x_lo; nzw = z_hi - z_lo + 1; nxw = x_hi - x_lo + 1; }
  // smoothing a window equals smoothing the full line when the window
  // holds the whole support (rect 2 spreads one cell each way)
  m.assign((size_t)nzw * nxw, 0.f);
  m[(size_t)(sx - xs) * nzw + (sz - zs)] = 1.f;
  for (int j = 0; j < nxw; j++) smooth_line_host(2, nzw, m.data(), (long long)j * nzw, 1, tmp);
  for (int j = 0; j < nzw; j++) smooth_line_host(2, nxw, m.data(), j, nzw, tmp);
  sg.nsrc = 0;
  sg.sx0 = sg.sz0 = 1 << 30;
  sg.sx1 = sg.sz1 = -1;
  for (int ix = 0; ix < nxw; ix++)
    for (int iz = 0; iz < nzw; iz++) {
      const float w = m[(size_t)ix * nzw + iz];
      if (w != 0.f) {
        PW_CHECK(sg.nsrc < MAXSRCW, PW_ERR_SHAPE, "source map has too many cells");
        const int gz = iz + zs, gx = ix + xs;
        PW_CHECK(gz >= 4 && gz < pnz - 4 && gx >= 4 && gx < pnx - 4, PW_ERR_SHAPE,
                 "source map reaches the zero border of the padded grid");
        sg.scell[sg.nsrc] = (gx << 16) | gz;
        sg.sw[sg.nsrc] = w;
        sg.nsrc++;
        sg.sx0 = std::min(sg.sx0, gx);
        sg.sx1 = std::max(sg.sx1, gx);
        sg.sz0 = std::min(sg.sz0, gz);
        sg.sz1 = std::max(sg.sz1, gz);
      }
    }
  return PW_OK;
}

// Exhaustive check of DivC against __fdiv_rn over the 2^23 significands of
// x in [scale, 2*scale) (a binade where every intermediate value is normal).
__device__ unsigned int fastdiv_bad;
__global__ void fastdiv_check_kernel(float d, float zh, float zl, float scale) {
  const unsigned int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (1u << 23)) return;
  const float x = __fmul_rn(scale, __uint_as_float(0x3f800000u | m));  // exact (power of 2)
  const float q = __fmaf_rn(x, zh, __fmul_rn(x, zl));
  if (__float_as_uint(q) != __float_as_uint(__fdiv_rn(x, d))) atomicAdd(&fastdiv_bad, 1u);
}

// div_small against __fdiv_rn for every float with bits in [1, umin), both signs
__global__ void smalldiv_check_kernel(DivC c) {
  const unsigned int stride = gridDim.x * blockDim.x;
  unsigned int bad = 0;
  for (unsigned int u = 1 + blockIdx.x * blockDim.x + threadIdx.x; u < c.umin; u += stride) {
    const float x = __uint_as_float(u), y = -x;
    bad += __float_as_uint(div_small(x, c)) != __float_as_uint(__fdiv_rn(x, c.d));
    bad += __float_as_uint(div_small(y, c)) != __float_as_uint(__fdiv_rn(y, c.d));
  }
  if (bad) atomicAdd(&fastdiv_bad, bad);
}

// DivC for d (cached per process: the result depends on d only).
static int prepare_div(float d, DivC &c) {
  static std::mutex mu;
  static std::map<unsigned int, DivC> cache;
  unsigned int key;
  memcpy(&key, &d, 4);
  std::lock_guard<std::mutex> lock(mu);
  auto hit = cache.find(key);
  if (hit != cache.end()) {
    c = hit->second;
    return PW_OK;
  }
  c.d = d;
  c.ok = 0;
  c.zh = c.zl = 0.f;
  c.xmin = 1.f;
  c.xmax = 0.f;
  c.umin = c.uspan = c.umax = 0;
  if (d > 0.f && std::isfinite(d)) {
    // zh: the float nearest 1/d (float x float products are exact in double,
    // and 1 - zh*d is exact by Sterbenz's lemma)
    const float z0 = (float)(1.0 / (double)d);
    float zh = z0;
    double err = std::fabs(1.0 - (double)z0 * d);
    for (float cand : {std::nextafter(z0, 0.f), std::nextafter(z0, INFINITY)}) {
      const double e = std::fabs(1.0 - (double)cand * d);
      unsigned int cb;
      memcpy(&cb, &cand, 4);
      if (e < err || (e == err && (cb & 1u) == 0)) {
        zh = cand;
        err = e;
      }
    }
    const float zl = (float)((1.0 - (double)zh * d) / (double)d);
    // keep x*zh, x*zl and x/d normal and finite with a factor-4 margin
    const double fmin = (double)FLT_MIN, fmax = (double)FLT_MAX;
    double lo = std::max(fmin / zh, fmin * d);
    if (zl != 0.f) lo = std::max(lo, fmin / std::fabs((double)zl));
    lo *= 4;
    const double hi = std::min({fmax / 4 / zh, fmax / 4 * d, fmax});  // finite numerators only
    if (lo * 4 < hi) {
      c.zh = zh;
      c.zl = zl;
      c.xmin = (float)lo;
      c.xmax = (float)hi;
      memcpy(&c.umin, &c.xmin, 4);
      memcpy(&c.umax, &c.xmax, 4);
      c.uspan = c.umax - c.umin;
      c.sup = std::ldexp(1.f, DIV_SMALL_K);
      c.sdn = std::ldexp(1.f, -DIV_SMALL_K);
      c.sgrid = std::ldexp(1.f, 149 - DIV_SMALL_K);
      // x in (0, xmin) scales into [2^(K-149), xmin * 2^K], inside [xmin, xmax]
      const bool small_ok = lo <= std::ldexp(1.0, DIV_SMALL_K - 149) &&
                            lo * std::ldexp(1.0, DIV_SMALL_K) <= hi;
      const double scale = std::ldexp(1.0, (int)std::ceil(std::log2(lo)));
      unsigned int bad = 0;
      PW_CUDA(cudaMemcpyToSymbol(fastdiv_bad, &bad, sizeof bad));
      fastdiv_check_kernel<<<(1u << 23) / 256, 256>>>(d, zh, zl, (float)scale);
      PW_CUDA(cudaGetLastError());
      if (small_ok) {
        smalldiv_check_kernel<<<4 * 148, 256>>>(c);
        PW_CUDA(cudaGetLastError());
      }
      PW_CUDA(cudaMemcpyFromSymbol(&bad, fastdiv_bad, sizeof bad));
      c.ok = small_ok && bad == 0;
    }
  }
  if (getenv("PW_PFWI_VERBOSE"))
    fprintf(stderr, "pfwi: division by %.9g: zh %.9g zl %.9g range [%.3g, %.3g] fast %d\n", d,
            c.zh, c.zl, c.xmin, c.xmax, c.ok);
  cache[key] = c;
  return PW_OK;
}

struct Setup {
  pw_fwi_args a;
  DivC divx, divz;
  int pnz, pnx, lz;
  long long fstride;  // floats per field (incl. halo)
  int nr, rz, drv, sz;
  std::vector<ShotGeo> geo;
  std::vector<float> bz, bx;
  int zw, ztiles, nsm;
  size_t smem;
};

// passive: distributed sources (pfwi mode 4) -- no point source per shot
static int setup(const pw_fwi_args *a, Setup &S, bool passive = false) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  S.a = *a;
  PW_CHECK(a->nz >= 1 && a->nx >= 1 && a->nt >= 1 && a->ns >= 1 && a->nb >= 1, PW_ERR_SHAPE,
           "sizes must be positive (nz=%d nx=%d nt=%d ns=%d nb=%d)", a->nz, a->nx, a->nt, a->ns,
           a->nb);
  PW_CHECK(a->dx > 0 && a->dz > 0 && a->dt > 0, PW_ERR_VALUE, "spacings must be positive");
  const int nb = a->nb;
  S.pnz = a->nz + 2 * nb;
  S.pnx = a->nx + 2 * nb;
  PW_CHECK(S.pnx < 65536 && S.pnz < 65536, PW_ERR_SHAPE, "grid too large");
  S.lz = (int)round_up(HZ + round_up(S.pnz, 4) + 4, 32);
  PW_TRY(prepare_div(a->dx * a->dx, S.divx));
  PW_TRY(prepare_div(a->dz * a->dz, S.divz));
  S.fstride = (long long)S.lz * (S.pnx + 2 * HX) + 64;
  // preparation (wave_fwiutil.c:31-71) with pfwi.c's fixed acquisition
  std::vector<float> bc(nb);
  for (int i = 0; i < nb; i++) {
    float tmp = a->coef * (nb - i);
    bc[i] = expf(-tmp * tmp);
  }
  auto axis = [&](int n, std::vector<float> &f) {
    f.assign(n, 1.f);
    for (int i = 0; i < nb; i++) f[i] = bc[i];
    for (int i = n - nb; i < n; i++) f[i] = bc[n - i - 1];
  };
  axis(S.pnz, S.bz);
  axis(S.pnx, S.bx);
  const float dx = a->dx;
  const int ds_v = (int)(a->ds / dx + 0.5);
  const int s0_v = (int)(a->os / dx + 0.5 + nb);
  S.sz = a->sz + nb;
  S.rz = a->rz + nb;
  S.nr = a->nx;
  const float dr = dx, r0 = a->ox, x0 = a->ox;
  S.drv = (int)(dr / dx + 0.5);
  PW_CHECK(S.drv >= 1, PW_ERR_SHAPE, "receiver interval below one cell");
  const float xend = x0 + (a->nx - 1) * dx;
  S.geo.assign(a->ns, ShotGeo{});
  for (int is = 0; is < a->ns; is++) {
    ShotGeo &g = S.geo[is];
    if (a->acqui_type == 1) {
      g.r0v = (int)((r0 - x0) / dx + 0.5 + nb);
      g.r02 = 0;
      g.nr2 = S.nr;
    } else {
      const float sx = a->os + a->ds * is;
      const float rbegin = (sx + r0 < x0) ? x0 : sx + r0;
      float rend = sx + r0 + (S.nr - 1) * dr;
      rend = (rend < xend) ? rend : xend;
      g.r0v = (int)(rbegin / dx + 0.5 + nb);
      g.r02 = (int)((rbegin - sx - r0) / dx + 0.5);
      g.nr2 = (int)((rend - rbegin) / dx + 1.5);
    }
    PW_CHECK(g.r02 >= 0 && g.r02 + g.nr2 <= S.nr && g.r0v >= 0 &&
                 g.r0v + (g.nr2 - 1) * S.drv < S.pnx,
             PW_ERR_SHAPE, "shot %d: receivers outside the grid", is);
    if (passive) {  // an empty source map
      g.nsrc = 0;
      g.sx0 = g.sz0 = 1;
      g.sx1 = g.sz1 = 0;
      continue;
    }
    const int sx = s0_v + is * ds_v;
    PW_CHECK(sx >= 0 && sx < S.pnx && S.sz >= 0 && S.sz < S.pnz, PW_ERR_SHAPE,
             "shot %d: source (x=%d, z=%d) outside the padded grid", is, sx, S.sz);
    PW_TRY(source_map(sx, S.sz, S.pnz, S.pnx, g));
  }
  PW_CHECK(S.rz >= 4 && S.rz < S.pnz - 4, PW_ERR_SHAPE, "receiver depth in the zero border");
  // tile: one z segment of ZW float4 (whole column when it fits)
  const int nz4 = ceil_div(S.pnz, 4);
  S.zw = nz4 <= 64 ? 64 : 128;
  const int ztiles = ceil_div(nz4, S.zw);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  S.ztiles = ztiles;
  S.nsm = nsm;
  if (getenv("PW_PFWI_VERBOSE"))
    fprintf(stderr, "pfwi plan: padded %d x %d, ZW=%d ztiles=%d\n", S.pnz, S.pnx, S.zw, S.ztiles);
  return PW_OK;
}

// prefetch depth (planes): one plane ahead is enough once the x chunks are
// short, and the smaller ring lets more CTAs share an SM (32 shots of 420 x
// 720 at nt 500: forward 36.3 -> 33.0 ms, exact gradient 79.5 -> 70.7 ms
// against 3 planes)
constexpr int PFP = 1;

static size_t smem_for(int zw, int mode) {
  return sizeof(float4) * ((size_t)(PFP + 10) * (zw + 2) + (size_t)(mode == ADJ_EXACT ? 4 : 2) *
                                                               (PFP + 2) * zw);
}

template <int ZW, int MODE, bool PAS = false>
static int launch_one(const Setup &S, const PfArgs &p, cudaStream_t st) {
  // the forward step with passive sources adds a ring of source planes
  const size_t smem = smem_for(ZW, MODE) + (PAS ? (size_t)(PFP + 2) * ZW * sizeof(float4) : 0);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(pf_step_kernel<ZW, PFP, MODE, PAS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  // x planes per CTA: long enough to amortise the 8-plane prologue, short
  // enough that shots x chunks x z tiles give every SM 12 CTAs (about three
  // waves of the 4 that fit).  Small batches go down to one plane per CTA:
  // a step is then a few dependent plane updates instead of a long chain
  // (the passive demos' grid, 3 shots: 175 ms per gradient at 16 planes,
  // 46 ms at 1), the re-read halo planes staying in L2; 32 shots of 420 x
  // 720 run 8 planes (2.94 gradients/s, 2.69 at 16)
  int xch = 128;
  while (xch > 1 && (long long)p.nshots * S.ztiles * ceil_div(S.pnx, xch) < 12LL * S.nsm) xch /= 2;
  const dim3 grid(p.nshots, ceil_div(S.pnx, xch), S.ztiles);
  pf_step_kernel<ZW, PFP, MODE, PAS><<<grid, ZW, smem, st>>>(p, xch);
  PW_CUDA(cudaGetLastError());
  return PW_OK;
}

static int launch(const Setup &S, const PfArgs &p, int mode, cudaStream_t st) {
  if (mode == FWD && p.dsrc)
    return S.zw == 64 ? launch_one<64, FWD, true>(S, p, st) : launch_one<128, FWD, true>(S, p, st);
  if (S.zw == 64) {
    if (mode == FWD) return launch_one<64, FWD>(S, p, st);
    if (mode == ADJ_REF) return launch_one<64, ADJ_REF>(S, p, st);
    return launch_one<64, ADJ_EXACT>(S, p, st);
  }
  if (mode == FWD) return launch_one<128, FWD>(S, p, st);
  if (mode == ADJ_REF) return launch_one<128, ADJ_REF>(S, p, st);
  return launch_one<128, ADJ_EXACT>(S, p, st);
}

static void base_args(const Setup &S, PfArgs &p) {
  memset(&p, 0, sizeof p);
  p.pnz = S.pnz;
  p.pnx = S.pnx;
  p.lz = S.lz;
  p.nb = S.a.nb;
  p.nz = S.a.nz;
  p.nx = S.a.nx;
  const float c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
  p.c0 = c0; p.c1 = c1; p.c2 = c2; p.c3 = c3; p.c4 = c4;
  p.dx2 = S.a.dx * S.a.dx;
  p.dz2 = S.a.dz * S.a.dz;
  p.one = 1.f;
  p.divx = S.divx;
  p.divz = S.divz;
  p.nt = S.a.nt;
  p.rz = S.rz;
  p.drv = S.drv;
  p.nr = S.nr;
  p.fstride = S.fstride;
}

}  // namespace pf
}  // namespace pw

using namespace pw;
using namespace pw::pf;

extern "C" int pw_fwi_args_from_pararray(const float *p, int n, pw_fwi_args *o) {
  PW_CHECK(p && o && n >= 20, PW_ERR_VALUE, "pararray needs 20 values");
  memset(o, 0, sizeof *o);
  o->nz = (int)p[0]; o->nx = (int)p[1]; o->dz = p[2]; o->dx = p[3]; o->oz = p[4]; o->ox = p[5];
  o->nt = (int)p[6]; o->dt = p[7]; o->ot = p[8]; o->ns = (int)p[10]; o->ds = p[11];
  o->os = p[12]; o->nb = (int)p[14]; o->coef = p[15]; o->f0 = p[16];
  o->acqui_type = (int)p[17]; o->interval = (int)p[18]; o->niter = (int)p[19];
  o->sz = 5; o->rz = 1;  // pfwi.c:796-800
  return PW_OK;
}

// --------------------------------------------------------------- drivers --
namespace pw {
namespace pf {

// residual_weighting with oreo=false as fwic sets it up (wave_fwiutil.c:225-296,
// pfwi.c:849-855): 1 inside, 10-sample sine tapers on both axes.  [nr][nt].
// residual_weighting (wave_fwiutil.c:225-296), both branches; w [nr][nt].
// Taper samples that would fall outside the array (a window closer than 10
// samples to its edge, where the reference writes out of bounds) are skipped.
static void weights_window(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2, bool oreo,
                           float *w) {
  float sn[10];
  for (int i = 0; i < 10; i++) sn[i] = sinf(0.5 * M_PI * (i + 1) / 11.);
  float sink = 0.f;
  auto W = [&](int ir, int it) -> float & {
    return (ir >= 0 && ir < nr && it >= 0 && it < nt) ? w[(size_t)ir * nt + it] : sink;
  };
  if (oreo) {
    for (size_t i = 0; i < (size_t)nr * nt; i++) w[i] = 1.f;
    for (int ir = woffn1; ir <= woffn2; ir++)
      for (int it = wtn1; it <= wtn2; it++) W(ir, it) = 0.f;
    for (int ir = 0; ir < 10; ir++)
      for (int it = wtn1; it <= wtn2; it++) {
        if (woffn1 - ir > 0) W(woffn1 - ir, it) *= sn[ir];
        if (woffn2 + ir < nr) W(woffn2 + ir, it) *= sn[ir];
      }
    for (int it = 0; it < 10; it++) {
      for (int ir = 0; ir < woffn1; ir++) {
        W(ir, wtn1 + it) *= sn[it];
        W(ir, wtn2 - it) *= sn[it];
      }
      for (int ir = woffn2 + 1; ir < nr; ir++) {
        W(ir, wtn1 + it) *= sn[it];
        W(ir, wtn2 - it) *= sn[it];
      }
    }
    return;
  }
  for (size_t i = 0; i < (size_t)nr * nt; i++) w[i] = 0.f;
  for (int ir = woffn1; ir <= woffn2; ir++)
    for (int it = wtn1; it <= wtn2; it++) W(ir, it) = 1.f;
  for (int ir = 0; ir < 10; ir++)
    for (int it = wtn1; it <= wtn2; it++) {
      W(woffn1 + ir, it) *= sn[ir];
      W(woffn2 - ir, it) *= sn[ir];
    }
  for (int it = 0; it < 10; it++)
    for (int ir = woffn1; ir <= woffn2; ir++) {
      W(ir, wtn1 + it) *= sn[it];
      W(ir, wtn2 - it) *= sn[it];
    }
}

static void residual_weights(const pw_fwi_args &a, int nr, std::vector<float> &w) {
  const int nt = a.nt;
  const float t0 = a.ot, dt = a.dt, r0 = a.ox, dr = a.dx;
  const float wt1 = t0, wt2 = t0 + (nt - 1) * dt;
  const float woff1 = r0, woff2 = r0 + (nr - 1) * dr;
  const int wtn1 = (int)((wt1 - t0) / dt + 0.5), wtn2 = (int)((wt2 - t0) / dt + 0.5);
  const int woffn1 = (int)((woff1 - r0) / dr + 0.5), woffn2 = (int)((woff2 - r0) / dr + 0.5);
  w.assign((size_t)nr * nt, 0.f);
  weights_window(nt, nr, wtn1, wtn2, woffn1, woffn2, false, w.data());
}

struct Fields {
  float *V = nullptr;
  float *A = nullptr, *B = nullptr;  // [nshots][fstride] each
  ShotGeo *geo = nullptr;
  float *bz = nullptr, *bx = nullptr, *wav = nullptr;
};

// Common device state of a call: V, the two wavefield sets, geometry.
static int bind_common(const Setup &S, int nsb, Carve &cv, size_t &o_V, size_t &o_A, size_t &o_B,
                       size_t &o_geo, size_t &o_bz, size_t &o_bx, size_t &o_wav) {
  o_V = cv.add(S.fstride * 4);
  o_A = cv.add((size_t)nsb * S.fstride * 4);
  o_B = cv.add((size_t)nsb * S.fstride * 4);
  o_geo = cv.add(sizeof(ShotGeo) * S.a.ns);
  o_bz = cv.add(S.bz.size() * 4);
  o_bx = cv.add(S.bx.size() * 4);
  o_wav = cv.add((size_t)S.a.nt * 4);
  return PW_OK;
}

static int upload_common(const Setup &S, char *base, size_t o_geo, size_t o_bz, size_t o_bx,
                         size_t o_wav, const float *wav, bool host, cudaStream_t st) {
  PW_CUDA(cudaMemcpyAsync(base + o_geo, S.geo.data(), sizeof(ShotGeo) * S.a.ns,
                          cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bz, S.bz.data(), S.bz.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bx, S.bx.data(), S.bx.size() * 4, cudaMemcpyHostToDevice, st));
  if (wav) PW_TRY(to_device(base + o_wav, wav, (size_t)S.a.nt * 4, host, st));
  return PW_OK;
}

static int check_vel_cfl(const Setup &S, const float *vel_dev, size_t n, cudaStream_t st,
                         unsigned *scratch) {
  // largest velocity (CFL) and a flag for non-finite / non-positive values
  PW_CUDA(cudaMemsetAsync(scratch, 0, 8, st));
  vel_check_kernel<<<296, 256, 0, st>>>(vel_dev, (long long)n, scratch);
  PW_CUDA(cudaGetLastError());
  unsigned hv[2] = {0, 0};
  PW_CUDA(cudaMemcpyAsync(hv, scratch, 8, cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  float vmax;
  memcpy(&vmax, &hv[0], 4);
  PW_CHECK(hv[1] == 0 && vmax > 0.f, PW_ERR_VALUE, "velocity has non-finite or non-positive values");
  if (S.a.flags & PW_NO_CFL_CHECK) return PW_OK;
  // 8th-order leapfrog in 2-D: v dt / h <= 0.555 (measured limit)
  const float hmin = std::min(S.a.dx, S.a.dz);
  const float cfl = vmax * S.a.dt / hmin;
  PW_CHECK(cfl <= 0.555f, PW_ERR_CFL, "unstable: vmax*dt/h = %g exceeds 0.555", cfl);
  return PW_OK;
}

}  // namespace pf
}  // namespace pw

extern "C" int pw_pfwi_forward(const pw_fwi_args *a, const float *vel, const float *wav,
                               float *data, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  Setup S;
  PW_TRY(setup(a, S));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr;
  const int nsb = std::min(ns, MAXS);
  const size_t nvel = (size_t)a->nz * a->nx;
  Carve cv;
  size_t o_V, o_A, o_B, o_geo, o_bz, o_bx, o_wav;
  bind_common(S, nsb, cv, o_V, o_A, o_B, o_geo, o_bz, o_bx, o_wav);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_rec = cv.add((size_t)ns * nt * nr * 4);
  const size_t o_out = cv.add(host ? (size_t)ns * nt * nr * 4 : 0);
  const size_t o_mx = cv.add(16);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  const float *d_vel = vel;
  if (host) {
    PW_TRY(to_device(base + o_vel, vel, nvel * 4, true, st));
    d_vel = at<float>(base, o_vel);
  }
  PW_TRY(check_vel_cfl(S, d_vel, nvel, st, at<unsigned>(base, o_mx)));
  PW_TRY(upload_common(S, base, o_geo, o_bz, o_bx, o_wav, wav, host, st));
  float *V = at<float>(base, o_V);
  pad_V_kernel<<<1184, 256, 0, st>>>(d_vel, a->nz, a->nx, a->nb, S.pnz, S.pnx, S.lz, a->dt * a->dt, V);
  PW_CUDA(cudaGetLastError());
  float *rec = at<float>(base, o_rec);
  PfArgs p;
  base_args(S, p);
  p.V = V;
  p.bz = at<float>(base, o_bz);
  p.bx = at<float>(base, o_bx);
  p.wav = at<float>(base, o_wav);
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  for (int s0 = 0; s0 < ns; s0 += nsb) {
    const int nb_ = std::min(nsb, ns - s0);
    float *A[MAXS], *B[MAXS];
    for (int s = 0; s < nb_; s++) {
      A[s] = at<float>(base, o_A) + (size_t)s * S.fstride;
      B[s] = at<float>(base, o_B) + (size_t)s * S.fstride;
    }
    PW_CUDA(cudaMemsetAsync(base + o_A, 0, (size_t)nsb * S.fstride * 4, st));
    PW_CUDA(cudaMemsetAsync(base + o_B, 0, (size_t)nsb * S.fstride * 4, st));
    p.nshots = nb_;
    p.geo = at<ShotGeo>(base, o_geo) + s0;
    p.rec = rec + (size_t)s0 * nt * nr;
    for (int it = 0; it < nt; it++) {
      p.it = it;
      for (int s = 0; s < nb_; s++) {
        p.cur[s] = A[s];
        p.nxt[s] = B[s];
      }
      PW_TRY(launch(S, p, FWD, st));
      launches++;
      for (int s = 0; s < nb_; s++) std::swap(A[s], B[s]);
    }
  }
  timer.stop();
  // [shot][nt][nr] -> [shot][nr][nt]
  float *dst = host ? at<float>(base, o_out) : data;
  for (int s = 0; s < ns; s++) {
    dim3 tb(32, 8), tg(ceil_div(nr, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb, 0, st>>>(rec + (size_t)s * nt * nr, dst + (size_t)s * nt * nr, nt, nr);
  }
  PW_CUDA(cudaGetLastError());
  if (host) PW_TRY(to_host(data, dst, (size_t)ns * nt * nr * 4, true, st));
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(launches, launches + 3 + ns);
  return PW_OK;
}

// Checkpoint plan of the exact gradient under an HBM budget.  The working
// set of a batch of nsb shots is, in field-sized buffers per shot: the two
// wavefield pairs, the gradient slice and traces (about 5), the checkpoints
// (two fields every k steps) and the segment buffer of k forward terms.  The
// forward pass keeps the terms of the last segment, so the backward pass
// recomputes the (nck - 1) k steps before it: the recompute factor (forward
// steps run / nt) is 1 + (nck - 1) k / nt.  Once the shots of a batch fill
// the GPU a step costs in proportion to its shots, so the planner picks,
// over batch sizes nsb = ns, ns/2, ..., 1 (every batch sums its shots' slices
// into the gradient in shot order, so the result does not depend on nsb),
// the largest k that fits the budget, and among those the plan with the
// least recompute, then the largest batch.  k = nt stores every term and
// recomputes nothing; a fixed ckpt_k > 0 keeps k and only shrinks the batch
// if needed.
struct ExactPlan {
  int k = 0, nsb = 0;
  double recompute = 1.0;
  size_t bytes = 0;
};

static ExactPlan plan_exact(const Setup &S, int ckpt_k, size_t held) {
  const int nt = S.a.nt;
  size_t freeb = 0, totb = 0;
  if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) {
    cudaGetLastError();
    freeb = totb = (size_t)32 << 30;
  }
  // budget: the caller's, or a quarter of the device; never more than 80% of
  // what is free plus the workspace this call reuses
  double budget = S.a.hbm_budget > 0 ? (double)S.a.hbm_budget : 0.25 * (double)totb;
  budget = std::min(budget, 0.8 * (double)(freeb + held));
  const double fb = (double)S.fstride * 4;
  auto need = [&](int kk, int nb) {
    const int nck = (nt + kk - 1) / kk;
    return fb * nb * (5.0 + 2.0 * nck + kk) + fb * 2;
  };
  auto recompute = [&](int kk) {
    const int nck = (nt + kk - 1) / kk;
    return 1.0 + (double)(nck - 1) * kk / nt;
  };
  const int kmin = std::min(nt, std::max(1, (int)std::lround(std::sqrt(2.0 * nt))));
  const int nsb_max = std::min(S.a.ns, MAXS);
  ExactPlan best;
  for (int nb = nsb_max; nb >= 1; nb = (nb + 1) / 2) {
    int k;
    if (ckpt_k > 0) {
      k = std::min(ckpt_k, nt);
      if (need(k, nb) > budget && nb > 1) continue;
    } else if (need(nt, nb) <= budget) {
      k = nt;
    } else if (need(kmin, nb) <= budget) {
      // need() rises with k above kmin: the largest k in [kmin, nt) that fits
      int lo = kmin, hi = nt;
      while (hi - lo > 1) {
        const int mid = lo + (hi - lo) / 2;
        if (need(mid, nb) <= budget) lo = mid;
        else hi = mid;
      }
      k = lo;
    } else {
      k = 0;
    }
    if (k > 0) {
      const double rc = recompute(k);
      if (best.k == 0 || rc < best.recompute - 1e-12) {
        best.k = k;
        best.nsb = nb;
        best.recompute = rc;
        best.bytes = (size_t)need(k, nb);
      }
      if (ckpt_k > 0 || rc == 1.0) break;  // nothing better below
    }
    if (nb == 1) break;
  }
  if (best.k == 0) {
    // nothing fits the budget: the smallest working set (one shot, k =
    // sqrt(2 nt)); the allocation reports if even that fails
    best.nsb = 1;
    best.k = ckpt_k > 0 ? std::min(ckpt_k, nt) : kmin;
    best.recompute = recompute(best.k);
    best.bytes = (size_t)need(best.k, best.nsb);
  }
  return best;
}

// Per-thread record of the last exact gradient's checkpoint plan.
struct PlanRecord {
  int k = 0, nsb = 0;
  long long bytes = 0;
  double recompute = 0.0;
};
static PlanRecord &plan_record() {
  static thread_local PlanRecord r;
  return r;
}

namespace pw {
namespace pf {
// The gradient of pw_pfwi_gradient (wav: point sources) and of
// pw_pfwi_gradient_passive (dsrc: a source field per shot, [ns][nt][nx][nz]).
static int gradient_impl(const pw_fwi_args *a, int mode, const float *vel, const float *wav,
                         const float *dsrc, const float *dobs, const float *weight, float *grad,
                         double *misfit, int ckpt_k, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  PW_CHECK(mode == PW_GRAD_REFERENCE || mode == PW_GRAD_EXACT, PW_ERR_VALUE, "bad gradient mode");
  PW_CHECK(vel && dobs && grad && (wav || dsrc), PW_ERR_VALUE, "null array");
  Setup S;
  PW_TRY(setup(a, S, dsrc != nullptr));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const bool per_shot = (a->flags & PW_PER_SHOT) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr, nz = a->nz, nx = a->nx;
  const size_t nvel = (size_t)nz * nx;
  const bool exact = mode == PW_GRAD_EXACT;
  const int interval = std::max(1, a->interval);
  const int wnt = (nt - 1) / interval + 1;
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  int k = 0, nsb = per_shot ? 1 : std::min(ns, MAXS);
  if (exact) {
    const ExactPlan ep = plan_exact(S, ckpt_k, ws.capacity());
    k = ep.k;
    nsb = per_shot ? 1 : ep.nsb;
    plan_record().k = k;
    plan_record().nsb = nsb;
    plan_record().recompute = ep.recompute;
  }
  const int nck = exact ? (nt + k - 1) / k : 0;
  std::vector<float> wts;
  if (weight == nullptr) residual_weights(*a, nr, wts);
  // multiscale residual filter (gradient_pas_init, wave_fwigradient.c:657-658:
  // soupar's cutoffs times dt, compared in double)
  const float flo_dt = a->flo * a->dt, fhi_dt = a->fhi * a->dt;
  const bool use_lo = flo_dt > 0.0001, use_hi = a->fhi > 0.f && fhi_dt < 0.5 - 0.0001;
  PW_CHECK(!(exact && (use_lo || use_hi)), PW_ERR_VALUE,
           "the multiscale residual filter applies to the reference-mode gradient only");
  const ButterCoef blo = use_lo ? butter_coef(false, flo_dt, 3) : ButterCoef{};
  const ButterCoef bhi = use_hi ? butter_coef(true, fhi_dt, 3) : ButterCoef{};

  Carve cv;
  size_t o_V, o_A, o_B, o_geo, o_bz, o_bx, o_wav;
  bind_common(S, nsb, cv, o_V, o_A, o_B, o_geo, o_bz, o_bx, o_wav);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_w = cv.add((size_t)nr * nt * 4);
  const size_t o_dobs = cv.add((size_t)ns * nt * nr * 4);    // [shot][nt][nr]
  const size_t o_dobs_in = cv.add(host ? (size_t)ns * nt * nr * 4 : 0);
  const size_t o_d = cv.add((size_t)nsb * nt * nr * 4);      // recorded [shot][nt][nr]
  const size_t o_res = cv.add((size_t)nsb * nt * nr * 4);
  const size_t o_snap = cv.add(exact ? 0 : (size_t)nsb * wnt * nvel * 4);
  const size_t o_ck = cv.add(exact ? (size_t)nsb * nck * 2 * S.fstride * 4 : 0);
  const size_t o_tb = cv.add(exact ? (size_t)nsb * k * S.fstride * 4 : 0);
  const size_t o_ga = cv.add(exact ? (size_t)S.fstride * 4 : 0);
  // shots of one launch run in different CTAs: each accumulates its gradient
  // in its own slice, summed into the total in shot order after the batch
  const size_t gslice = exact ? (size_t)S.fstride : nvel;
  // exact mode: always through the slices (one shot per batch too), so the
  // shots are summed in the same order whatever the batch size
  const bool sliced = exact || nsb > 1;
  const size_t o_gs = cv.add(sliced ? (size_t)nsb * gslice * 4 : 0);
  const size_t o_grad = cv.add(nvel * 4);
  const size_t o_m2v3 = cv.add(exact ? 0 : nvel * 4);
  const size_t o_mis = cv.add(8 * (1 + RESID_BLOCKS));
  const size_t o_mx = cv.add(16);
  const size_t nsrcf = (size_t)nvel * nt;  // one shot's source field
  const size_t o_dsrc = cv.add(dsrc && host ? (size_t)ns * nsrcf * 4 : 0);
  PW_TRY(ws.reserve(cv.total()));
  if (exact) plan_record().bytes = (long long)cv.total();
  char *base = ws.base();
  // snapshots, checkpoints and segment terms are written before they are
  // read: zero the rest only (the term buffer alone is tens of GB)
  PW_CUDA(cudaMemsetAsync(base, 0, o_snap, st));
  PW_CUDA(cudaMemsetAsync(base + o_ga, 0, cv.total() - o_ga, st));
  const float *d_vel = vel;
  if (host) {
    PW_TRY(to_device(base + o_vel, vel, nvel * 4, true, st));
    d_vel = at<float>(base, o_vel);
  }
  PW_TRY(check_vel_cfl(S, d_vel, nvel, st, at<unsigned>(base, o_mx)));
  PW_TRY(upload_common(S, base, o_geo, o_bz, o_bx, o_wav, wav, host, st));
  const float *d_dsrc = dsrc;
  if (dsrc && host) {
    PW_TRY(to_device(base + o_dsrc, dsrc, (size_t)ns * nsrcf * 4, true, st));
    d_dsrc = at<float>(base, o_dsrc);
  }
  if (weight) PW_TRY(to_device(base + o_w, weight, (size_t)nr * nt * 4, host, st));
  else PW_CUDA(cudaMemcpyAsync(base + o_w, wts.data(), wts.size() * 4, cudaMemcpyHostToDevice, st));
  {
    // dobs [shot][nr][nt] -> [shot][nt][nr]
    const float *src = dobs;
    if (host) {
      PW_TRY(to_device(base + o_dobs_in, dobs, (size_t)ns * nt * nr * 4, true, st));
      src = at<float>(base, o_dobs_in);
    }
    for (int s = 0; s < ns; s++) {
      dim3 tb(32, 8), tg(ceil_div(nt, 32), ceil_div(nr, 32));
      transpose_kernel<<<tg, tb, 0, st>>>(src + (size_t)s * nr * nt,
                                          at<float>(base, o_dobs) + (size_t)s * nt * nr, nr, nt);
    }
    PW_CUDA(cudaGetLastError());
  }
  float *V = at<float>(base, o_V);
  pad_V_kernel<<<1184, 256, 0, st>>>(d_vel, nz, nx, a->nb, S.pnz, S.pnx, S.lz, a->dt * a->dt, V);
  PW_CUDA(cudaGetLastError());
  float *gdev = at<float>(base, o_grad);
  float *gacc = at<float>(base, o_ga);
  double *dmis = at<double>(base, o_mis);
  PfArgs p;
  base_args(S, p);
  p.V = V;
  p.bz = at<float>(base, o_bz);
  p.bx = at<float>(base, o_bx);
  p.wav = at<float>(base, o_wav);
  if (!exact) {
    m2v3_kernel<<<592, 256, 0, st>>>(d_vel, nvel, at<float>(base, o_m2v3));
    PW_CUDA(cudaGetLastError());
    p.m2v3 = at<float>(base, o_m2v3);
  }
  p.wdt2 = (a->dt * interval) * (a->dt * interval);
  float *gtotal = exact ? gacc : gdev;
  float *gslices = at<float>(base, o_gs);
  p.grad = sliced ? gslices : gtotal;
  p.gstride = sliced ? (long long)gslice : 0;
  const size_t fs = (size_t)S.fstride;
  long long launches = 0;
  LoopTimer timer(st);
  timer.start();
  for (int s0 = 0; s0 < ns; s0 += nsb) {
    const int nb_ = std::min(nsb, ns - s0);
    float *A[MAXS], *B[MAXS];
    auto reset = [&]() -> int {
      for (int s = 0; s < nb_; s++) {
        A[s] = at<float>(base, o_A) + s * fs;
        B[s] = at<float>(base, o_B) + s * fs;
      }
      PW_CUDA(cudaMemsetAsync(base + o_A, 0, (size_t)nsb * fs * 4, st));
      PW_CUDA(cudaMemsetAsync(base + o_B, 0, (size_t)nsb * fs * 4, st));
      return PW_OK;
    };
    auto step = [&](int mode_, int it) -> int {
      p.it = it;
      for (int s = 0; s < nb_; s++) {
        p.cur[s] = A[s];
        p.nxt[s] = B[s];
      }
      PW_TRY(launch(S, p, mode_, st));
      launches++;
      for (int s = 0; s < nb_; s++) std::swap(A[s], B[s]);
      return PW_OK;
    };
    p.nshots = nb_;
    p.geo = at<ShotGeo>(base, o_geo) + s0;
    p.dsrc = d_dsrc ? d_dsrc + (size_t)s0 * nsrcf : nullptr;
    p.dsrc_stride = (long long)nsrcf;
    float *dd = at<float>(base, o_d);
    float *res = at<float>(base, o_res);
    float *ck = at<float>(base, o_ck);
    float *tb = at<float>(base, o_tb);
    float *snap = at<float>(base, o_snap);
    // ---- forward: traces, and snapshots (reference) or checkpoints (exact)
    PW_TRY(reset());
    p.rec = dd;
    p.tout = nullptr;
    p.snap_stride = (long long)wnt * nvel;
    const int n_last = exact ? (nck - 1) * k : nt;  // first step of the last segment
    p.tout_stride = (long long)k * fs;
    for (int it = 0; it < nt; it++) {
      if (exact && it % k == 0 && it < n_last) {
        const int m = it / k;
        for (int s = 0; s < nb_; s++) {
          float *c = ck + ((size_t)s * nck + m) * 2 * fs;
          PW_CUDA(cudaMemcpyAsync(c, A[s], fs * 4, cudaMemcpyDeviceToDevice, st));
          PW_CUDA(cudaMemcpyAsync(c + fs, B[s], fs * 4, cudaMemcpyDeviceToDevice, st));
        }
      }
      p.snap = (!exact && it % interval == 0) ? snap + (size_t)(it / interval) * nvel : nullptr;
      // the last segment's terms, which the backward pass reads first
      p.tout = it >= n_last ? tb + (size_t)(it - n_last) * fs : nullptr;
      PW_TRY(step(FWD, it));
    }
    p.rec = nullptr;
    p.snap = nullptr;
    p.tout = nullptr;
    // ---- residual and FP64 misfit
    const bool filt = use_lo || use_hi;  // weights applied after the filter
    residual_kernel<<<RESID_BLOCKS, 256, 0, st>>>(dd, at<float>(base, o_dobs) + (size_t)s0 * nt * nr,
                                                  filt ? nullptr : at<float>(base, o_w), res, nb_,
                                                  nt, nr, exact ? 1 : 0, dmis);
    misfit_sum_kernel<<<1, 32, 0, st>>>(dmis, RESID_BLOCKS);
    PW_CUDA(cudaGetLastError());
    if (filt) {
      butter_residual_kernel<<<ceil_div((long long)nb_ * nr, 128), 128, 0, st>>>(
          blo, bhi, use_lo, use_hi, res, nb_, nt, nr, at<float>(base, o_w));
      PW_CUDA(cudaGetLastError());
    }
    p.res = res;
    if (!exact) {
      // ---- backward with gradient_av's imaging (wave_fwigradient.c:201-241)
      PW_TRY(reset());
      p.wstride = (long long)wnt * nvel;
      for (int it = nt - 1; it >= 0; it--) {
        const int wit = it / interval;
        p.imaging = (it % interval == 0) && wit != wnt - 1 && wit != 0;
        if (p.imaging) {
          p.wprev = snap + (size_t)(wit - 1) * nvel;
          p.wcur = snap + (size_t)wit * nvel;
          p.wnext = snap + (size_t)(wit + 1) * nvel;
        }
        PW_TRY(step(ADJ_REF, it));
      }
    } else {
      // ---- backward by segments: restore checkpoint, recompute the forward
      // terms of the segment, run the exact adjoint over it
      float *PA[MAXS], *PB[MAXS];
      for (int s = 0; s < nb_; s++) {
        PA[s] = at<float>(base, o_A) + s * fs;  // reused: adjoint after the forward
        PB[s] = at<float>(base, o_B) + s * fs;
      }
      // the adjoint needs its own pair; the forward recompute restores from
      // the checkpoints into the segment buffer's first two slots
      PW_CUDA(cudaMemsetAsync(base + o_A, 0, (size_t)nsb * fs * 4, st));
      PW_CUDA(cudaMemsetAsync(base + o_B, 0, (size_t)nsb * fs * 4, st));
      float *adjA[MAXS], *adjB[MAXS];
      for (int s = 0; s < nb_; s++) {
        adjA[s] = PA[s];
        adjB[s] = PB[s];
      }
      p.tout_stride = (long long)k * fs;
      p.tin_stride = (long long)k * fs;
      for (int m = nck - 1; m >= 0; m--) {
        const int n0 = m * k, n1 = std::min(nt, n0 + k);
        // recompute: fwd pair lives in checkpoint m (overwritten, no longer needed)
        float *FA[MAXS], *FB[MAXS];
        for (int s = 0; s < nb_; s++) {
          FA[s] = ck + ((size_t)s * nck + m) * 2 * fs;
          FB[s] = FA[s] + fs;
        }
        for (int n = n0; n < n1 && m < nck - 1; n++) {  // the last segment is kept
          p.it = n;
          for (int s = 0; s < nb_; s++) {
            p.cur[s] = FA[s];
            p.nxt[s] = FB[s];
          }
          p.tout = tb + (size_t)(n - n0) * fs;
          PW_TRY(launch(S, p, FWD, st));
          launches++;
          for (int s = 0; s < nb_; s++) std::swap(FA[s], FB[s]);
        }
        p.tout = nullptr;
        for (int n = n1 - 1; n >= n0; n--) {
          p.it = n;
          for (int s = 0; s < nb_; s++) {
            p.cur[s] = adjA[s];
            p.nxt[s] = adjB[s];
          }
          p.tin = tb + (size_t)(n - n0) * fs;
          p.imaging = 1;
          PW_TRY(launch(S, p, ADJ_EXACT, st));
          launches++;
          for (int s = 0; s < nb_; s++) std::swap(adjA[s], adjB[s]);
        }
      }
      p.tin = nullptr;
      p.imaging = 0;
    }
    if (sliced) {
      sum_slices_kernel<<<592, 256, 0, st>>>(gslices, nb_, (long long)gslice, gtotal);
      PW_CUDA(cudaGetLastError());
      PW_CUDA(cudaMemsetAsync(gslices, 0, (size_t)nb_ * gslice * 4, st));
      launches++;
    }
  }
  timer.stop();
  if (exact) {
    fold_grad_kernel<<<592, 256, 0, st>>>(gacc, d_vel, nz, nx, a->nb, S.pnz, S.pnx, S.lz, gdev);
    PW_CUDA(cudaGetLastError());
  }
  PW_TRY(to_host(grad, gdev, nvel * 4, host, st));
  if (misfit) PW_CUDA(cudaMemcpyAsync(misfit, dmis, 8, cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(launches, launches + 8);
  return PW_OK;
}
}  // namespace pf
}  // namespace pw

extern "C" int pw_butter_apply(int n, int ntr, int low, float cutoff, int npoles, float *x,
                               int flags, void *stream) {
  PW_CHECK(x && n >= 0 && ntr >= 0, PW_ERR_VALUE, "bad arguments");
  PW_CHECK(npoles >= 1 && npoles <= BUTTER_MAXP, PW_ERR_VALUE, "npoles must be 1..%d", BUTTER_MAXP);
  if (n == 0 || ntr == 0) return PW_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const bool host = (flags & PW_HOST_PTRS) != 0;
  const ButterCoef b = butter_coef(low != 0, cutoff, npoles);
  const size_t bytes = (size_t)n * ntr * 4;
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  float *d = x;
  if (host) {
    PW_TRY(ws.reserve(bytes));
    d = reinterpret_cast<float *>(ws.base());
    PW_TRY(to_device(d, x, bytes, true, st));
  }
  butter_traces_kernel<<<ceil_div(ntr, 128), 128, 0, st>>>(b, d, n, ntr);
  PW_CUDA(cudaGetLastError());
  if (host) PW_TRY(to_host(x, d, bytes, true, st));
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

extern "C" int pw_residual_weights(int nt, int nr, int wtn1, int wtn2, int woffn1, int woffn2,
                                   int oreo, float *w) {
  PW_CHECK(w && nt >= 1 && nr >= 1, PW_ERR_VALUE, "bad arguments");
  PW_CHECK(0 <= wtn1 && wtn1 <= wtn2 && wtn2 < nt && 0 <= woffn1 && woffn1 <= woffn2 &&
               woffn2 < nr,
           PW_ERR_SHAPE, "window [%d,%d] x [%d,%d] must lie in %d x %d", woffn1, woffn2, wtn1,
           wtn2, nr, nt);
  weights_window(nt, nr, wtn1, wtn2, woffn1, woffn2, oreo != 0, w);
  return PW_OK;
}

extern "C" int pw_pfwi_gradient(const pw_fwi_args *a, int mode, const float *vel, const float *wav,
                                const float *dobs, const float *weight, float *grad,
                                double *misfit, int ckpt_k, void *stream) {
  PW_CHECK(wav != nullptr, PW_ERR_VALUE, "null wavelet");
  return gradient_impl(a, mode, vel, wav, nullptr, dobs, weight, grad, misfit, ckpt_k, stream);
}

extern "C" int pw_pfwi_gradient_passive(const pw_fwi_args *a, int mode, const float *vel,
                                        const float *src, const float *dobs, const float *weight,
                                        float *grad, double *misfit, int ckpt_k, void *stream) {
  PW_CHECK(src != nullptr, PW_ERR_VALUE, "null source field");
  return gradient_impl(a, mode, vel, nullptr, src, dobs, weight, grad, misfit, ckpt_k, stream);
}

// ------------------------------------------------------- visco-acoustic --
// forward_modeling (wave_fwimodeling.c:116-220) and gradient_v
// (wave_fwigradient.c:264-452): the pfwi scheme with a memory variable r,
//   r2 = (tau/taus*L + (idt - 0.5/taus)*r1) / (idt + 0.5/taus),
//   term = L*(1 + tau) - (r2 + r1)*0.5 + rr*w,  p2 = 2 p1 - p0 + V term,
// sponge on p0, p1 and r1; the adjoint pass forms r2 and tmp = p1*(1 + tau)
// - 0.5*(r2 + r1) from p1, r1 and takes the Laplacian of tmp.  The
// reference mixes float and double in these expressions; each operation is
// written with the matching explicitly rounded intrinsic.  Fields use a plain
// [pnx][pnz] layout; one thread per padded cell, Laplacian loads through L2.
// Only the cells [4, pad-4) change: the reference's forward_modeling also
// updates the 4-cell rim, where everything stays zero as long as no source
// cell lies there (the drivers check that).  As in the acoustic scheme, a
// field whose sponged value the step reads is stored before its last sponge
// (B for p0, R for r1), so p and r need no third buffer.
namespace pw {
namespace pf {

struct ViscoArgs {
  int pnz, pnx, nb, nz, nx;
  float c0, c1, c2, c3, c4, dx2, dz2, idt;
  const float *V, *tau, *taus, *bz, *bx;
  const float *A;        // p1 (sponged)
  float *B;              // in: p0 before its second sponge; out: the new p1
  float *R;              // in: r1 before its sponge; out: r2
  const float *rr;       // forward: dense source maps [shot][pnx][pnz]
  const float *wav;
  int it, nt;
  const ShotGeo *geo;
  int rz, drv, nr;
  float *rec;            // forward: traces [shot][nt][nr] or null
  float *snap;           // forward: interior snapshot of this step [nx][nz] or null
  long long fstride;     // floats per field (per shot)
  // adjoint
  const float *T;        // tmp field
  const float *res;      // residual [nt][nr] of the shot
  int imaging;
  const float *wprev, *wcur, *wnext, *m2v3;
  float wdt2;
  float *grad;
};

__device__ __forceinline__ float visco_lap(const ViscoArgs &a, const float *p, long long j) {
  const long long s = a.pnz;
  float tx = fmul(a.c0, p[j]);
  tx = fadd(tx, fmul(a.c1, fadd(p[j + s], p[j - s])));
  tx = fadd(tx, fmul(a.c2, fadd(p[j + 2 * s], p[j - 2 * s])));
  tx = fadd(tx, fmul(a.c3, fadd(p[j + 3 * s], p[j - 3 * s])));
  tx = fadd(tx, fmul(a.c4, fadd(p[j + 4 * s], p[j - 4 * s])));
  float tz = fmul(a.c0, p[j]);
  tz = fadd(tz, fmul(a.c1, fadd(p[j + 1], p[j - 1])));
  tz = fadd(tz, fmul(a.c2, fadd(p[j + 2], p[j - 2])));
  tz = fadd(tz, fmul(a.c3, fadd(p[j + 3], p[j - 3])));
  tz = fadd(tz, fmul(a.c4, fadd(p[j + 4], p[j - 4])));
  return fadd(fdiv(tx, a.dx2), fdiv(tz, a.dz2));
}

__device__ __forceinline__ float visco_sponge(const ViscoArgs &a, float v, int ix, int iz) {
  return fmul(a.bx[ix], fmul(a.bz[iz], v));  // z faces, then x faces (apply_sponge)
}

// one forward step of every shot of the batch (blockIdx.y = shot)
__global__ void visco_fwd_kernel(const ViscoArgs a) {
  const int s = blockIdx.y;
  const long long n = (long long)a.pnz * a.pnx;
  const float *A = a.A + s * a.fstride;
  float *B = a.B + s * a.fstride, *R = a.R + s * a.fstride;
  const float *rr = a.rr + s * n;
  const ShotGeo &g = a.geo[s];
  const float wv = a.wav[a.it];
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(j / a.pnz), iz = (int)(j - (long long)ix * a.pnz);
    const float p1 = A[j];
    if (a.rec && iz == a.rz) {  // traces read p1 before the step (wave_fwimodeling.c:181-185)
      const int d = ix - g.r0v;
      if (d >= 0 && d % a.drv == 0 && d / a.drv < g.nr2)
        a.rec[((size_t)s * a.nt + a.it) * a.nr + g.r02 + d / a.drv] = p1;
    }
    if (a.snap && ix >= a.nb && ix < a.nb + a.nx && iz >= a.nb && iz < a.nb + a.nz)
      a.snap[s * (long long)a.nx * a.nz + (long long)(ix - a.nb) * a.nz + (iz - a.nb)] = p1;
    if (ix < 4 || ix >= a.pnx - 4 || iz < 4 || iz >= a.pnz - 4) continue;
    const float L = visco_lap(a, A, j);
    const float tau = a.tau[j], taus = a.taus[j];
    const float r1 = visco_sponge(a, R[j], ix, iz);
    const double hts = __ddiv_rn(0.5, (double)taus);
    const double num = __dadd_rn((double)fmul(fdiv(tau, taus), L),
                                 __dmul_rn(__dsub_rn((double)a.idt, hts), (double)r1));
    const float r2 = __double2float_rn(__ddiv_rn(num, __dadd_rn((double)a.idt, hts)));
    const double tt = __dadd_rn(__dsub_rn(__dmul_rn((double)L, __dadd_rn(1.0, (double)tau)),
                                          __dmul_rn((double)fadd(r2, r1), 0.5)),
                                (double)fmul(rr[j], wv));
    const float t = __double2float_rn(tt);
    const float p0 = visco_sponge(a, B[j], ix, iz);
    const float p2 = fadd(fsub(fmul(2.f, p1), p0), fmul(a.V[j], t));
    B[j] = visco_sponge(a, p2, ix, iz);
    R[j] = r2;
  }
}

// adjoint, first half of a step: r2 and tmp from p1 and r1 (wave_fwigradient.c:393-403)
__global__ void visco_adj_pre_kernel(const ViscoArgs a) {
  const long long n = (long long)a.pnz * a.pnx;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(j / a.pnz), iz = (int)(j - (long long)ix * a.pnz);
    if (ix < 4 || ix >= a.pnx - 4 || iz < 4 || iz >= a.pnz - 4) continue;
    const float p1 = a.A[j], tau = a.tau[j], taus = a.taus[j];
    const float r1 = visco_sponge(a, a.R[j], ix, iz);
    const double hts = __ddiv_rn(0.5, (double)taus);
    const double nidt = -(double)a.idt;
    const double num = __dadd_rn((double)fmul(fdiv(-tau, taus), p1),
                                 __dmul_rn(__dadd_rn(nidt, hts), (double)r1));
    const float r2 = __double2float_rn(__ddiv_rn(num, __dsub_rn(nidt, hts)));
    const double tm = __dsub_rn(__dmul_rn((double)p1, __dadd_rn(1.0, (double)tau)),
                                __dmul_rn(0.5, (double)fadd(r2, r1)));
    const_cast<float *>(a.T)[j] = __double2float_rn(tm);
    a.R[j] = r2;
  }
}

// adjoint, second half: Laplacian of tmp plus the residual, the update, and
// gradient_av's imaging with p1 (wave_fwigradient.c:405-438)
__global__ void visco_adj_kernel(const ViscoArgs a) {
  const long long n = (long long)a.pnz * a.pnx;
  const ShotGeo &g = a.geo[0];
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(j / a.pnz), iz = (int)(j - (long long)ix * a.pnz);
    if (ix < 4 || ix >= a.pnx - 4 || iz < 4 || iz >= a.pnz - 4) continue;
    float L = visco_lap(a, a.T, j);
    if (iz == a.rz) {
      const int d = ix - g.r0v;
      if (d >= 0 && d % a.drv == 0 && d / a.drv < g.nr2)
        L = fadd(L, a.res[(size_t)a.it * a.nr + g.r02 + d / a.drv]);
    }
    const float p1 = a.A[j];
    const float p0 = visco_sponge(a, a.B[j], ix, iz);
    const float p2 = fadd(fsub(fmul(2.f, p1), p0), fmul(a.V[j], L));
    if (a.imaging && ix >= a.nb && ix < a.nb + a.nx && iz >= a.nb && iz < a.nb + a.nz) {
      const size_t k = (size_t)(ix - a.nb) * a.nz + (iz - a.nb);
      const double w = __dadd_rn(__dsub_rn((double)a.wnext[k], __dmul_rn(2., (double)a.wcur[k])),
                                 (double)a.wprev[k]);
      const double gsum = __dmul_rn(__dmul_rn(__ddiv_rn(w, (double)a.wdt2), (double)p1),
                                    (double)a.m2v3[k]);
      a.grad[k] = __double2float_rn(__dadd_rn((double)a.grad[k], gsum));
    }
    a.B[j] = visco_sponge(a, p2, ix, iz);
  }
}

// preparation's tau, taus (wave_fwiutil.c:90-96) and the pad2d copies
static void visco_tables(const Setup &S, const float *q_host, std::vector<float> &tp,
                         std::vector<float> &tsp, std::vector<float> &Vp, const float *vel_host) {
  const pw_fwi_args &a = S.a;
  const double pi = 3.14159265358979323846264338328;
  const size_t nzx = (size_t)a.nz * a.nx, np = (size_t)S.pnz * S.pnx;
  std::vector<float> t1(nzx), ts1(nzx);
  for (size_t i = 0; i < nzx; i++) {
    const float qq = q_host[i];
    const float tmp = sqrtf(qq * qq + 1);
    const float taue = (tmp + 1) / (2. * pi * a.f0 * qq);
    ts1[i] = (tmp - 1) / (2. * pi * a.f0 * qq);
    t1[i] = taue / ts1[i] - 1;
  }
  const float dt2 = a.dt * a.dt;
  tp.resize(np);
  tsp.resize(np);
  Vp.resize(np);
  for (int ix = 0; ix < S.pnx; ix++)
    for (int iz = 0; iz < S.pnz; iz++) {
      const int jx = std::min(std::max(ix - a.nb, 0), a.nx - 1);
      const int jz = std::min(std::max(iz - a.nb, 0), a.nz - 1);
      const size_t j = (size_t)ix * S.pnz + iz, k = (size_t)jx * a.nz + jz;
      tp[j] = t1[k];
      tsp[j] = ts1[k];
      const float v = vel_host[k];
      Vp[j] = (v * v) * dt2;
    }
}

// the shots' source maps as dense fields, checked clear of the 4-cell rim
static int visco_sources(const Setup &S, int ns, std::vector<float> &rr) {
  const size_t np = (size_t)S.pnz * S.pnx;
  rr.assign(np * ns, 0.f);
  for (int is = 0; is < ns; is++) {
    const ShotGeo &g = S.geo[is];
    for (int k = 0; k < g.nsrc; k++) {
      const int x = g.scell[k] >> 16, z = g.scell[k] & 0xffff;
      PW_CHECK(x >= 4 && x < S.pnx - 4 && z >= 4 && z < S.pnz - 4, PW_ERR_SHAPE,
               "visco-acoustic path: shot %d's source map reaches the 4-cell rim", is);
      rr[np * is + (size_t)x * S.pnz + z] = g.sw[k];
    }
  }
  return PW_OK;
}

static void visco_base(const Setup &S, ViscoArgs &v) {
  v = ViscoArgs{};
  v.pnz = S.pnz;
  v.pnx = S.pnx;
  v.nb = S.a.nb;
  v.nz = S.a.nz;
  v.nx = S.a.nx;
  const float c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
  v.c0 = c0; v.c1 = c1; v.c2 = c2; v.c3 = c3; v.c4 = c4;
  v.dx2 = S.a.dx * S.a.dx;
  v.dz2 = S.a.dz * S.a.dz;
  v.idt = 1. / S.a.dt;
  v.nt = S.a.nt;
  v.rz = S.rz;
  v.drv = S.drv;
  v.nr = S.nr;
  v.fstride = (long long)S.pnz * S.pnx;
}

// the acoustic path's stability limit on the host copy of the velocity
static int check_cfl_host(const Setup &S, const std::vector<float> &vh) {
  if (S.a.flags & PW_NO_CFL_CHECK) return PW_OK;
  float vmax = 0.f;
  for (float v : vh) vmax = std::max(vmax, v);
  const float cfl = vmax * S.a.dt / std::min(S.a.dx, S.a.dz);
  PW_CHECK(cfl <= 0.555f, PW_ERR_CFL, "unstable: vmax*dt/h = %g exceeds 0.555", cfl);
  return PW_OK;
}

// the host copies a visco call needs: velocity and quality factor
static int visco_host_inputs(const pw_fwi_args *a, const float *vel, const float *q,
                             std::vector<float> &vh, std::vector<float> &qh, cudaStream_t st) {
  const size_t nzx = (size_t)a->nz * a->nx;
  vh.resize(nzx);
  qh.resize(nzx);
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  if (host) {
    memcpy(vh.data(), vel, nzx * 4);
    memcpy(qh.data(), q, nzx * 4);
  } else {
    PW_CUDA(cudaMemcpyAsync(vh.data(), vel, nzx * 4, cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaMemcpyAsync(qh.data(), q, nzx * 4, cudaMemcpyDeviceToHost, st));
    PW_CUDA(cudaStreamSynchronize(st));
  }
  for (size_t i = 0; i < nzx; i++)
    PW_CHECK(vh[i] > 0.f && std::isfinite(vh[i]) && qh[i] > 0.f && std::isfinite(qh[i]),
             PW_ERR_VALUE, "velocity and quality factor must be finite and positive");
  return PW_OK;
}

}  // namespace pf
}  // namespace pw

extern "C" int pw_pfwi_forward_visco(const pw_fwi_args *a, const float *vel, const float *q,
                                     const float *wav, float *data, void *stream) {
  PW_CHECK(a && vel && q && wav && data, PW_ERR_VALUE, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  Setup S;
  PW_TRY(setup(a, S));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr;
  std::vector<float> vh, qh, tp, tsp, Vp, rr;
  PW_TRY(visco_host_inputs(a, vel, q, vh, qh, st));
  PW_TRY(check_cfl_host(S, vh));
  visco_tables(S, qh.data(), tp, tsp, Vp, vh.data());
  PW_TRY(visco_sources(S, ns, rr));
  const size_t np = (size_t)S.pnz * S.pnx;
  Carve cv;
  const size_t o_V = cv.add(np * 4), o_t = cv.add(np * 4), o_ts = cv.add(np * 4);
  const size_t o_A = cv.add((size_t)ns * np * 4), o_B = cv.add((size_t)ns * np * 4);
  const size_t o_R = cv.add((size_t)ns * np * 4), o_rr = cv.add((size_t)ns * np * 4);
  const size_t o_bz = cv.add(S.bz.size() * 4), o_bx = cv.add(S.bx.size() * 4);
  const size_t o_w = cv.add((size_t)nt * 4), o_geo = cv.add(sizeof(ShotGeo) * ns);
  const size_t o_rec = cv.add((size_t)ns * nt * nr * 4), o_out = cv.add((size_t)ns * nt * nr * 4);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  struct Drain {
    cudaStream_t st;
    ~Drain() { cudaStreamSynchronize(st); }
  } drain{st};
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  PW_CUDA(cudaMemcpyAsync(base + o_V, Vp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_t, tp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_ts, tsp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_rr, rr.data(), rr.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bz, S.bz.data(), S.bz.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bx, S.bx.data(), S.bx.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_geo, S.geo.data(), sizeof(ShotGeo) * ns,
                          cudaMemcpyHostToDevice, st));
  PW_TRY(to_device(base + o_w, wav, (size_t)nt * 4, host, st));
  ViscoArgs v;
  visco_base(S, v);
  v.V = at<float>(base, o_V);
  v.tau = at<float>(base, o_t);
  v.taus = at<float>(base, o_ts);
  v.bz = at<float>(base, o_bz);
  v.bx = at<float>(base, o_bx);
  v.rr = at<float>(base, o_rr);
  v.wav = at<float>(base, o_w);
  v.geo = at<ShotGeo>(base, o_geo);
  v.rec = at<float>(base, o_rec);
  v.R = at<float>(base, o_R);
  float *A = at<float>(base, o_A), *B = at<float>(base, o_B);
  const dim3 grid((unsigned)std::min<long long>(ceil_div((long long)np, 256), 1184), (unsigned)ns);
  LoopTimer timer(st);
  timer.start();
  for (int it = 0; it < nt; it++) {
    v.it = it;
    v.A = A;
    v.B = B;
    visco_fwd_kernel<<<grid, 256, 0, st>>>(v);
    PW_CUDA(cudaGetLastError());
    std::swap(A, B);
  }
  timer.stop();
  // traces [shot][nt][nr] -> data [shot][nr][nt]
  float *out = at<float>(base, o_out);
  for (int s = 0; s < ns; s++) {
    dim3 tb(32, 8), tg(ceil_div(nr, 32), ceil_div(nt, 32));
    transpose_kernel<<<tg, tb, 0, st>>>(v.rec + (size_t)s * nt * nr, out + (size_t)s * nr * nt,
                                        nt, nr);
  }
  PW_CUDA(cudaGetLastError());
  PW_TRY(to_host(data, out, (size_t)ns * nr * nt * 4, host, st));
  timer.finish(nt, nt + ns);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

extern "C" int pw_pfwi_gradient_visco(const pw_fwi_args *a, const float *vel, const float *q,
                                      const float *wav, const float *dobs, const float *weight,
                                      float *grad, double *misfit, void *stream) {
  PW_CHECK(a && vel && q && wav && dobs && grad, PW_ERR_VALUE, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  Setup S;
  PW_TRY(setup(a, S));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr, nz = a->nz, nx = a->nx;
  const size_t nzx = (size_t)nz * nx, np = (size_t)S.pnz * S.pnx;
  const int interval = std::max(1, a->interval);
  const int wnt = (nt - 1) / interval + 1;
  std::vector<float> vh, qh, tp, tsp, Vp, rr, wts;
  PW_TRY(visco_host_inputs(a, vel, q, vh, qh, st));
  PW_TRY(check_cfl_host(S, vh));
  visco_tables(S, qh.data(), tp, tsp, Vp, vh.data());
  PW_TRY(visco_sources(S, ns, rr));
  if (weight == nullptr) residual_weights(*a, nr, wts);
  Carve cv;
  const size_t o_V = cv.add(np * 4), o_t = cv.add(np * 4), o_ts = cv.add(np * 4);
  const size_t o_A = cv.add(np * 4), o_B = cv.add(np * 4), o_R = cv.add(np * 4);
  const size_t o_T = cv.add(np * 4), o_rr = cv.add((size_t)ns * np * 4);
  const size_t o_bz = cv.add(S.bz.size() * 4), o_bx = cv.add(S.bx.size() * 4);
  const size_t o_w = cv.add((size_t)nt * 4), o_geo = cv.add(sizeof(ShotGeo) * ns);
  const size_t o_wt = cv.add((size_t)nr * nt * 4);
  const size_t o_dobs = cv.add((size_t)ns * nt * nr * 4), o_din = cv.add((size_t)ns * nt * nr * 4);
  const size_t o_rec = cv.add((size_t)nt * nr * 4), o_res = cv.add((size_t)nt * nr * 4);
  const size_t o_snap = cv.add((size_t)wnt * nzx * 4);
  const size_t o_m2v3 = cv.add(nzx * 4), o_vel = cv.add(nzx * 4), o_grad = cv.add(nzx * 4);
  const size_t o_mis = cv.add(8 * (1 + RESID_BLOCKS));
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  struct Drain {
    cudaStream_t st;
    ~Drain() { cudaStreamSynchronize(st); }
  } drain{st};
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  PW_CUDA(cudaMemcpyAsync(base + o_V, Vp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_t, tp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_ts, tsp.data(), np * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_rr, rr.data(), rr.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bz, S.bz.data(), S.bz.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_bx, S.bx.data(), S.bx.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_geo, S.geo.data(), sizeof(ShotGeo) * ns,
                          cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + o_vel, vh.data(), nzx * 4, cudaMemcpyHostToDevice, st));
  PW_TRY(to_device(base + o_w, wav, (size_t)nt * 4, host, st));
  if (weight) PW_TRY(to_device(base + o_wt, weight, (size_t)nr * nt * 4, host, st));
  else PW_CUDA(cudaMemcpyAsync(base + o_wt, wts.data(), wts.size() * 4, cudaMemcpyHostToDevice, st));
  {
    PW_TRY(to_device(base + o_din, dobs, (size_t)ns * nt * nr * 4, host, st));
    for (int s = 0; s < ns; s++) {  // dobs [shot][nr][nt] -> [shot][nt][nr]
      dim3 tb(32, 8), tg(ceil_div(nt, 32), ceil_div(nr, 32));
      transpose_kernel<<<tg, tb, 0, st>>>(at<float>(base, o_din) + (size_t)s * nr * nt,
                                          at<float>(base, o_dobs) + (size_t)s * nt * nr, nr, nt);
    }
    PW_CUDA(cudaGetLastError());
  }
  m2v3_kernel<<<592, 256, 0, st>>>(at<float>(base, o_vel), nzx, at<float>(base, o_m2v3));
  PW_CUDA(cudaGetLastError());
  ViscoArgs v;
  visco_base(S, v);
  v.V = at<float>(base, o_V);
  v.tau = at<float>(base, o_t);
  v.taus = at<float>(base, o_ts);
  v.bz = at<float>(base, o_bz);
  v.bx = at<float>(base, o_bx);
  v.wav = at<float>(base, o_w);
  v.R = at<float>(base, o_R);
  v.T = at<float>(base, o_T);
  v.m2v3 = at<float>(base, o_m2v3);
  v.grad = at<float>(base, o_grad);
  v.wdt2 = (a->dt * interval) * (a->dt * interval);
  float *snap = at<float>(base, o_snap);
  double *dmis = at<double>(base, o_mis);
  const dim3 g1((unsigned)std::min<long long>(ceil_div((long long)np, 256), 1184), 1);
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  // one shot at a time: the gradient sums the shots in the reference's order
  for (int is = 0; is < ns; is++) {
    float *A = at<float>(base, o_A), *B = at<float>(base, o_B);
    PW_CUDA(cudaMemsetAsync(A, 0, np * 4, st));
    PW_CUDA(cudaMemsetAsync(B, 0, np * 4, st));
    PW_CUDA(cudaMemsetAsync(v.R, 0, np * 4, st));
    v.geo = at<ShotGeo>(base, o_geo) + is;
    v.rr = at<float>(base, o_rr) + (size_t)is * np;
    v.rec = at<float>(base, o_rec);
    for (int it = 0; it < nt; it++) {
      v.it = it;
      v.A = A;
      v.B = B;
      v.snap = it % interval == 0 ? snap + (size_t)(it / interval) * nzx : nullptr;
      visco_fwd_kernel<<<g1, 256, 0, st>>>(v);
      PW_CUDA(cudaGetLastError());
      launches++;
      std::swap(A, B);
    }
    v.snap = nullptr;
    v.rec = nullptr;
    residual_kernel<<<RESID_BLOCKS, 256, 0, st>>>(at<float>(base, o_rec),
                                                  at<float>(base, o_dobs) + (size_t)is * nt * nr,
                                                  at<float>(base, o_wt), at<float>(base, o_res), 1,
                                                  nt, nr, 0, dmis);
    misfit_sum_kernel<<<1, 32, 0, st>>>(dmis, RESID_BLOCKS);
    PW_CUDA(cudaGetLastError());
    v.res = at<float>(base, o_res);
    PW_CUDA(cudaMemsetAsync(A, 0, np * 4, st));
    PW_CUDA(cudaMemsetAsync(B, 0, np * 4, st));
    PW_CUDA(cudaMemsetAsync(v.R, 0, np * 4, st));
    for (int it = nt - 1; it >= 0; it--) {
      const int wit = it / interval;
      v.it = it;
      v.A = A;
      v.B = B;
      v.imaging = (it % interval == 0) && wit != wnt - 1 && wit != 0;
      if (v.imaging) {
        v.wprev = snap + (size_t)(wit - 1) * nzx;
        v.wcur = snap + (size_t)wit * nzx;
        v.wnext = snap + (size_t)(wit + 1) * nzx;
      }
      visco_adj_pre_kernel<<<g1, 256, 0, st>>>(v);
      visco_adj_kernel<<<g1, 256, 0, st>>>(v);
      PW_CUDA(cudaGetLastError());
      launches += 2;
      std::swap(A, B);
    }
  }
  timer.stop();
  PW_TRY(to_host(grad, at<float>(base, o_grad), nzx * 4, host, st));
  if (misfit) PW_CUDA(cudaMemcpyAsync(misfit, dmis, 8, cudaMemcpyDeviceToHost, st));
  timer.finish(launches, launches + 4 * ns + 2);
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

extern "C" int pw_last_fwi_plan(int *ckpt_k, int *shots_per_batch, long long *bytes,
                                double *recompute) {
  const PlanRecord &r = plan_record();
  if (ckpt_k) *ckpt_k = r.k;
  if (shots_per_batch) *shots_per_batch = r.nsb;
  if (bytes) *bytes = r.bytes;
  if (recompute) *recompute = r.recompute;
  return PW_OK;
}

extern "C" int pw_gradient_postprocess(int nz, int nx, int rect, int waterz, float *grad,
                                       float *scaling, int flags, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  PW_CHECK(nz >= 1 && nx >= 1 && grad && scaling, PW_ERR_VALUE, "bad arguments");
  const bool host = (flags & PW_HOST_PTRS) != 0;
  const size_t n = (size_t)nz * nx;
  Carve cv;
  const size_t o_g = cv.add(host ? n * 4 : 0);
  const size_t o_tmp = cv.add(rect > 1 ? (size_t)std::max(nz, nx) * (std::max(nz, nx) + 2 * rect) * 4 : 0);
  const size_t o_mx = cv.add(16);
  const size_t o_sc = cv.add(16);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  float *g = host ? at<float>(base, o_g) : grad;
  if (host) PW_TRY(to_device(g, grad, n * 4, true, st));
  unsigned *mx = at<unsigned>(base, o_mx);
  float *sc = at<float>(base, o_sc);
  PW_CUDA(cudaMemsetAsync(mx, 0, 4, st));
  PW_CUDA(cudaMemcpyAsync(sc, scaling, 4, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
  // the first-call scale comes from the raw gradient (wave_fwigradient.c:245-251)
  absmax_kernel<<<296, 256, 0, st>>>(g, (long long)n, mx);
  if (rect > 1) {
    float *tmp = at<float>(base, o_tmp);
    smooth_lines_kernel<<<ceil_div(nx, 128), 128, 0, st>>>(g, nx, nz, nz, 1, rect, tmp);
    smooth_lines_kernel<<<ceil_div(nz, 128), 128, 0, st>>>(g, nz, nx, 1, nz, rect, tmp);
  }
  finish_kernel<<<296, 256, 0, st>>>(g, nz, nx, waterz, mx, sc);
  PW_CUDA(cudaGetLastError());
  if (host) PW_TRY(to_host(grad, g, n * 4, true, st));
  PW_CUDA(cudaMemcpyAsync(scaling, sc, 4, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
  PW_CUDA(cudaStreamSynchronize(st));
  return PW_OK;
}

// =========================================================================
// 3-D extension of the pfwi scheme (config: 400 x 400 x 200 batched FWI
// gradient).  The reference has no 3-D FWI; the scheme restates its 2-D
// acoustic step (wave_fwimodeling.c:21-114, wave_fwiutil.c:19-223) on three
// axes, exactly as the FP64 / FP32 oracle of oracle/pw_oracle3d_body.h does:
//   term = ((Tx / dx^2 + Tz / dz^2) + Ty / dy^2) + r w_n   (each T the
//          8th-order sum, zero outside [4, pad-4) on every axis; the
//          divisions as products with 1/h^2 rounded to float),
//   next = S(2 a - S b + V term),  S = Sy(Sx(Sz u)),  V = (v v) dt^2.
// Field layout: z contiguous with a 4-cell halo in front, 4 halo columns and
// 4 halo planes on each side:  off(iz, ix, iy) = (iz + 4) + sx (ix + 4) +
// sy (iy + 4), sx = lz (a multiple of 32 floats), sy = lz (pnx + 8).
// =========================================================================
namespace pw {
namespace pf3 {

using pf::FWD;
using pf::ADJ_EXACT;
constexpr int MAXS3 = 16;    // shots per launch
constexpr int MAXSRC = 64;   // source-map cells per shot
constexpr int XT = 16;       // columns per CTA
constexpr int NR = 3;        // ring planes (plane y, y + 1, y + 2 in flight)

struct Shot {
  int nsrc;
  int sz0, sz1, sx0, sx1, sy0, sy1;  // bounding box of the source cells
  int scell[MAXSRC];                 // iz | ix << 11 | iy << 22
  float sw[MAXSRC];
};

struct Args {
  int pnz, pnx, pny, lz;
  long long sx, sy, fstride;
  int nz4, ZT, nzc, ych;
  float c0, c1, c2, c3, c4, rdx2, rdz2, rdy2;
  float one;  // 1.0f at run time: keeps packed products unfused (pk2 helpers)
  int nshots;
  const float *cur[MAXS3];
  float *nxt[MAXS3];
  const float *V;
  const float *bz, *bx, *by;
  int it, nt;
  const Shot *shots;
  int rz, nrx, nr;
  const int *rxmap, *rymap;  // receiver index along x / y, or -1
  const float *wav;
  float *rec;                // FWD: traces [shot][nt][nr] or null
  float *tout;               // FWD: term of this step [shot] (field layout) or null
  long long tout_stride;
  const float *res;          // ADJ: residual [shot][nt][nr]
  const float *tin;          // ADJ: forward term of this step [shot]
  long long tin_stride;
  float *grad;               // ADJ: phi * term accumulators (field layout) [shot]
  long long gstride;
};

__host__ __device__ inline long long off3(const Args &a, int iz, int ix, int iy) {
  return (long long)(iz + 4) + a.sx * (ix + 4) + a.sy * (iy + 4);
}

// One step over the CTA's ZT float4 x XT column tile, marching y: the tile of
// plane y (with a 1-float4 z halo and 4 halo columns each side) is staged in
// a 3-plane cp.async ring with one CTA barrier per plane; the y neighbours
// come from a 9-deep register queue of the thread's own float4.
template <int MODE>
__global__ void __launch_bounds__(512) pf3_step_kernel(const __grid_constant__ Args a) {
  extern __shared__ float4 sm3[];
  constexpr int NST = MODE == FWD ? 2 : 4;  // own streams: prev, V (, term, gradient)
  const int ZT = a.ZT, TZ = ZT + 2, TX = XT + 8;
  const int nthr = ZT * XT;
  const int tid = threadIdx.x, zt = tid % ZT, xt = tid / ZT;
  const int s = blockIdx.z;
  const int zc = blockIdx.x % a.nzc, xc = blockIdx.x / a.nzc;
  const int z4 = zc * ZT + zt, x = xc * XT + xt;
  const int y0 = blockIdx.y * a.ych, y1 = min(a.pny, y0 + a.ych);
  const bool live = z4 < a.nz4 && x < a.pnx;
  const int iz0 = 4 * z4;
  const int tile_n = TZ * TX, slot_n = tile_n + NST * nthr;
  const float *cur = a.cur[s];
  float *nxt = a.nxt[s];
  const float *tin = MODE == ADJ_EXACT ? a.tin + s * a.tin_stride : nullptr;
  float *gs = MODE == ADJ_EXACT ? a.grad + s * a.gstride : nullptr;
  const long long sy = a.sy;
  // own float4 in plane 0 (a safe in-range cell for idle threads)
  const long long o0 = live ? off3(a, iz0, x, 0) : off3(a, 0, 0, 0);
  // tile copies: element e = tid + k nthr of the TZ x TX tile, tz fastest
  constexpr int MAXCP = 4;  // TZ * TX <= 4 * nthr for ZT >= 4
  long long cpo[MAXCP];
  bool cok[MAXCP];
#pragma unroll
  for (int k = 0; k < MAXCP; k++) {
    const int e = tid + k * nthr;
    const int tz = e % TZ, tx = e / TZ;
    const int zz = zc * ZT - 1 + tz, col = xc * XT - 4 + tx;
    // the float4 at 4 zz + 4 must lie in the column, the column in the halo
    cok[k] = e < tile_n && zz >= -1 && 4 * zz + 8 <= a.lz && col >= -4 && col < a.pnx + 4;
    cpo[k] = cok[k] ? (long long)(4 * zz + 4) + a.sx * (col + 4) + sy * 4 : 0;
  }
  auto issue = [&](int p, int rs) {  // plane p into ring slot rs
    if (p < y1) {
      float4 *dst = sm3 + rs * slot_n;
      const long long py = sy * p;
#pragma unroll
      for (int k = 0; k < MAXCP; k++) {
        const int e = tid + k * nthr;
        if (e < tile_n) pf::cp16(dst + e, cur + (cok[k] ? cpo[k] + py : 0), cok[k]);
      }
      float4 *own = dst + tile_n + tid;
      pf::cp16(own, nxt + o0 + py, live);
      pf::cp16(own + nthr, a.V + o0 + py, live);
      if (MODE == ADJ_EXACT) {
        pf::cp16(own + 2 * nthr, tin + o0 + py, live);
        pf::cp16(own + 3 * nthr, gs + o0 + py, live);
      }
    }
    pf::cp_commit();
  };

  float bzf[4];
  bool lz_ok[4], zin[4];
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int iz = iz0 + e;
    bzf[e] = (live && iz < a.pnz) ? a.bz[iz] : 1.f;
    lz_ok[e] = iz >= 4 && iz < a.pnz - 4;
    zin[e] = iz < a.pnz;
  }
  const float bxf = live ? a.bx[x] : 1.f;
  const bool lx_ok = x >= 4 && x < a.pnx - 4;
  const bool rec_row = live && a.rz >= iz0 && a.rz < iz0 + 4;
  const int rx_i = rec_row ? a.rxmap[x] : -1;
  const Shot &sh = a.shots[s];
  const bool src_zx = MODE == FWD && live && iz0 <= sh.sz1 && iz0 + 3 >= sh.sz0 && x >= sh.sx0 &&
                      x <= sh.sx1;
  const int ci = (xt + 4) * TZ + zt + 1;  // own float4 in the tile

  // y queue: q[k] = own float4 of plane y - 4 + k
  float4 q[9];
  const float *pc = cur + o0;
#pragma unroll
  for (int k = 0; k < 8; k++) q[k] = __ldg(reinterpret_cast<const float4 *>(pc + sy * (y0 - 4 + k)));
  float4 qn = __ldg(reinterpret_cast<const float4 *>(pc + sy * (y0 + 4)));
  issue(y0, 0);
  issue(y0 + 1, 1);
  int rs = 0;  // ring slot of plane y
  for (int y = y0; y < y1; y++) {
    pf::cp_wait<1>();
    __syncthreads();  // plane y staged; every thread is done with plane y - 1
    issue(y + 2, rs == 0 ? 2 : rs - 1);  // into the slot plane y - 1 left
    q[8] = qn;
    if (y + 1 < y1) qn = __ldg(reinterpret_cast<const float4 *>(pc + sy * (y + 5)));
    const float4 *tile = sm3 + rs * slot_n;
    const float4 *own = tile + tile_n + tid;
    if (live) {
      const float4 c = q[4];
      const float4 L = tile[ci - 1], R = tile[ci + 1];
      const float4 xm1 = tile[ci - TZ], xp1 = tile[ci + TZ];
      const float4 xm2 = tile[ci - 2 * TZ], xp2 = tile[ci + 2 * TZ];
      const float4 xm3 = tile[ci - 3 * TZ], xp3 = tile[ci + 3 * TZ];
      const float4 xm4 = tile[ci - 4 * TZ], xp4 = tile[ci + 4 * TZ];
      const float4 pv = own[0], V4 = own[nthr];
      const float byf = a.by[y];
      const bool ly_ok = y >= 4 && y < a.pny - 4;
      const long long o = o0 + sy * y;
      int trace = -1;
      if (rec_row && rx_i >= 0) {
        const int ry_j = a.rymap[y];
        if (ry_j >= 0) trace = ry_j * a.nrx + rx_i;
      }
      if (MODE == FWD && trace >= 0 && a.rec)
        a.rec[((size_t)s * a.nt + a.it) * a.nr + trace] = pf::el(c, a.rz - iz0);
      const bool src_here = src_zx && y >= sh.sy0 && y <= sh.sy1;
      float4 term4, res4, lap4;
      const f2 k1 = pk2(a.one, a.one);
      {
        // the 8th-order sums along x, z and y in the reference's order, and
        // (tx / dx^2 + tz / dz^2) + ty / dy^2, for cells (0, 1) and (2, 3)
        // of the float4 per f32x2 op; the z neighbours at odd distances are
        // the float4s shifted by one cell
        const f2 kc[5] = {pk2(a.c0, a.c0), pk2(a.c1, a.c1), pk2(a.c2, a.c2), pk2(a.c3, a.c3),
                          pk2(a.c4, a.c4)};
        const f2 rx2 = pk2(a.rdx2, a.rdx2), rz2 = pk2(a.rdz2, a.rdz2), ry2 = pk2(a.rdy2, a.rdy2);
        const f2 cl = lo2(c), ch = hi2(c);
        const f2 s_wx = pk2(L.w, c.x), s_yz = pk2(c.y, c.z), s_wR = pk2(c.w, R.x);
        const f2 s_Lyz = pk2(L.y, L.z), s_Ryz = pk2(R.y, R.z);
        const f2 zp[2][4] = {{s_yz, ch, s_wR, lo2(R)}, {s_wR, lo2(R), s_Ryz, hi2(R)}};
        const f2 zm[2][4] = {{s_wx, hi2(L), s_Lyz, lo2(L)}, {s_yz, cl, s_wx, hi2(L)}};
        const float4 *xp[4] = {&xp1, &xp2, &xp3, &xp4}, *xm[4] = {&xm1, &xm2, &xm3, &xm4};
        f2 t2[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const f2 cv2 = h ? ch : cl;
          f2 tx = mul2(mul2(kc[0], cv2), k1), tz = tx, ty = tx;
#pragma unroll
          for (int d = 1; d <= 4; d++) {
            const f2 xs = h ? add2(hi2(*xp[d - 1]), hi2(*xm[d - 1]))
                            : add2(lo2(*xp[d - 1]), lo2(*xm[d - 1]));
            tx = add2(tx, mul2(mul2(kc[d], xs), k1));
          }
#pragma unroll
          for (int d = 1; d <= 4; d++)
            tz = add2(tz, mul2(mul2(kc[d], add2(zp[h][d - 1], zm[h][d - 1])), k1));
#pragma unroll
          for (int d = 1; d <= 4; d++) {
            const f2 ys = h ? add2(hi2(q[4 + d]), hi2(q[4 - d])) : add2(lo2(q[4 + d]), lo2(q[4 - d]));
            ty = add2(ty, mul2(mul2(kc[d], ys), k1));
          }
          const f2 sxz = add2(mul2(mul2(tx, rx2), k1), mul2(mul2(tz, rz2), k1));
          t2[h] = add2(sxz, mul2(mul2(ty, ry2), k1));
        }
        lap4 = join2(t2[0], t2[1]);
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        float t = (lz_ok[e] && lx_ok && ly_ok) ? pf::el(lap4, e) : 0.f;
        const int iz = iz0 + e;
        if (MODE == FWD) {
          if (src_here) {
            const int key = iz | (x << 11) | (y << 22);
            for (int k = 0; k < sh.nsrc; k++)
              if (sh.scell[k] == key) t = fadd(t, fmul(sh.sw[k], a.wav[a.it]));
          }
        } else if (trace >= 0 && iz == a.rz) {
          t = fadd(t, a.res[((size_t)s * a.nt + a.it) * a.nr + trace]);
        }
        pf::set_el(term4, e, t);
      }
      {
        // taper of the stored u_{k-1} (z, then x, then y faces), the update
        // with 2 c as c + c (the same bits, no product to fuse), the taper
        const f2 bx2 = pk2(bxf, bxf), by2 = pk2(byf, byf);
        f2 r2[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const f2 bz2 = pk2(bzf[2 * h], bzf[2 * h + 1]);
          const f2 cv2 = h ? hi2(c) : lo2(c);
          const f2 p = mul2(mul2(by2, mul2(bx2, mul2(bz2, h ? hi2(pv) : lo2(pv)))), k1);
          const f2 vt = mul2(mul2(h ? hi2(V4) : lo2(V4), h ? hi2(term4) : lo2(term4)), k1);
          const f2 v = add2(sub2(add2(cv2, cv2), p), vt);
          r2[h] = mul2(by2, mul2(bx2, mul2(bz2, v)));
        }
        res4 = join2(r2[0], r2[1]);
#pragma unroll
        for (int e = 0; e < 4; e++)
          if (!zin[e]) pf::set_el(res4, e, 0.f);
      }
      *reinterpret_cast<float4 *>(nxt + o) = res4;
      if (MODE == FWD && a.tout)
        *reinterpret_cast<float4 *>(a.tout + s * a.tout_stride + o) = term4;
      if (MODE == ADJ_EXACT) {
        const float4 tf = own[2 * nthr];
        const float4 g0 = own[3 * nthr];
        const float4 g = join2(add2(lo2(g0), mul2(mul2(lo2(c), lo2(tf)), k1)),
                               add2(hi2(g0), mul2(mul2(hi2(c), hi2(tf)), k1)));
        *reinterpret_cast<float4 *>(gs + o) = g;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) q[k] = q[k + 1];
    rs = rs == 2 ? 0 : rs + 1;
  }
  pf::cp_wait_all();
}

// V = (v v) dt^2 on the padded grid (edge replication on every face)
__global__ void pad_V3_kernel(const float *vel, int nz, int nx, int ny, int nb, Args g, float dt2,
                              float *V) {
  const long long n = (long long)g.pnz * g.pnx * g.pny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int iz = int(i % g.pnz), ix = int((i / g.pnz) % g.pnx), iy = int(i / ((long long)g.pnz * g.pnx));
    const int jz = min(max(iz - nb, 0), nz - 1), jx = min(max(ix - nb, 0), nx - 1);
    const int jy = min(max(iy - nb, 0), ny - 1);
    const float v = vel[((size_t)jy * nx + jx) * nz + jz];
    V[off3(g, iz, ix, iy)] = fmul(fmul(v, v), dt2);
  }
}

// dJ/dv = 2 / v * sum of the accumulators of the padded cells that pad3d
// copies from the interior cell (edge replication adjoint)
__global__ void fold_grad3_kernel(const float *gacc, const float *vel, int nz, int nx, int ny,
                                  int nb, Args g, float *grad) {
  const long long n = (long long)nz * nx * ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int jz = int(i % nz), jx = int((i / nz) % nx), jy = int(i / ((long long)nz * nx));
    const int z_lo = jz == 0 ? 0 : jz + nb, z_hi = jz == nz - 1 ? g.pnz - 1 : jz + nb;
    const int x_lo = jx == 0 ? 0 : jx + nb, x_hi = jx == nx - 1 ? g.pnx - 1 : jx + nb;
    const int y_lo = jy == 0 ? 0 : jy + nb, y_hi = jy == ny - 1 ? g.pny - 1 : jy + nb;
    double s = 0.0;
    for (int iy = y_lo; iy <= y_hi; iy++)
      for (int ix = x_lo; ix <= x_hi; ix++)
        for (int iz = z_lo; iz <= z_hi; iz++) s += (double)gacc[off3(g, iz, ix, iy)];
    grad[i] = (float)(2.0 * s / (double)vel[i]);
  }
}

struct Setup3 {
  pw_fwi3d_args a;
  Args g;  // geometry part of the step arguments
  std::vector<float> bz, bx, by;
  std::vector<Shot> shots;
  std::vector<int> rxmap, rymap;
  int nr;
};

// Source map of one shot: the spike at padded (sz, sx, sy) smoothed by the
// rect-2 triangle along z and x (pf::source_map) and along y.
static int source_map3(int sz, int sx, int sy, const Setup3 &S, Shot &sh) {
  pf::ShotGeo g2;
  PW_TRY(pf::source_map(sx, sz, S.g.pnz, S.g.pnx, g2));
  const int pny = S.g.pny, r = 6;
  const int y_lo = std::max(0, sy - r), y_hi = std::min(pny - 1, sy + r);
  const bool full = y_lo == 0 || y_hi == pny - 1;
  const int ys = full ? 0 : y_lo, nyw = full ? pny : y_hi - y_lo + 1;
  std::vector<float> fy(nyw, 0.f), tmp;
  fy[sy - ys] = 1.f;
  pf::smooth_line_host(2, nyw, fy.data(), 0, 1, tmp);
  sh.nsrc = 0;
  sh.sz0 = sh.sx0 = sh.sy0 = 1 << 30;
  sh.sz1 = sh.sx1 = sh.sy1 = -1;
  for (int j = 0; j < nyw; j++) {
    if (fy[j] == 0.f) continue;
    const int gy = j + ys;
    PW_CHECK(gy >= 4 && gy < pny - 4, PW_ERR_SHAPE,
             "source map reaches the zero border of the padded grid");
    for (int k = 0; k < g2.nsrc; k++) {
      PW_CHECK(sh.nsrc < MAXSRC, PW_ERR_SHAPE, "source map has too many cells");
      const int gx = g2.scell[k] >> 16, gz = g2.scell[k] & 0xffff;
      sh.scell[sh.nsrc] = gz | (gx << 11) | (gy << 22);
      sh.sw[sh.nsrc] = g2.sw[k] * fy[j];
      sh.nsrc++;
      sh.sz0 = std::min(sh.sz0, gz); sh.sz1 = std::max(sh.sz1, gz);
      sh.sx0 = std::min(sh.sx0, gx); sh.sx1 = std::max(sh.sx1, gx);
      sh.sy0 = std::min(sh.sy0, gy); sh.sy1 = std::max(sh.sy1, gy);
    }
  }
  return PW_OK;
}

static int setup3(const pw_fwi3d_args *a, Setup3 &S) {
  PW_CHECK(a != nullptr, PW_ERR_VALUE, "null args");
  S.a = *a;
  PW_CHECK(a->nz >= 1 && a->nx >= 1 && a->ny >= 1 && a->nt >= 1 && a->ns >= 1 && a->nb >= 5,
           PW_ERR_SHAPE, "sizes must be positive and nb >= 5 (nz=%d nx=%d ny=%d nt=%d ns=%d nb=%d)",
           a->nz, a->nx, a->ny, a->nt, a->ns, a->nb);
  PW_CHECK(a->dx > 0 && a->dy > 0 && a->dz > 0 && a->dt > 0, PW_ERR_VALUE,
           "spacings must be positive");
  PW_CHECK(a->src && a->rx && a->ry && a->nrx >= 1 && a->nry >= 1, PW_ERR_VALUE,
           "sources and receivers are required");
  Args &g = S.g;
  memset(&g, 0, sizeof g);
  const int nb = a->nb;
  g.pnz = a->nz + 2 * nb;
  g.pnx = a->nx + 2 * nb;
  g.pny = a->ny + 2 * nb;
  PW_CHECK(g.pnz < 2048 && g.pnx < 2048 && g.pny < 512, PW_ERR_SHAPE,
           "padded grid beyond 2047 x 2047 x 511");
  g.lz = (int)round_up(4 + round_up(g.pnz, 4) + 4, 32);
  g.sx = g.lz;
  g.sy = (long long)g.lz * (g.pnx + 8);
  g.fstride = g.sy * (g.pny + 8) + 64;
  g.nz4 = ceil_div(g.pnz, 4);
  const int nzc = ceil_div(g.nz4, 32);
  g.ZT = std::max(4, ceil_div(g.nz4, nzc));
  g.nzc = ceil_div(g.nz4, g.ZT);
  const float c0 = -205. / 72, c1 = 8. / 5, c2 = -1. / 5, c3 = 8. / 315, c4 = -1. / 560;
  g.c0 = c0; g.c1 = c1; g.c2 = c2; g.c3 = c3; g.c4 = c4;
  g.rdz2 = 1.f / (a->dz * a->dz);
  g.rdx2 = 1.f / (a->dx * a->dx);
  g.rdy2 = 1.f / (a->dy * a->dy);
  g.one = 1.f;
  g.nt = a->nt;
  std::vector<float> bc(nb);
  for (int i = 0; i < nb; i++) {
    const float tmp = a->coef * (nb - i);
    bc[i] = expf(-tmp * tmp);
  }
  auto axis = [&](int n, std::vector<float> &f) {
    f.assign(n, 1.f);
    for (int i = 0; i < nb; i++) f[i] = bc[i];
    for (int i = n - nb; i < n; i++) f[i] = bc[n - i - 1];
  };
  axis(g.pnz, S.bz);
  axis(g.pnx, S.bx);
  axis(g.pny, S.by);
  // receivers: the nrx x nry grid (rx[i], ry[j]) at depth rz, trace j nrx + i
  PW_CHECK(a->rz >= 0 && a->rz < a->nz, PW_ERR_SHAPE, "receiver depth outside the model");
  g.rz = a->rz + nb;
  g.nrx = a->nrx;
  S.nr = a->nrx * a->nry;
  g.nr = S.nr;
  S.rxmap.assign(g.pnx, -1);
  S.rymap.assign(g.pny, -1);
  for (int i = 0; i < a->nrx; i++) {
    PW_CHECK(a->rx[i] >= 0 && a->rx[i] < a->nx, PW_ERR_SHAPE, "receiver x index %d outside", i);
    PW_CHECK(S.rxmap[a->rx[i] + nb] < 0, PW_ERR_SHAPE, "receiver x index %d repeated", i);
    S.rxmap[a->rx[i] + nb] = i;
  }
  for (int j = 0; j < a->nry; j++) {
    PW_CHECK(a->ry[j] >= 0 && a->ry[j] < a->ny, PW_ERR_SHAPE, "receiver y index %d outside", j);
    PW_CHECK(S.rymap[a->ry[j] + nb] < 0, PW_ERR_SHAPE, "receiver y index %d repeated", j);
    S.rymap[a->ry[j] + nb] = j;
  }
  S.shots.assign(a->ns, Shot{});
  for (int is = 0; is < a->ns; is++) {
    const int z = a->src[3 * is], x = a->src[3 * is + 1], y = a->src[3 * is + 2];
    PW_CHECK(z >= 0 && z < a->nz && x >= 0 && x < a->nx && y >= 0 && y < a->ny, PW_ERR_SHAPE,
             "shot %d: source (z=%d, x=%d, y=%d) outside the model", is, z, x, y);
    PW_TRY(source_map3(z + nb, x + nb, y + nb, S, S.shots[is]));
  }
  return PW_OK;
}

static size_t smem3(const Args &g, int mode) {
  const int nthr = g.ZT * XT;
  const int slot = (g.ZT + 2) * (XT + 8) + (mode == FWD ? 2 : 4) * nthr;
  return (size_t)NR * slot * sizeof(float4);
}

template <int MODE>
static int launch3_t(const Args &p, cudaStream_t st) {
  const size_t smem = smem3(p, MODE);
  static bool attr = false;
  if (!attr) {
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncSetAttribute(pf3_step_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
    cudaGetLastError();
    attr = true;
  }
  const dim3 grid((unsigned)(p.nzc * ceil_div(p.pnx, XT)), (unsigned)ceil_div(p.pny, p.ych),
                  (unsigned)p.nshots);
  pf3_step_kernel<MODE><<<grid, p.ZT * XT, smem, st>>>(p);
  PW_CUDA(cudaGetLastError());
  return PW_OK;
}
static int launch3(const Args &p, int mode, cudaStream_t st) {
  return mode == FWD ? launch3_t<FWD>(p, st) : launch3_t<ADJ_EXACT>(p, st);
}

// planes per CTA: enough CTAs for every SM a few times over
static int plan_ych(const Args &g, int nshots) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long cols = (long long)g.nzc * ceil_div(g.pnx, XT) * nshots;
  int ych = g.pny;
  while (ych > 16 && cols * ceil_div(g.pny, ych) < 8LL * nsm) ych = (ych + 1) / 2;
  return ych;
}

}  // namespace pf3
}  // namespace pw

using namespace pw::pf3;

// common device state of a 3-D call
namespace pw {
namespace pf3 {
struct Bound3 {
  size_t o_V, o_A, o_B, o_bz, o_bx, o_by, o_shots, o_rxm, o_rym, o_wav;
};
static void carve3(const Setup3 &S, int nsb, Carve &cv, Bound3 &b) {
  const size_t fb = (size_t)S.g.fstride * 4;
  b.o_V = cv.add(fb);
  b.o_A = cv.add((size_t)nsb * fb);
  b.o_B = cv.add((size_t)nsb * fb);
  b.o_bz = cv.add(S.bz.size() * 4);
  b.o_bx = cv.add(S.bx.size() * 4);
  b.o_by = cv.add(S.by.size() * 4);
  b.o_shots = cv.add(sizeof(Shot) * S.shots.size());
  b.o_rxm = cv.add(S.rxmap.size() * 4);
  b.o_rym = cv.add(S.rymap.size() * 4);
  b.o_wav = cv.add((size_t)S.a.nt * 4);
}
static int upload3(const Setup3 &S, char *base, const Bound3 &b, const float *wav, bool host,
                   cudaStream_t st) {
  PW_CUDA(cudaMemcpyAsync(base + b.o_bz, S.bz.data(), S.bz.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + b.o_bx, S.bx.data(), S.bx.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + b.o_by, S.by.data(), S.by.size() * 4, cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + b.o_shots, S.shots.data(), sizeof(Shot) * S.shots.size(),
                          cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + b.o_rxm, S.rxmap.data(), S.rxmap.size() * 4,
                          cudaMemcpyHostToDevice, st));
  PW_CUDA(cudaMemcpyAsync(base + b.o_rym, S.rymap.data(), S.rymap.size() * 4,
                          cudaMemcpyHostToDevice, st));
  PW_TRY(to_device(base + b.o_wav, wav, (size_t)S.a.nt * 4, host, st));
  return PW_OK;
}
static void bind3(const Setup3 &S, char *base, const Bound3 &b, Args &p) {
  p = S.g;
  p.V = at<float>(base, b.o_V);
  p.bz = at<float>(base, b.o_bz);
  p.bx = at<float>(base, b.o_bx);
  p.by = at<float>(base, b.o_by);
  p.shots = at<Shot>(base, b.o_shots);
  p.rxmap = at<int>(base, b.o_rxm);
  p.rymap = at<int>(base, b.o_rym);
  p.wav = at<float>(base, b.o_wav);
}
static int prep_vel3(const Setup3 &S, const float *vel, bool host, char *base, size_t o_vel,
                     size_t o_mx, const Bound3 &b, const float **d_vel, cudaStream_t st) {
  const size_t nvel = (size_t)S.a.nz * S.a.nx * S.a.ny;
  *d_vel = vel;
  if (host) {
    PW_TRY(to_device(base + o_vel, vel, nvel * 4, true, st));
    *d_vel = at<float>(base, o_vel);
  }
  unsigned *mx = at<unsigned>(base, o_mx);
  PW_CUDA(cudaMemsetAsync(mx, 0, 8, st));
  pf::vel_check_kernel<<<296, 256, 0, st>>>(*d_vel, (long long)nvel, mx);
  PW_CUDA(cudaGetLastError());
  unsigned hv[2] = {0, 0};
  PW_CUDA(cudaMemcpyAsync(hv, mx, 8, cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  float vmax;
  memcpy(&vmax, &hv[0], 4);
  PW_CHECK(hv[1] == 0 && vmax > 0.f, PW_ERR_VALUE, "velocity has non-finite or non-positive values");
  if (!(S.a.flags & PW_NO_CFL_CHECK)) {
    // 8th-order leapfrog in 3-D: v dt / h <= 0.453 (measured limit)
    const float h = std::min(S.a.dx, std::min(S.a.dy, S.a.dz));
    const float cfl = vmax * S.a.dt / h;
    PW_CHECK(cfl <= 0.453f, PW_ERR_CFL, "unstable: vmax*dt/h = %g exceeds 0.453", cfl);
  }
  pad_V3_kernel<<<1184, 256, 0, st>>>(*d_vel, S.a.nz, S.a.nx, S.a.ny, S.a.nb, S.g,
                                      S.a.dt * S.a.dt, at<float>(base, b.o_V));
  PW_CUDA(cudaGetLastError());
  return PW_OK;
}
}  // namespace pf3
}  // namespace pw

extern "C" int pw_pfwi3d_forward(const pw_fwi3d_args *a, const float *vel, const float *wav,
                                 float *data, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  Setup3 S;
  PW_TRY(setup3(a, S));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr;
  const int nsb = std::min(ns, MAXS3);
  const size_t nvel = (size_t)a->nz * a->nx * a->ny;
  const size_t fs = (size_t)S.g.fstride;
  Carve cv;
  Bound3 b;
  carve3(S, nsb, cv, b);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_rec = cv.add((size_t)ns * nt * nr * 4);
  const size_t o_out = cv.add(host ? (size_t)ns * nt * nr * 4 : 0);
  const size_t o_mx = cv.add(16);
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  PW_TRY(ws.reserve(cv.total()));
  char *base = ws.base();
  PW_CUDA(cudaMemsetAsync(base, 0, cv.total(), st));
  const float *d_vel;
  PW_TRY(upload3(S, base, b, wav, host, st));
  PW_TRY(prep_vel3(S, vel, host, base, o_vel, o_mx, b, &d_vel, st));
  Args p;
  bind3(S, base, b, p);
  float *rec = at<float>(base, o_rec);
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  for (int s0 = 0; s0 < ns; s0 += nsb) {
    const int nb_ = std::min(nsb, ns - s0);
    float *A[MAXS3], *B[MAXS3];
    for (int s = 0; s < nb_; s++) {
      A[s] = at<float>(base, b.o_A) + s * fs;
      B[s] = at<float>(base, b.o_B) + s * fs;
    }
    PW_CUDA(cudaMemsetAsync(base + b.o_A, 0, (size_t)nsb * fs * 4, st));
    PW_CUDA(cudaMemsetAsync(base + b.o_B, 0, (size_t)nsb * fs * 4, st));
    p.nshots = nb_;
    p.shots = at<Shot>(base, b.o_shots) + s0;
    p.rec = rec + (size_t)s0 * nt * nr;
    p.ych = plan_ych(S.g, nb_);
    for (int it = 0; it < nt; it++) {
      p.it = it;
      for (int s = 0; s < nb_; s++) {
        p.cur[s] = A[s];
        p.nxt[s] = B[s];
      }
      PW_TRY(launch3(p, FWD, st));
      launches++;
      for (int s = 0; s < nb_; s++) std::swap(A[s], B[s]);
    }
  }
  timer.stop();
  // [shot][nt][nr] -> [shot][nr][nt]
  float *dst = host ? at<float>(base, o_out) : data;
  for (int s = 0; s < ns; s++) {
    dim3 tb(32, 8), tg(ceil_div(nr, 32), ceil_div(nt, 32));
    pf::transpose_kernel<<<tg, tb, 0, st>>>(rec + (size_t)s * nt * nr, dst + (size_t)s * nt * nr,
                                            nt, nr);
  }
  PW_CUDA(cudaGetLastError());
  if (host) PW_TRY(to_host(data, dst, (size_t)ns * nt * nr * 4, true, st));
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(launches, launches + 3 + ns);
  return PW_OK;
}

extern "C" int pw_pfwi3d_gradient(const pw_fwi3d_args *a, const float *vel, const float *wav,
                                  const float *dobs, const float *weight, float *grad,
                                  double *misfit, int ckpt_k, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  Setup3 S;
  PW_TRY(setup3(a, S));
  const bool host = (a->flags & PW_HOST_PTRS) != 0;
  const int ns = a->ns, nt = a->nt, nr = S.nr;
  const size_t nvel = (size_t)a->nz * a->nx * a->ny;
  const size_t fs = (size_t)S.g.fstride;
  Workspace &ws = Workspace::for_current_device();
  std::lock_guard<std::mutex> lock(ws.mutex());
  // checkpoint plan: the 2-D planner's rule on 3-D fields
  pf::Setup P{};
  P.a.nt = nt;
  P.a.ns = std::min(ns, MAXS3);
  P.a.hbm_budget = a->hbm_budget;
  P.fstride = S.g.fstride;
  const ExactPlan ep = plan_exact(P, ckpt_k, ws.capacity());
  const int k = ep.k, nsb = ep.nsb, nck = (nt + k - 1) / k;
  plan_record().k = k;
  plan_record().nsb = nsb;
  plan_record().recompute = ep.recompute;
  Carve cv;
  Bound3 b;
  carve3(S, nsb, cv, b);
  const size_t o_vel = cv.add(host ? nvel * 4 : 0);
  const size_t o_w = cv.add(weight ? (size_t)nr * nt * 4 : 0);
  const size_t o_dobs = cv.add((size_t)ns * nt * nr * 4);  // [shot][nt][nr]
  const size_t o_dobs_in = cv.add(host ? (size_t)ns * nt * nr * 4 : 0);
  const size_t o_d = cv.add((size_t)nsb * nt * nr * 4);
  const size_t o_res = cv.add((size_t)nsb * nt * nr * 4);
  const size_t o_ck = cv.add((size_t)nsb * nck * 2 * fs * 4);
  const size_t o_tb = cv.add((size_t)nsb * k * fs * 4);
  const size_t o_ga = cv.add(fs * 4);
  const size_t o_gs = cv.add((size_t)nsb * fs * 4);  // shot slices, summed in shot order
  const size_t o_grad = cv.add(nvel * 4);
  const size_t o_mis = cv.add(8 * (1 + RESID_BLOCKS));
  const size_t o_mx = cv.add(16);
  PW_TRY(ws.reserve(cv.total()));
  plan_record().bytes = (long long)cv.total();
  char *base = ws.base();
  // checkpoints and segment terms are written before they are read
  PW_CUDA(cudaMemsetAsync(base, 0, o_ck, st));
  PW_CUDA(cudaMemsetAsync(base + o_ga, 0, cv.total() - o_ga, st));
  const float *d_vel;
  PW_TRY(upload3(S, base, b, wav, host, st));
  PW_TRY(prep_vel3(S, vel, host, base, o_vel, o_mx, b, &d_vel, st));
  float *d_w = nullptr;
  if (weight) {
    PW_TRY(to_device(base + o_w, weight, (size_t)nr * nt * 4, host, st));
    d_w = at<float>(base, o_w);
  }
  {
    const float *src = dobs;
    if (host) {
      PW_TRY(to_device(base + o_dobs_in, dobs, (size_t)ns * nt * nr * 4, true, st));
      src = at<float>(base, o_dobs_in);
    }
    for (int s = 0; s < ns; s++) {
      dim3 tb(32, 8), tg(ceil_div(nt, 32), ceil_div(nr, 32));
      pf::transpose_kernel<<<tg, tb, 0, st>>>(src + (size_t)s * nr * nt,
                                              at<float>(base, o_dobs) + (size_t)s * nt * nr, nr,
                                              nt);
    }
    PW_CUDA(cudaGetLastError());
  }
  Args p;
  bind3(S, base, b, p);
  float *gacc = at<float>(base, o_ga), *gslices = at<float>(base, o_gs);
  double *dmis = at<double>(base, o_mis);
  p.grad = gslices;
  p.gstride = (long long)fs;
  LoopTimer timer(st);
  timer.start();
  long long launches = 0;
  for (int s0 = 0; s0 < ns; s0 += nsb) {
    const int nb_ = std::min(nsb, ns - s0);
    float *A[MAXS3], *B[MAXS3];
    for (int s = 0; s < nb_; s++) {
      A[s] = at<float>(base, b.o_A) + s * fs;
      B[s] = at<float>(base, b.o_B) + s * fs;
    }
    PW_CUDA(cudaMemsetAsync(base + b.o_A, 0, (size_t)nsb * fs * 4, st));
    PW_CUDA(cudaMemsetAsync(base + b.o_B, 0, (size_t)nsb * fs * 4, st));
    p.nshots = nb_;
    p.shots = at<Shot>(base, b.o_shots) + s0;
    p.ych = plan_ych(S.g, nb_);
    float *dd = at<float>(base, o_d), *res = at<float>(base, o_res);
    float *ck = at<float>(base, o_ck), *tb = at<float>(base, o_tb);
    // ---- forward: traces, checkpoints, the last segment's terms
    p.rec = dd;
    p.tout_stride = (long long)k * fs;
    const int n_last = (nck - 1) * k;
    for (int it = 0; it < nt; it++) {
      if (it % k == 0 && it < n_last) {
        const int m = it / k;
        for (int s = 0; s < nb_; s++) {
          float *c = ck + ((size_t)s * nck + m) * 2 * fs;
          PW_CUDA(cudaMemcpyAsync(c, A[s], fs * 4, cudaMemcpyDeviceToDevice, st));
          PW_CUDA(cudaMemcpyAsync(c + fs, B[s], fs * 4, cudaMemcpyDeviceToDevice, st));
        }
      }
      p.tout = it >= n_last ? tb + (size_t)(it - n_last) * fs : nullptr;
      p.it = it;
      for (int s = 0; s < nb_; s++) {
        p.cur[s] = A[s];
        p.nxt[s] = B[s];
      }
      PW_TRY(launch3(p, FWD, st));
      launches++;
      for (int s = 0; s < nb_; s++) std::swap(A[s], B[s]);
    }
    p.rec = nullptr;
    p.tout = nullptr;
    // ---- FP64 misfit and the weighted residual
    pf::residual_kernel<<<pf::RESID_BLOCKS, 256, 0, st>>>(
        dd, at<float>(base, o_dobs) + (size_t)s0 * nt * nr, d_w, res, nb_, nt, nr, 1, dmis);
    pf::misfit_sum_kernel<<<1, 32, 0, st>>>(dmis, pf::RESID_BLOCKS);
    PW_CUDA(cudaGetLastError());
    p.res = res;
    // ---- backward by segments (the adjoint pair reuses the forward pair)
    PW_CUDA(cudaMemsetAsync(base + b.o_A, 0, (size_t)nsb * fs * 4, st));
    PW_CUDA(cudaMemsetAsync(base + b.o_B, 0, (size_t)nsb * fs * 4, st));
    float *adjA[MAXS3], *adjB[MAXS3];
    for (int s = 0; s < nb_; s++) {
      adjA[s] = at<float>(base, b.o_A) + s * fs;
      adjB[s] = at<float>(base, b.o_B) + s * fs;
    }
    p.tin_stride = (long long)k * fs;
    for (int m = nck - 1; m >= 0; m--) {
      const int n0 = m * k, n1 = std::min(nt, n0 + k);
      float *FA[MAXS3], *FB[MAXS3];
      for (int s = 0; s < nb_; s++) {
        FA[s] = ck + ((size_t)s * nck + m) * 2 * fs;
        FB[s] = FA[s] + fs;
      }
      for (int n = n0; n < n1 && m < nck - 1; n++) {  // the last segment is kept
        p.it = n;
        for (int s = 0; s < nb_; s++) {
          p.cur[s] = FA[s];
          p.nxt[s] = FB[s];
        }
        p.tout = tb + (size_t)(n - n0) * fs;
        PW_TRY(launch3(p, FWD, st));
        launches++;
        for (int s = 0; s < nb_; s++) std::swap(FA[s], FB[s]);
      }
      p.tout = nullptr;
      for (int n = n1 - 1; n >= n0; n--) {
        p.it = n;
        for (int s = 0; s < nb_; s++) {
          p.cur[s] = adjA[s];
          p.nxt[s] = adjB[s];
        }
        p.tin = tb + (size_t)(n - n0) * fs;
        PW_TRY(launch3(p, ADJ_EXACT, st));
        launches++;
        for (int s = 0; s < nb_; s++) std::swap(adjA[s], adjB[s]);
      }
    }
    p.tin = nullptr;
    {
      pf::sum_slices_kernel<<<592, 256, 0, st>>>(gslices, nb_, (long long)fs, gacc);
      PW_CUDA(cudaGetLastError());
      PW_CUDA(cudaMemsetAsync(gslices, 0, (size_t)nb_ * fs * 4, st));
      launches++;
    }
  }
  timer.stop();
  float *gdev = at<float>(base, o_grad);
  fold_grad3_kernel<<<592, 256, 0, st>>>(gacc, d_vel, a->nz, a->nx, a->ny, a->nb, S.g, gdev);
  PW_CUDA(cudaGetLastError());
  PW_TRY(to_host(grad, gdev, nvel * 4, host, st));
  if (misfit) PW_CUDA(cudaMemcpyAsync(misfit, dmis, 8, cudaMemcpyDeviceToHost, st));
  PW_CUDA(cudaStreamSynchronize(st));
  timer.finish(launches, launches + 8);
  return PW_OK;
}
