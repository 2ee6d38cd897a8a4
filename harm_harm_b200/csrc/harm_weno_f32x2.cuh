// harm_weno_f32x2.cuh -- the FP32 WENO5 weights and edge values of two cells at once on
// Blackwell's packed FP32 pipe (add/mul/fma on float2: one instruction, two lanes).
//
// The arithmetic is that of smono_indicator / weno5_cell_weights / weno3_unopt / weno_frac /
// weno5_edges for T = float (harm_device.cuh), lane by lane; operations without a packed form (reciprocals, compares,
// selects, min/max) run on each lane.  Where the scalar code branches on f > 0 (the WENO3
// blend of the stencil reduction), the packed code evaluates the blend for both lanes when
// either needs it: with f = 0 it multiplies by 1 and adds zeros, so a lane's value is the
// one its scalar branch gives (the WENO3 weights are finite: every epsilon keeps its square
// a normal FP32 number).
#pragma once
#include "harm_device.cuh"

namespace hb {

// F2 is a float2: the compiler's float2 intrinsics of the packed pipe (add, mul, fma with
// round-to-nearest; no contraction across them) let it keep the pairs in adjacent registers,
// so packing and unpacking cost no moves
using F2 = float2;

__device__ __forceinline__ F2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ F2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ void f2split(F2 x, float& a, float& b) {
  a = x.x;
  b = x.y;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 ffma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
// lane-wise helpers
template <typename Fn>
__device__ __forceinline__ F2 lanes(F2 x, Fn fn) {
  float a, b;
  f2split(x, a, b);
  return f2(fn(a), fn(b));
}
template <typename Fn>
__device__ __forceinline__ F2 lanes(F2 x, F2 y, Fn fn) {
  float a, b, c, d;
  f2split(x, a, b);
  f2split(y, c, d);
  return f2(fn(a, c), fn(b, d));
}
__device__ __forceinline__ F2 rcp2(F2 x) {
  return lanes(x, [](float a) { return __fdividef(1.0f, a); });
}

__device__ __forceinline__ F2 symsum3(F2 a0, F2 a1, F2 a2) { return (a0 + a2) + a1; }
__device__ __forceinline__ F2 symsum2(F2 a0, F2 a1) { return a0 + a1; }

// limit_weight<float> of two weights: the two ramps in the scalar code's operations on the
// packed pipe, the clamps per lane
template <int ORDER>
__device__ __forceinline__ F2 limit_weight_f2(F2 w) {
  constexpr float avg = 1.0f / (float)ORDER, w1 = 0.2f * avg, w2 = (1.0f - 0.2f) * avg, w3 = (1.0f + 0.2f) * avg,
                  w4 = 1.0f;
  const F2 lo = (f2(avg) * (w - f2(w1))) * f2(1.0f / (w2 - w1));
  const F2 up = ((w - f2(w3)) * f2(w4 - avg)) * f2(1.0f / (w4 - w3));
  return f2(fmaxf(fminf(lo.x, avg), 0.0f), fmaxf(fminf(lo.y, avg), 0.0f)) + f2(fmaxf(up.x, 0.0f), fmaxf(up.y, 0.0f));
}
__device__ __forceinline__ F2 limit_weight3_f2(F2 w) { return limit_weight_f2<3>(w); }
__device__ __forceinline__ F2 limit_weight2_f2(F2 w) { return limit_weight_f2<2>(w); }

// weno5_unopt of two cells: u points at the cells' centre values (u[-2..2])
__device__ __forceinline__ void weno5_unopt_f2(const F2* u, F2* w) {
  const F2 c3 = f2(3.0f), c4 = f2(4.0f), c2 = f2(2.0f), k13 = f2((float)(13. / 12.)), k14 = f2(0.25f);
  const F2 fd0 = (c4 * u[1]) - ffma2(c3, u[0], u[2]);
  const F2 fd1 = u[1] - u[-1];
  const F2 fd2 = ffma2(c3, u[0], u[-2]) - (c4 * u[-1]);
  const F2 sd0 = (u[0] + u[2]) - (c2 * u[1]);
  const F2 sd1 = (u[-1] + u[1]) - (c2 * u[0]);
  const F2 sd2 = (u[0] + u[-2]) - (c2 * u[-1]);
  F2 b[3];
  b[0] = ffma2(k13 * sd0, sd0, k14 * fd0 * fd0);
  b[1] = ffma2(k13 * sd1, sd1, k14 * fd1 * fd1);
  b[2] = ffma2(k13 * sd2, sd2, k14 * fd2 * fd2);
  const F2 normu = ffma2(u[0], u[0], ffma2(u[-1], u[-1], u[1] * u[1]) + ffma2(u[-2], u[-2], u[2] * u[2]));
  const F2 ee = normu * f2(WenoEps<float>::eps);
#pragma unroll
  for (int s = 0; s < 3; s++) b[s] = b[s] + ee;
  const F2 rb = rcp2(symsum3(b[0], b[1], b[2]) + f2(WenoEps<float>::tiny));
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const F2 t = ffma2(b[s], rb, f2(WenoEps<float>::weps));  // contracted, as the scalar FP32 code
    w[s] = rcp2(t * t);
  }
  const F2 r1 = rcp2(symsum3(w[0], w[1], w[2]));
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = limit_weight3_f2(w[s] * r1);
  const F2 r2 = rcp2(symsum3(w[0], w[1], w[2]));
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = w[s] * r2;
}

__device__ __forceinline__ void weno3_unopt_f2(const F2* u, F2* w) {
  const F2 fd0 = u[1] - u[0], fd1 = u[0] - u[-1];
  F2 b[2] = {fd0 * fd0, fd1 * fd1};
  const F2 normu = ffma2(u[0], u[0], ffma2(u[-1], u[-1], u[1] * u[1]));
  const F2 ee = normu * f2(WenoEps<float>::eps);
  b[0] = b[0] + ee;
  b[1] = b[1] + ee;
  const F2 rb = rcp2(symsum2(b[0], b[1]) + f2(WenoEps<float>::tiny));
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const F2 t = ffma2(b[s], rb, f2(WenoEps<float>::weps));  // contracted, as the scalar FP32 code
    w[s] = rcp2(t * t);
  }
  const F2 r1 = rcp2(symsum2(w[0], w[1]));
  w[0] = limit_weight2_f2(w[0] * r1);
  w[1] = limit_weight2_f2(w[1] * r1);
  const F2 r2 = rcp2(symsum2(w[0], w[1]));
  w[0] = w[0] * r2;
  w[1] = w[1] * r2;
}

// Weights times stencil values: eno_cvt skips zero weights; for the finite stencil values of
// finite data the product of a zero weight is a zero anyway (at most of the other sign, which
// no later sum can tell apart), so the packed path multiplies (and fuses the sums).
__device__ __forceinline__ F2 nz_mul(F2 wgt, F2 x) { return wgt * x; }

// smono_indicator<float> of two cells: the derivative combinations on the packed pipe, the
// min-mods and clamps per lane
__device__ __forceinline__ F2 smono_indicator_f2(const F2* y) {
  const F2 r12 = f2(1.0f / 12.0f), h = f2(0.5f);
  const F2 ld1 = (((f2(-3.f) * y[-2] + y[2]) + (f2(-10.f) * y[-1] - f2(6.f) * y[1])) + f2(18.f) * y[0]) * r12;
  const F2 ld2 = (((f2(11.f) * y[-2] - y[2]) + (f2(-20.f) * y[-1] + f2(4.f) * y[1])) + f2(6.f) * y[0]) * r12;
  const F2 ld3 = (((f2(-3.f) * y[-2] - y[2]) + (f2(10.f) * y[-1] + f2(6.f) * y[1])) - f2(12.f) * y[0]) * h;
  const F2 rd1 = (((y[2] * f2(3.f) - y[-2]) + (f2(6.f) * y[-1] + f2(10.f) * y[1])) - f2(18.f) * y[0]) * r12;
  const F2 rd2 = (((y[2] * f2(11.f) - y[-2]) + (f2(4.f) * y[-1] - f2(20.f) * y[1])) + f2(6.f) * y[0]) * r12;
  const F2 rd3 = (((y[-2] + f2(3.f) * y[2]) - (f2(6.f) * y[-1] + f2(10.f) * y[1])) + f2(12.f) * y[0]) * h;
  const F2 d1l = y[-1] - y[-2], d1r = y[2] - y[1];
  auto one = [](float y0, float ym1, float yp1, float ym2, float yp2, float l1, float l2, float l3, float r1, float r2,
                float r3, float dl, float dr) {
    auto mm = [](float a, float b) { return (a * b <= 0.0f) ? 0.0f : ((fabsf(a) < fabsf(b)) ? a : b); };
    l1 = mm(l1, dl);
    r1 = mm(r1, dr);
    const float minabs = fminf(fminf(fabsf(mm(l1, r1)), fabsf(mm(l2, r2))), fabsf(mm(l3, r3)));
    const float norm = fabsf(y0) + ((fabsf(ym1) + fabsf(yp1)) + (fabsf(ym2) + fabsf(yp2)));
    const float v = __fdividef(minabs, norm * WenoEps<float>::smono + WenoEps<float>::tiny);
    return fmaxf(fminf(v, 1.0f), 0.0f);
  };
  return f2(one(y[0].x, y[-1].x, y[1].x, y[-2].x, y[2].x, ld1.x, ld2.x, ld3.x, rd1.x, rd2.x, rd3.x, d1l.x, d1r.x),
            one(y[0].y, y[-1].y, y[1].y, y[-2].y, y[2].y, ld1.y, ld2.y, ld3.y, rd1.y, rd2.y, rd3.y, d1l.y, d1r.y));
}

// weno5_cell_weights<float> of two cells: (1 - m) w + m/3 is w itself for m = 0 and exactly
// 1/3 for m = 1 (finite w), so both lanes take the blend; the unoptimised weights are skipped
// when both cells are monotone
__device__ __forceinline__ void weno5_cell_weights_f2(const F2* u, F2 m, F2* w) {
  if (m.x == 1.0f && m.y == 1.0f) {
    w[0] = w[1] = w[2] = f2(1.0f / 3.0f);
    return;
  }
  weno5_unopt_f2(u, w);
  const F2 omm = f2(1.0f) - m, mt = m * f2(1.0f / 3.0f);
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = ffma2(omm, w[s], mt);
}

// weno_frac<float> of two cells
__device__ __forceinline__ F2 weno_frac_f2(const F2* w, const F2* wm, const F2* wp) {
  const F2 E = f2(WenoEps<float>::eps);
  const F2 rl = (w[2] + E) * rcp2(wm[0] + E);  // the weight ratios: a fast reciprocal per lane
  const F2 rr = (w[0] + E) * rcp2(wp[2] + E);
  const F2 ratio = lanes(rl, rr, [](float a, float b) { return fminf(a, b); });
  return lanes((ratio - f2(1.3f)) * f2(1.0f / (1.6f - 1.3f)), [](float a) { return fmaxf(0.0f, fminf(a, 1.0f)); });
}

// weno5_edges<float> of two cells from their weights w, final lower-order fractions f and
// SMONO indicators m.  (1 - m) out + m y5 is out for m = 0 and y5 for m = 1 (finite out), so
// the packed code blends both lanes; it skips the WENO sums when both cells are monotone and
// the 5-point values when neither is partly monotone.
// Offset form: every candidate edge value is the cell's value plus a combination of the
// differences d_k = u_k - u_0 (each stencil's coefficients sum to one), and the weighted
// combination is u_0 + sum_k w_k (rec_k - u_0).  In exact arithmetic this is the scalar
// code's sum_k w_k rec_k (the normalised weights sum to one); in FP32 the rounding of the
// weights' normalisation then scales only the offsets, not the cell value, so a constant
// line reconstructs to its value exactly and the reconstruction carries no bias of the
// order of that rounding times the value, which a near-steady flow would accumulate step
// after step.
__device__ __forceinline__ void weno5_edges_f2(const F2* u, const F2* w, F2 f, F2 m, F2& yl, F2& yr) {
  const F2 dm2 = u[-2] - u[0], dm1 = u[-1] - u[0], dp1 = u[1] - u[0], dp2 = u[2] - u[0];
  F2 o5l = f2(0.0f), o5r = f2(0.0f);
  if (m.x != 0.0f || m.y != 0.0f) {
    const F2 c0 = f2(-5.f / 128.f), c1 = f2(15.f / 32.f), c3 = f2(-5.f / 32.f), c4 = f2(3.f / 128.f);
    o5l = ffma2(c1, dm1, c3 * dp1) + ffma2(c0, dm2, c4 * dp2);
    o5r = ffma2(c3, dm1, c1 * dp1) + ffma2(c4, dm2, c0 * dp2);
    if (m.x >= 1.0f && m.y >= 1.0f) {
      yl = u[0] + o5l;
      yr = u[0] + o5r;
      return;
    }
  }
  F2 wl[3] = {w[0] * f2(1.f / 16.f), w[1] * f2(5.f / 8.f), w[2] * f2(5.f / 16.f)};
  F2 wr[3] = {w[0] * f2(5.f / 16.f), w[1] * f2(5.f / 8.f), w[2] * f2(1.f / 16.f)};
  const F2 nl = rcp2(symsum3(wl[0], wl[1], wl[2]) + f2(WenoEps<float>::tiny));
  const F2 nr = rcp2(symsum3(wr[0], wr[1], wr[2]) + f2(WenoEps<float>::tiny));
  float fa, fb;
  f2split(f, fa, fb);
  const bool two = (0.0f < fa) || (0.0f < fb);
  const F2 omf = f2(1.0f) - f;
#pragma unroll
  for (int s = 0; s < 3; s++) {
    wl[s] = wl[s] * nl;
    wr[s] = wr[s] * nr;
    if (two) {
      wl[s] = wl[s] * omf;
      wr[s] = wr[s] * omf;
    }
  }
  const F2 k54 = f2(-5.f / 4.f), k38 = f2(3.f / 8.f), k34 = f2(3.f / 4.f), k18 = f2(-1.f / 8.f);
  // the stencils' edge values less u_0: (15/8, -5/4, 3/8) -> -5/4 d1 + 3/8 d2, and so on
  const F2 recl0 = ffma2(k54, dp1, k38 * dp2);
  const F2 recl1 = ffma2(k38, dm1, k18 * dp1);
  const F2 recl2 = ffma2(k18, dm2, k34 * dm1);
  const F2 recr0 = ffma2(k34, dp1, k18 * dp2);
  const F2 recr1 = ffma2(k18, dm1, k38 * dp1);
  const F2 recr2 = ffma2(k38, dm2, k54 * dm1);
  auto poly3 = [](F2 k0, F2 x0, F2 k1, F2 x1, F2 k2, F2 x2) { return ffma2(k1, x1, ffma2(k0, x0, k2 * x2)); };
  F2 outl = poly3(wl[0], recl0, wl[1], recl1, wl[2], recl2);
  F2 outr = poly3(wr[0], recr0, wr[1], recr1, wr[2], recr2);
  if (two) {
    F2 w3[2];
    weno3_unopt_f2(u, w3);
    F2 l3[2] = {w3[0] * f2(0.25f), w3[1] * f2(0.75f)};
    F2 r3[2] = {w3[0] * f2(0.75f), w3[1] * f2(0.25f)};
    const F2 nl3 = rcp2(symsum2(l3[0], l3[1]) + f2(WenoEps<float>::tiny));
    const F2 nr3 = rcp2(symsum2(r3[0], r3[1]) + f2(WenoEps<float>::tiny));
#pragma unroll
    for (int s = 0; s < 2; s++) {
      l3[s] = (l3[s] * nl3) * f;
      r3[s] = (r3[s] * nr3) * f;
    }
    const F2 h = f2(0.5f), km12 = f2(-0.5f);
    // (3/2, -1/2) -> -1/2 d1; (1/2, 1/2) -> 1/2 d-1; (1/2, 1/2) -> 1/2 d1; (-1/2, 3/2) -> -1/2 d-1
    outl = outl + ffma2(l3[0], km12 * dp1, nz_mul(l3[1], h * dm1));
    outr = outr + ffma2(r3[0], h * dp1, nz_mul(r3[1], km12 * dm1));
  }
  const F2 omm = f2(1.0f) - m;
  yl = u[0] + ffma2(omm, outl, m * o5l);
  yr = u[0] + ffma2(omm, outr, m * o5r);
}

}  // namespace hb
