// harm_geometry_fp64.cu -- the metric, connection and floor tables built on the device.
//
// set_grid (set_grid.c:114) and set_connection (set_grid.c:1033) of the torus problem:
// Kerr-Schild metric in modified Kerr-Schild coordinates (KSCOORDS, LOGRSINTH coord.c:930),
//     r = R0 + exp(x1),  theta = pi x2 + (1-h)/2 sin(2 pi x2),  phi = 2 pi x3,
// the inverse metric in closed form, and the connection from central differences of the
// metric extrapolated with Ridders' method (the reference differentiates numerically as well,
// with its DIFFNUMREC scheme).  The algorithm is the host builder's (host_setup.c), operation
// for operation, compiled without FMA contraction, so the tables agree with the host's to the
// last bits of the math library (sin, cos, exp, pow).  Every record depends on (i,j) only.
//
// Kernels: k_geom_records (one thread per location and (i,j): the four metric records),
// k_geom_dg (one thread per (i,j), direction and metric component: Ridders' extrapolated
// derivative), k_geom_conn (one thread per (i,j): the connection and the floor table).
#include <math.h>
#include "harm_common.cuh"
#include "harm_paths.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSingSmall = 1e-13;  // COORDSINGFIX offset from the poles
constexpr double kSmallD = 1e-300;

struct GridC {
  double a, hslope, R0, startx1, startx2, dx1, dx2, rho_floor_coef, u_floor_coef;
  int ng, n1e, n2e;
  size_t plane;
};

__device__ __forceinline__ int symi(int m, int n) {
  return (m <= n) ? ((m == 0) ? n : (m == 1) ? 3 + n : (m == 2) ? 5 + n : 9)
                  : ((n == 0) ? m : (n == 1) ? 3 + m : (n == 2) ? 5 + m : 9);
}

// Boyer-Lindquist theta of x2: both branches of coord.c:953-959, COORDSINGFIX clamp
__device__ double theta_of_x2(const GridC& g, double x2) {
  double th;
  if (x2 < 0.5)
    th = kPi * x2 + 0.5 * (1.0 - g.hslope) * sin(2.0 * kPi * x2);
  else
    th = kPi - kPi * (1.0 - x2) - 0.5 * (1.0 - g.hslope) * sin(2.0 * kPi * (1.0 - x2));
  if (fabs(th) < kSingSmall) th = (th >= 0) ? kSingSmall : -kSingSmall;
  if (fabs(kPi - th) < kSingSmall) th = (th >= kPi) ? kPi + kSingSmall : kPi - kSingSmall;
  return th;
}

__device__ double dthdx2(const GridC& g, double x2) {
  if (x2 < 0.5) return kPi + (1.0 - g.hslope) * kPi * cos(2.0 * kPi * x2);
  return kPi + (1.0 - g.hslope) * kPi * cos(2.0 * kPi * (1.0 - x2));
}

// the Kerr-Schild quantities of a point
struct KS {
  double r, s2, rho2, z, d[4];
};
__device__ KS ks_at(const GridC& g, double x1, double x2, double& sth) {
  KS k;
  k.r = g.R0 + exp(x1);
  const double th = theta_of_x2(g, x2);
  const double cth = cos(th);
  sth = sin(th);
  k.s2 = sth * sth;
  k.rho2 = k.r * k.r + g.a * g.a * cth * cth;
  k.z = 2.0 * k.r / k.rho2;
  k.d[0] = 1.0;
  k.d[1] = k.r - g.R0;
  k.d[2] = dthdx2(g, x2);
  k.d[3] = 2.0 * kPi;
  return k;
}

// entry (m, n) of the Kerr-Schild metric before the coordinate factors
__device__ double ks_k(const GridC& g, const KS& k, int m, int n) {
  const double a = g.a;
  const int lo = m < n ? m : n, hi = m < n ? n : m;
  if (lo == 0 && hi == 0) return -1.0 + k.z;
  if (lo == 0 && hi == 1) return k.z;
  if (lo == 0 && hi == 3) return -k.z * a * k.s2;
  if (lo == 1 && hi == 1) return 1.0 + k.z;
  if (lo == 1 && hi == 3) return -a * k.s2 * (1.0 + k.z);
  if (lo == 2 && hi == 2) return k.rho2;
  if (lo == 3 && hi == 3) return k.s2 * (k.rho2 + a * a * k.s2 * (1.0 + k.z));
  return 0.0;
}

// g_{mn} in MKS coordinates (the product in the host builder's order: k d_m d_n)
__device__ double gcov_mn(const GridC& g, double x1, double x2, int m, int n) {
  double sth;
  const KS k = ks_at(g, x1, x2, sth);
  return ks_k(g, k, m, n) * k.d[m] * k.d[n];
}

// one location record: gcov, gcon (closed form), lapse, shift, sqrt(-g)
__device__ void metric_record(const GridC& g, double x1, double x2, double* rec) {
  double sth;
  const KS k = ks_at(g, x1, x2, sth);
  const double a = g.a, r = k.r, rho2 = k.rho2, z = k.z;
  double kc[4][4];
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) kc[m][n] = 0.0;
  kc[0][0] = -(1.0 + z);
  kc[0][1] = kc[1][0] = z;
  kc[1][1] = (r * r - 2.0 * r + a * a) / rho2;
  kc[1][3] = kc[3][1] = a / rho2;
  kc[2][2] = 1.0 / rho2;
  kc[3][3] = 1.0 / (rho2 * k.s2);
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = m; n < 4; n++) {
      rec[HARM_G_GCOV + symi(m, n)] = ks_k(g, k, m, n) * k.d[m] * k.d[n];
      rec[HARM_G_GCON + symi(m, n)] = kc[m][n] / (k.d[m] * k.d[n]);
    }
  rec[HARM_G_GCOVPERT_TT] = z;
  const double alpha = 1.0 / sqrt(fabs(rec[HARM_G_GCON + 0]));
  rec[HARM_G_ALPHA] = alpha;
  double bsq = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) bsq += rec[HARM_G_GCOV + symi(0, j)] * rec[HARM_G_GCON + symi(0, j)];
  rec[HARM_G_BETASQOALPHASQ] = bsq;
#pragma unroll
  for (int j = 1; j < 4; j++) rec[HARM_G_BETA + j - 1] = rec[HARM_G_GCON + symi(0, j)] * alpha * alpha;
  const double gdet = rho2 * fabs(sth) * k.d[1] * k.d[2] * k.d[3];
  rec[HARM_G_GDET] = gdet;
  rec[HARM_G_IGDET] = ((gdet > 0) - (gdet < 0)) / (fabs(gdet) + kSmallD);
}

__device__ __forceinline__ void cell_x(const GridC& g, size_t c, int loc, double& x1, double& x2) {
  const int jj = (int)(c / g.n1e), ii = (int)(c % g.n1e);
  const int i = ii - g.ng, j = jj - g.ng;
  const bool f1 = (loc == HARM_LOC_FACE1 || loc == HARM_LOC_CORN3);
  const bool f2 = (loc == HARM_LOC_FACE2 || loc == HARM_LOC_CORN3);
  x1 = f1 ? g.startx1 + i * g.dx1 : g.startx1 + (i + 0.5) * g.dx1;
  x2 = f2 ? g.startx2 + j * g.dx2 : g.startx2 + (j + 0.5) * g.dx2;
}

__global__ void k_geom_records(GridC g, double* __restrict__ geom) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)HARM_NLOC * g.plane) return;
  const int loc = (int)(t / g.plane);
  const size_t c = t % g.plane;
  double x1, x2;
  cell_x(g, c, loc, x1, x2);
  double rec[HARM_NGF];
  metric_record(g, x1, x2, rec);
#pragma unroll
  for (int f = 0; f < HARM_NGF; f++) geom[((size_t)loc * HARM_NGF + f) * g.plane + c] = rec[f];
}

// d g_{mn} / d x^dir at the cell centre (dir 1 or 2) by Ridders' polynomial extrapolation of
// central differences (initial step 0.2 dx, step ratio 1.4, at most 10 steps, stop when the
// error grows); dg[(dir-1)*16 + m*4 + n][c]
__global__ void k_geom_dg(GridC g, double* __restrict__ dg) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)32 * g.plane) return;
  const int comp = (int)(t / g.plane);
  const size_t c = t % g.plane;
  const int dir = 1 + comp / 16, m = (comp % 16) / 4, n = comp % 4;
  double x1, x2;
  cell_x(g, c, HARM_LOC_CENT, x1, x2);
  constexpr int NTAB = 10;
  const double CON = 1.4, CON2 = CON * CON, SAFE = 2.0;
  double hh = (dir == 1) ? 0.01 * g.dx1 * 20.0 : 0.01 * g.dx2 * 20.0;
  double prev[NTAB], cur[NTAB];
  double err = 1e300, ans = 0.0;
  for (int it = 0; it < NTAB; it++) {
    const double gp = (dir == 1) ? gcov_mn(g, x1 + hh, x2, m, n) : gcov_mn(g, x1, x2 + hh, m, n);
    const double gm = (dir == 1) ? gcov_mn(g, x1 - hh, x2, m, n) : gcov_mn(g, x1, x2 - hh, m, n);
    cur[0] = (gp - gm) / (2.0 * hh);
    if (it == 0) {
      ans = cur[0];
      hh /= CON;
      prev[0] = cur[0];
      continue;
    }
    double fac = CON2;
    for (int j = 1; j <= it; j++) {
      cur[j] = (cur[j - 1] * fac - prev[j - 1]) / (fac - 1.0);
      fac *= CON2;
      const double errt = fmax(fabs(cur[j] - cur[j - 1]), fabs(cur[j] - prev[j - 1]));
      if (errt <= err) {
        err = errt;
        ans = cur[j];
      }
    }
    if (fabs(cur[it] - prev[it - 1]) >= SAFE * err) break;
    hh /= CON;
    for (int q = 0; q <= it; q++) prev[q] = cur[q];
  }
  dg[(size_t)comp * g.plane + c] = ans;
}

// Gamma^k_{l j} = 1/2 g^{k m} (d_j g_{m l} + d_l g_{m j} - d_m g_{l j}); the floors
__global__ void k_geom_conn(GridC g, const double* __restrict__ geom, const double* __restrict__ dgt,
                            double* __restrict__ conn, double* __restrict__ aux) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.plane) return;
  auto dg = [&](int l, int m, int n) -> double {
    return (l == 1 || l == 2) ? dgt[(size_t)((l - 1) * 16 + m * 4 + n) * g.plane + c] : 0.0;
  };
  double gcon[4][4];
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) gcon[m][n] = geom[(size_t)(HARM_LOC_CENT * HARM_NGF + HARM_G_GCON + symi(m, n)) * g.plane + c];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++)
      for (int j = 0; j < 4; j++) {
        double s = 0.0;
        for (int m = 0; m < 4; m++) s += gcon[k][m] * (dg(j, m, l) + dg(l, m, j) - dg(m, l, j));
        conn[(size_t)((k * 4 + l) * 4 + j) * g.plane + c] = 0.5 * s;
      }
  double x1, x2;
  cell_x(g, c, HARM_LOC_CENT, x1, x2);
  const double r = g.R0 + exp(x1);
  aux[(size_t)HARM_AUX_R * g.plane + c] = r;
  aux[(size_t)HARM_AUX_RHOFLOOR * g.plane + c] = g.rho_floor_coef * pow(r, -1.5);
  aux[(size_t)HARM_AUX_UFLOOR * g.plane + c] = g.u_floor_coef * pow(r, -2.5);
}

__global__ void k_geom_to_f32(size_t n, const double* __restrict__ src, float* __restrict__ dst) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (float)src[t];
}

}  // namespace

// The FP32 copy of the metric tables used by the mixed path's flux kernels.
int hp_geometry_f32(harm_ctx* c) {
  const size_t n = (size_t)HARM_NLOC * HARM_NGF * c->plane;
  k_geom_to_f32<<<nblk((long long)n), 256, 0, c->stream>>>(n, c->d_geom, c->d_geomf);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// The context's metric (d_geom), connection (d_conn) and floor (d_aux) tables from its grid.
int hp_geometry_build(harm_ctx* c) {
  const harm_grid& hg = c->g;
  GridC g;
  g.a = hg.a;
  g.hslope = hg.hslope;
  g.R0 = hg.R0;
  g.startx1 = hg.startx[1];
  g.startx2 = hg.startx[2];
  g.dx1 = hg.dx[1];
  g.dx2 = hg.dx[2];
  g.rho_floor_coef = hg.rho_floor_coef;
  g.u_floor_coef = hg.u_floor_coef;
  g.ng = hg.ng;
  g.n1e = hg.n1e;
  g.n2e = hg.n2e;
  g.plane = (size_t)hg.n1e * hg.n2e;
  double* dg = nullptr;
  CK(cudaMalloc(&dg, (size_t)32 * g.plane * sizeof(double)));
  k_geom_records<<<nblk((long long)HARM_NLOC * g.plane), 256, 0, c->stream>>>(g, c->d_geom);
  k_geom_dg<<<nblk((long long)32 * g.plane, 128), 128, 0, c->stream>>>(g, dg);
  k_geom_conn<<<nblk((long long)g.plane, 128), 128, 0, c->stream>>>(g, c->d_geom, dg, c->d_conn, c->d_aux);
  c->launches += 3;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(dg);
  if (e != cudaSuccess) return hb_seterr("device geometry build", e);
  return 0;
}
