// harm_dump_fp64.cu -- the reference's main dump file written from device state.
//
// dump() (dump.c:256) through dump_gen (dumpgen.c:5): a header (dump_header_general,
// dump.c:320) and, for every active cell in the order k, j, i (i fastest; DUMPLOOP,
// global.loops.diagnostics.h:15), the 52 columns of dump_content (dump.c:449) with
// CALCFARADAYANDCURRENTS = 0:
//    ti tj tk | x1 x2 x3 | r th ph | rho u v1 v2 v3 B1 B2 B3 | p cs2 Sden | U0..U7 | divb |
//    uu0..uu3 | ud0..ud3 | bu0..bu3 | bd0..bd3 | v1m v1p v2m v2p v3m v3p | gdet
// Formats (dump_gen's bintxt): TEXT -- the header line of "%21.15g"/"%d"/"%ld" fields and one
// line per cell of "%21.15g " columns (myfwrite, mpi_fileio.c:2316); BINARY -- the header
// as raw fields (no defcoord) and raw doubles; MIXED -- the text header and raw doubles.
// The columns are computed on the device (FP64, without FMA contraction, in the reference's
// order of operations) a k-slab at a time and written by the host.
#include <stdio.h>
#include <algorithm>
#include <vector>
#include "harm_common.cuh"
#include "harm_paths.h"

int hb_setmsg(const char* msg, int code);

namespace {

constexpr int kDumpCols = 52;
constexpr double kPiD = 3.14159265358979323846;
constexpr double kSmallD = 1e-300;  // SMALL (global.depnmemonics.h:493)
constexpr double kBigD = 1e100;     // BIG

struct DumpC {
  double startx1, startx2, startx3, dx1, dx2, dx3, R0, hslope, gam;
};

// bl_coord (coord.c:930, LOGRSINTH): r, theta, phi of MKS (x1, x2, x3)
__device__ void bl_coord_v(const DumpC& c, const double* X, double* V) {
  V[1] = c.R0 + exp(X[1]);
  if (X[2] < 0.5)
    V[2] = kPiD * X[2] + ((1. - c.hslope) / 2.) * sin(2. * kPiD * X[2]);
  else
    V[2] = kPiD - (kPiD * (1.0 - X[2])) + ((1. - c.hslope) / 2.) * (-sin(2. * kPiD * (1.0 - X[2])));
  V[3] = 2.0 * kPiD * X[3];
}

// compute_entropy_simple (phys.tools.c:3212) with the ideal gas (idealgaseos.c:71)
__device__ double entropy_simple(double rho0, double u, double gam) {
  if (rho0 < kSmallD) rho0 = kSmallD;
  if (u < kSmallD) u = kSmallD;
  double pressure = (gam - 1.0) * u;
  const double indexn = 1.0 / (gam - 1.0);
  double entropy;
  if (rho0 < kSmallD && pressure < kSmallD) {
    entropy = 0.0;
  } else if (rho0 < kSmallD) {
    entropy = 0.0;
  } else if (pressure < kSmallD) {
    entropy = -kBigD;
  } else {
    entropy = rho0 * log(pow(pressure, indexn) / pow(rho0, indexn + 1.0));
  }
  if (!isfinite(entropy)) entropy = -kBigD * fmax(rho0, kSmallD);
  return entropy;
}

__global__ void k_dump_cols(Dims d, DumpC c, const double* __restrict__ P, const double* __restrict__ U,
                            const double* __restrict__ geom, int k0, int nk, double* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)d.n1 * d.n2 * nk;
  if (t >= n) return;
  const int i = (int)(t % d.n1);
  const long long r = t / d.n1;
  const int j = (int)(r % d.n2), k = k0 + (int)(r / d.n2);
  const int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
  Geo<double> g;
  load_geo<double, double>(geom, d.plane, c2, g);
  double pr[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) pr[p] = P[(size_t)p * d.cells + id];
  double* o = out + (size_t)t * kDumpCols;
  int col = 0;
  o[col++] = (double)i;
  o[col++] = (double)j;
  o[col++] = (double)k;
  double X[4], V[4];
  X[0] = 0.0;
  X[1] = c.startx1 + (i + 0.5) * c.dx1;
  X[2] = c.startx2 + (j + 0.5) * c.dx2;
  X[3] = c.startx3 + (k + 0.5) * c.dx3;
  bl_coord_v(c, X, V);
  for (int q = 1; q <= 3; q++) o[col++] = X[q];
  for (int q = 1; q <= 3; q++) o[col++] = V[q];
  for (int p = 0; p < NPR; p++) o[col++] = pr[p];
  const double rho = pr[HARM_RHO], u = pr[HARM_UU];
  const double pressure = (c.gam - 1.0) * u;
  const double h = rho + u + pressure;
  o[col++] = pressure;
  o[col++] = c.gam * pressure / h;
  o[col++] = entropy_simple(rho, u, c.gam);
  State<double> q;
  get_state<double>(pr, g, c.gam, q);
  if (U) {
    for (int p = 0; p < NPR; p++) o[col++] = U[(size_t)p * d.cells + id];
  } else {
    double Uc[NPR];
    primtoflux<double>(pr, q, 0, g, g.gdet, Uc);
    for (int p = 0; p < NPR; p++) o[col++] = Uc[p];
  }
  // divb: SETFDIVBFLUXCTTOTHPRIM (global.fieldmacros.h:383), the corner divergence of
  // gdet B at (i-1/2, j-1/2, k-1/2) normalised by the field's own gradients
  {
    const bool has3 = d.n3 > 1;
    auto Fg = [&](int a, int b, int e, int pl) -> double {
      return P[(size_t)pl * d.cells + cidx(d, a, b, e)] * __ldg(geom + (size_t)HARM_G_GDET * d.plane + (size_t)b * d.n1e + a);
    };
    auto aFg = [&](int a, int b, int e, int pl) -> double { return fabs(Fg(a, b, e, pl)); };
    const int km = has3 ? kk - 1 : kk;
    auto avg1 = [&](auto F, int a, int b, int e, int pl) { return 0.5 * (F(a, b, e, pl) + F(a - 1, b, e, pl)); };
    auto avg2 = [&](auto F, int a, int b, int e, int pl) { return 0.5 * (F(a, b, e, pl) + F(a, b - 1, e, pl)); };
    auto for1 = [&](auto F, int a, int b, int e) {
      const int em = has3 ? e - 1 : e;
      return 0.5 * (avg2(F, a, b, e, HARM_B1) + avg2(F, a, b, em, HARM_B1));
    };
    auto for2 = [&](auto F, int a, int b, int e) {
      const int em = has3 ? e - 1 : e;
      return 0.5 * (avg1(F, a, b, e, HARM_B2) + avg1(F, a, b, em, HARM_B2));
    };
    auto for3 = [&](auto F, int a, int b, int e) {
      return 0.5 * (avg2(F, a, b, e, HARM_B3) + avg2(F, a - 1, b, e, HARM_B3));
    };
    const double D1 = for1(Fg, ii, jj, kk) - for1(Fg, ii - 1, jj, kk);
    const double D2 = for2(Fg, ii, jj, kk) - for2(Fg, ii, jj - 1, kk);
    const double D3 = for3(Fg, ii, jj, kk) - for3(Fg, ii, jj, km);
    const double N1 = for1(aFg, ii, jj, kk) + for1(aFg, ii - 1, jj, kk);
    const double N2 = for2(aFg, ii, jj, kk) + for2(aFg, ii, jj - 1, kk);
    const double N3 = for3(aFg, ii, jj, kk) + for3(aFg, ii, jj, km);
    const double norm = 1.0 / (fabs(N1 / c.dx1 + N2 / c.dx2 + N3 / c.dx3) + kSmallD);
    o[col++] = fabs((D1 / c.dx1 + D2 / c.dx2 + D3 / c.dx3) * norm);
  }
  double bcon[4], bcov[4];
  bcon[0] = pr[HARM_B1] * q.ucov[1] + pr[HARM_B2] * q.ucov[2] + pr[HARM_B3] * q.ucov[3];
  for (int m = 1; m <= 3; m++) bcon[m] = (pr[HARM_B1 - 1 + m] + bcon[0] * q.ucon[m]) / q.ucon[0];
  lower<double>(bcon, g, bcov);
  for (int m = 0; m < 4; m++) o[col++] = q.ucon[m];
  for (int m = 0; m < 4; m++) o[col++] = q.ucov[m];
  for (int m = 0; m < 4; m++) o[col++] = bcon[m];
  for (int m = 0; m < 4; m++) o[col++] = bcov[m];
  for (int dir = 1; dir <= 3; dir++) {
    double vmax, vmin;
    vchar<double>(pr, q, dir, g, c.gam, vmax, vmin);
    o[col++] = vmin;
    o[col++] = vmax;
  }
  o[col++] = g.gdet;
}

}  // namespace

// dump.c's file from device state (see the top of this file): d_P with bounded ghost zones;
// d_U the conserved state to record (NULL: primtoU of d_P).
extern "C" int harm_b200_dump(harm_ctx* c, const double* d_P, const double* d_U, double t, double dt, long nstep,
                              int format, const char* path) {
  if (!c || !d_P || !path) return hb_setmsg("null argument", 1);
  if (format != HARM_DUMP_TEXT && format != HARM_DUMP_BINARY && format != HARM_DUMP_MIXED)
    return hb_setmsg("unknown dump format", 2);
  const harm_grid& hg = c->g;
  Dims d = dims_of(hg);
  DumpC dc;
  dc.startx1 = hg.startx[1];
  dc.startx2 = hg.startx[2];
  dc.startx3 = hg.startx[3];
  dc.dx1 = hg.dx[1];
  dc.dx2 = hg.dx[2];
  dc.dx3 = hg.dx[3];
  dc.R0 = hg.R0;
  dc.hslope = hg.hslope;
  dc.gam = hg.gam;
  FILE* fp = fopen(path, "wb");
  if (!fp) return hb_setmsg("cannot open the dump file", 4);
  // dump_header_general (dump.c:320): is..ke the evolved range 0..N-1 (initbase.c:2285)
  const int tot1 = hg.n1, tot2 = hg.n2, tot3 = hg.n3, is = 0, ie = hg.n1 - 1, js = 0, je = hg.n2 - 1, ks = 0,
            ke = hg.n3 - 1, whichdump = 3 /* MAINDUMPTYPE */, version = 0, ncol = kDumpCols, defcoord = 0 /* LOGRSINTH */;
  const double MBH = 1.0, QBH = 0.0;
  if (format == HARM_DUMP_BINARY) {
    auto wd = [&](double v) { fwrite(&v, sizeof(double), 1, fp); };
    auto wi = [&](int v) { fwrite(&v, sizeof(int), 1, fp); };
    wd(t);
    wi(tot1); wi(tot2); wi(tot3);
    wd(hg.startx[1]); wd(hg.startx[2]); wd(hg.startx[3]);
    wd(hg.dx[1]); wd(hg.dx[2]); wd(hg.dx[3]);
    fwrite(&nstep, sizeof(long), 1, fp);
    wd(hg.gam); wd(hg.a); wd(hg.R0); wd(hg.Rin); wd(hg.Rout); wd(hg.hslope); wd(dt); wd(MBH); wd(QBH);
    wi(is); wi(ie); wi(js); wi(je); wi(ks); wi(ke); wi(whichdump); wi(version); wi(ncol);
  } else {
    fprintf(fp,
            "%21.15g %d %d %d %21.15g %21.15g %21.15g %21.15g %21.15g %21.15g %ld %21.15g %21.15g %21.15g %21.15g "
            "%21.15g %21.15g %21.15g %d %21.15g %21.15g %d %d %d %d %d %d %d %d %d\n",
            t, tot1, tot2, tot3, hg.startx[1], hg.startx[2], hg.startx[3], hg.dx[1], hg.dx[2], hg.dx[3], nstep, hg.gam,
            hg.a, hg.R0, hg.Rin, hg.Rout, hg.hslope, dt, defcoord, MBH, QBH, is, ie, js, je, ks, ke, whichdump, version,
            ncol);
  }
  // the columns, a slab of k-planes at a time (at most ~64 MB of columns per slab)
  const long long per_k = (long long)d.n1 * d.n2;
  int nk = (int)std::max<long long>(1, (64ll << 20) / (per_k * kDumpCols * 8));
  nk = std::min(nk, d.n3);
  double* d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_out, (size_t)per_k * nk * kDumpCols * sizeof(double));
  if (e != cudaSuccess) {
    fclose(fp);
    return hb_seterr("dump buffer", e);
  }
  std::vector<double> h((size_t)per_k * nk * kDumpCols);
  int rc = 0;
  for (int k0 = 0; k0 < d.n3 && rc == 0; k0 += nk) {
    const int nkk = std::min(nk, d.n3 - k0);
    const long long n = per_k * nkk;
    k_dump_cols<<<nblk(n), 256, 0, c->stream>>>(d, dc, d_P, d_U, c->d_geom, k0, nkk, d_out);
    c->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_out, (size_t)n * kDumpCols * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      rc = hb_seterr("dump columns", e);
      break;
    }
    if (format == HARM_DUMP_TEXT) {
      for (long long s = 0; s < n; s++) {
        const double* row = h.data() + (size_t)s * kDumpCols;
        for (int q = 0; q < kDumpCols; q++) fprintf(fp, "%21.15g ", row[q]);
        fprintf(fp, "\n");
      }
    } else {
      if (fwrite(h.data(), sizeof(double), (size_t)n * kDumpCols, fp) != (size_t)n * kDumpCols) rc = hb_setmsg("dump write failed", 4);
    }
  }
  cudaFree(d_out);
  if (fclose(fp) != 0 && rc == 0) rc = hb_setmsg("dump write failed", 4);
  return rc;
}
