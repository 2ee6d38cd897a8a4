/*
 * driver.c -- driver that runs the reference HARM code itself (built from the reference's
 * own sources by oracle/ref/build.sh into oracle/_ref/) and writes what it computes as .npy
 * files.  TEST INFRASTRUCTURE ONLY: tests and the benchmark's CPU baseline run the binaries
 * this file is linked into as the checker; nothing in the product loads or calls them.
 *
 * It replaces the reference's main() (main.c:6), which would run its diagnostics and its own
 * time loop, by one that calls init() (initbase.c:7), then step_ch_full() (step_ch.c:35) step
 * by step, writing the state in between.  The torus problem's init_defcoord, init_grid and
 * init_global (initboundcode/init.fishmon.c:179,194,228) are renamed by the build recipe to
 * href_fishmon_*; the functions of the same names below call them and then apply the run
 * configuration of this build (modified Kerr-Schild LOGRSINTH coordinates with hslope 0.3,
 * R0 0, Rout 40; Toth flux-CT; rescaletype 0 floors 1e-6 r^-1.5 / 1e-8 r^-2.5; Courant 0.8;
 * fixed seed of the internal-energy perturbation; no diagnostics), with the reconstruction,
 * flux formula, time order and Courant factor taken from the environment:
 *   HREF_LIM        mc | para | paraline | weno5 | weno5bnd   (lim[1..3], default mc;
 *                   weno5 is lim WENO5, weno5bnd lim WENO5BND)
 *   HREF_FLUX       hll | laxf                          (fluxmethod, default hll)
 *   HREF_TIMEORDER  1 | 2 | 3 | 4                       (TIMEORDER, default 2: setup_rktimestep's
 *                                                        Euler, RK2 midpoint, TVD RK3, RK4)
 *   HREF_COUR       Courant factor                      (default 0.8)
 *   HREF_SEED       seed of ranc() for the perturbation (default 12345)
 *
 * Usage (the working directory receives the reference's own log files):
 *   harm_ref_<cfg> run    <outdir> <nthreads> <nsteps> <dumpevery>
 *       writes geom.npy conn.npy aux.npy (metric records of every (i,j) of the extended
 *       grid at k=0), p0.npy (t=0 state), p_<step>.npy every `dumpevery` steps and after the
 *       last, steps.npy (t, dt, nstroke per step) and grid.npy (grid parameters); for the
 *       steps listed in HREF_SUBSTEP_STEPS also every substep's advance() inputs and outputs
 *       (sub_<step>_<timeorder>_{pi,pb,pf,pflag,args,ndt}), its fluxcalc() fluxes
 *       (_F1,_F2,_F3,_ndtdir) and post_fixup()'s input and output (_fixin,_fixflag,_fixout),
 *       and every per-direction boundary call's input and output (bnd_<step>_<n>_{in,out,info}),
 *       as extended arrays [k][j][i][pl] with the ghost zones
 *   harm_ref_<cfg> points <outdir> <nthreads> <infile>
 *       Utoprimgen (utoprimgen.c:32) of every record of <infile> (raw doubles: i, j, U[8],
 *       guess P[8]; U in UEVOLVE form at CENT of cell (i,j,0)); writes points.npy with
 *       P[8], pflag and the Newton iteration count of each record
 *   harm_ref_<cfg> fixup  <outdir> <nthreads> <infile> [finalstep]
 *       post_fixup (fixup.c:53, with its bound_pflag and fixup_utoprim) of a given state on
 *       the final substep (finalstep 1, the default) or an earlier one (0):
 *       <infile> holds the extended primitive state [k][j][i][pl] (raw doubles, ghost zones
 *       filled by the caller) followed by the failure flag of every active cell [k][j][i]
 *       (raw doubles); writes fixout.npy (the extended state afterwards) and fixflag.npy
 *       (the extended flags afterwards)
 *   harm_ref_<cfg> time   <outdir> <nthreads> <nsteps>
 *       times <nsteps> full steps on <nthreads> OpenMP threads; writes time.npy
 *       (zone-cycles/s, seconds, steps, cells)
 */
/* defs.h, as in the reference main.c, defines the reference's global variables */
#include "defs.h"
#include <omp.h>
#include <sys/stat.h>
#include <sys/time.h>

int href_fishmon_init_defcoord(void);
int href_fishmon_init_grid(void);
int href_fishmon_init_global(void);

/* The reference's main.c also holds gocheck(), which polls the go.cont and go.go files of a
   run directory (continue from a restart, stop a running job).  This driver restarts
   nothing and is stopped by its step count, so the check does nothing here. */
int gocheck(int whichlocation)
{
  (void)whichlocation;
  return 0;
}

static const char *env_or(const char *name, const char *def)
{
  const char *s = getenv(name);
  return (s && *s) ? s : def;
}

int init_defcoord(void)
{
  int r = href_fishmon_init_defcoord();
  defcoord = LOGRSINTH;
  return r;
}

int init_grid(void)
{
  int r = href_fishmon_init_grid();
  R0 = 0.0;
  Rout = 40.0;
  hslope = 0.3;
  Rhor = rhor_calc(0);
  setRin_withchecks(&Rin);
  return r;
}

int init_global(void)
{
  int r = href_fishmon_init_global();
  int dir;
  const char *lim_s = env_or("HREF_LIM", "mc");
  int limv = MC;
  if (!strcmp(lim_s, "para")) limv = PARA;
  else if (!strcmp(lim_s, "paraline")) limv = PARALINE;
  else if (!strcmp(lim_s, "weno5")) limv = WENO5;
  else if (!strcmp(lim_s, "weno5bnd")) limv = WENO5BND;
  for (dir = 1; dir <= 3; dir++) lim[dir] = limv;
  fluxmethod = strcmp(env_or("HREF_FLUX", "hll"), "laxf") ? HLLFLUX : LAXFFLUX;
  FLUXB = FLUXCTTOTH;
  TIMEORDER = atoi(env_or("HREF_TIMEORDER", "2"));
  cour = atof(env_or("HREF_COUR", "0.8"));
  rescaletype = 0;
  prfloorcoef[RHO] = 1e-6;
  prfloorcoef[UU] = 1e-8;
  DODIAGS = 0;
  tf = 1e30;
  DTr = 1000000000;
  ranc(1, atoi(env_or("HREF_SEED", "12345")));
  return r;
}

/* ---- .npy writer (format version 1.0, little-endian, C order) ---- */
static void write_npy(const char *dir, const char *name, const char *descr, const void *data,
                      size_t elsize, int ndim, const long *shape)
{
  char path[4096], hdr[256], shp[160] = "";
  size_t n = 1, hl, pad;
  int d;
  FILE *f;
  for (d = 0; d < ndim; d++) {
    char t[32];
    snprintf(t, sizeof t, "%ld%s", shape[d], (ndim == 1) ? "," : (d + 1 < ndim ? ", " : ""));
    strcat(shp, t);
    n *= (size_t)shape[d];
  }
  snprintf(hdr, sizeof hdr, "{'descr': '%s', 'fortran_order': False, 'shape': (%s), }", descr, shp);
  hl = strlen(hdr);
  pad = 64 - (10 + hl + 1) % 64;
  if (pad == 64) pad = 0;
  snprintf(path, sizeof path, "%s/%s", dir, name);
  f = fopen(path, "wb");
  if (!f) { fprintf(stderr, "ref_driver: cannot write %s\n", path); exit(3); }
  {
    unsigned short hlen = (unsigned short)(hl + pad + 1);
    fwrite("\x93NUMPY\x01\x00", 1, 8, f);
    fwrite(&hlen, 2, 1, f);
    fwrite(hdr, 1, hl, f);
    for (; pad > 0; pad--) fputc(' ', f);
    fputc('\n', f);
  }
  fwrite(data, elsize, n, f);
  fclose(f);
}

/* state of the active cells in the reference's order [k][j][i][pl] */
static void dump_state(const char *dir, const char *name)
{
  long shape[4] = {N3, N2, N1, NPR};
  double *buf = (double *)malloc(sizeof(double) * N1 * N2 * N3 * NPR);
  size_t o = 0;
  int i, j, k, pl;
  for (k = 0; k < N3; k++)
    for (j = 0; j < N2; j++)
      for (i = 0; i < N1; i++)
        for (pl = 0; pl < NPR; pl++) buf[o++] = GLOBALMACP0A1(pglobal, i, j, k, pl);
  write_npy(dir, name, "<f8", buf, sizeof(double), 4, shape);
  free(buf);
}

/* metric records of every (i,j) of the extended grid at k=0, all NPG locations, in the
   field order of harm_b200.h (gcov[10] gcon[10] gcovpert_tt alpha betasqoalphasq beta[3]
   gdet igdetnosing); conn[64] at CENT; aux: Boyer-Lindquist r and the two floors */
static void dump_geometry(const char *dir)
{
  const int n1e = N1 + 2 * N1BND, n2e = N2 + 2 * N2BND;
  long gshape[4] = {NPG, 28, n2e, n1e};
  long cshape[3] = {64, n2e, n1e};
  long ashape[3] = {3, n2e, n1e};
  double *g = (double *)calloc((size_t)NPG * 28 * n2e * n1e, sizeof(double));
  double *c = (double *)calloc((size_t)64 * n2e * n1e, sizeof(double));
  double *a = (double *)calloc((size_t)3 * n2e * n1e, sizeof(double));
  int ii, jj, loc, m, n, f, p, q, s;
  for (jj = 0; jj < n2e; jj++)
    for (ii = 0; ii < n1e; ii++) {
      int i = ii - N1BND, j = jj - N2BND, k = 0;
      size_t cell = (size_t)jj * n1e + ii;
      for (loc = 0; loc < NPG; loc++) {
        struct of_geom geomdontuse, *ptrgeom = &geomdontuse;
        double *rec = g + (size_t)loc * 28 * n2e * n1e + cell;
        get_geometry(i, j, k, loc, ptrgeom);
        f = 0;
        for (m = 0; m < 4; m++)
          for (n = m; n < 4; n++) rec[(size_t)(f++) * n2e * n1e] = ptrgeom->gcov[GIND(m, n)];
        for (m = 0; m < 4; m++)
          for (n = m; n < 4; n++) rec[(size_t)(f++) * n2e * n1e] = ptrgeom->gcon[GIND(m, n)];
        rec[(size_t)(f++) * n2e * n1e] = ptrgeom->gcovpert[TT];
        rec[(size_t)(f++) * n2e * n1e] = ptrgeom->alphalapse;
        rec[(size_t)(f++) * n2e * n1e] = ptrgeom->betasqoalphasq;
        for (m = 1; m <= 3; m++) rec[(size_t)(f++) * n2e * n1e] = ptrgeom->beta[m];
        rec[(size_t)(f++) * n2e * n1e] = ptrgeom->gdet;
        rec[(size_t)(f++) * n2e * n1e] = ptrgeom->igdetnosing;
      }
      for (p = 0; p < 4; p++)
        for (q = 0; q < 4; q++)
          for (s = 0; s < 4; s++)
            c[(size_t)((p * 4 + q) * 4 + s) * n2e * n1e + cell] = GLOBALMETMACP0A3(conn, i, j, k, p, q, s);
      {
        struct of_geom geomdontuse, *ptrgeom = &geomdontuse;
        FTYPE V[NDIM], pr[NPR], prfloor[NPR];
        int pl;
        PALLLOOP(pl) pr[pl] = 0.0;
        get_geometry(i, j, k, CENT, ptrgeom);
        bl_coord_ijk(i, j, k, CENT, V);
        set_density_floors(ptrgeom, pr, prfloor);
        a[cell] = V[1];
        a[(size_t)n2e * n1e + cell] = prfloor[RHO];
        a[(size_t)2 * n2e * n1e + cell] = prfloor[UU];
      }
    }
  write_npy(dir, "geom.npy", "<f8", g, sizeof(double), 4, gshape);
  write_npy(dir, "conn.npy", "<f8", c, sizeof(double), 3, cshape);
  write_npy(dir, "aux.npy", "<f8", a, sizeof(double), 3, ashape);
  free(g); free(c); free(a);
}

/* CENT metric records and connection of every cell of the extended grid (all k), for checking
   that the reference's tables do not depend on x3: [n3e][n2e][n1e][28] and [..][64] */
static void dump_geometry_allk(const char *dir)
{
  const int n1e = N1 + 2 * N1BND, n2e = N2 + 2 * N2BND, n3e = N3 + 2 * N3BND;
  long gshape[4] = {n3e, n2e, n1e, 28};
  long cshape[4] = {n3e, n2e, n1e, 64};
  double *g = (double *)calloc((size_t)n3e * n2e * n1e * 28, sizeof(double));
  double *c = (double *)calloc((size_t)n3e * n2e * n1e * 64, sizeof(double));
  size_t o = 0, oc = 0;
  int i, j, k, m, n, p, q, r;
  for (k = -N3BND; k < N3 + N3BND; k++)
    for (j = -N2BND; j < N2 + N2BND; j++)
      for (i = -N1BND; i < N1 + N1BND; i++) {
        struct of_geom geomdontuse, *ptrgeom = &geomdontuse;
        get_geometry(i, j, k, CENT, ptrgeom);
        for (m = 0; m < 4; m++)
          for (n = m; n < 4; n++) g[o++] = ptrgeom->gcov[GIND(m, n)];
        for (m = 0; m < 4; m++)
          for (n = m; n < 4; n++) g[o++] = ptrgeom->gcon[GIND(m, n)];
        g[o++] = ptrgeom->gcovpert[TT];
        g[o++] = ptrgeom->alphalapse;
        g[o++] = ptrgeom->betasqoalphasq;
        for (m = 1; m <= 3; m++) g[o++] = ptrgeom->beta[m];
        g[o++] = ptrgeom->gdet;
        g[o++] = ptrgeom->igdetnosing;
        for (p = 0; p < 4; p++)
          for (q = 0; q < 4; q++)
            for (r = 0; r < 4; r++) c[oc++] = GLOBALMETMACP0A3(conn, i, j, k, p, q, r);
      }
  write_npy(dir, "geomk.npy", "<f8", g, sizeof(double), 4, gshape);
  write_npy(dir, "connk.npy", "<f8", c, sizeof(double), 4, cshape);
  free(g); free(c);
}

static void dump_grid(const char *dir)
{
  double v[24];
  long shape[1] = {24};
  int d;
  v[0] = N1; v[1] = N2; v[2] = N3; v[3] = MAXBND;
  for (d = 0; d < 4; d++) { v[4 + d] = startx[d]; v[8 + d] = dx[d]; }
  v[12] = a; v[13] = hslope; v[14] = R0; v[15] = Rin; v[16] = Rout; v[17] = Rhor;
  v[18] = gam; v[19] = cour; v[20] = lim[1]; v[21] = fluxmethod; v[22] = TIMEORDER; v[23] = dt;
  write_npy(dir, "grid.npy", "<f8", v, sizeof(double), 1, shape);
}

/* ---- substep records: the linker routes the reference's calls of advance() (advance.c:85,
   called from step_ch.c:798), fluxcalc() (flux.c:38, called from advance.c:312) and
   post_fixup() (fixup.c:53, called from step_ch.c's post_advance) through the __wrap_
   functions below (ld --wrap), which write their inputs and outputs for the steps listed in
   HREF_SUBSTEP_STEPS (comma-separated, 1-based) and call the reference's own functions. ---- */
static const char *sub_dir = NULL;
static int sub_active = 0;
static char sub_prefix[64];
static char adv_prefix[64]; /* sub_<step>_<timeorder> of the latest recorded advance() */

static int step_wanted(long step)
{
  const char *s = getenv("HREF_SUBSTEP_STEPS");
  char buf[256], *tok, *save;
  if (!s || !sub_dir) return 0;
  snprintf(buf, sizeof buf, "%s", s);
  for (tok = strtok_r(buf, ",", &save); tok; tok = strtok_r(NULL, ",", &save))
    if (atol(tok) == step) return 1;
  return 0;
}

/* an extended (ghost zones included) array of the reference, in the order [k][j][i][pl] */
static void dump_ext(const char *what, FTYPE (*p)[NSTORE2][NSTORE3][NPR])
{
  const int n1e = N1 + 2 * N1BND, n2e = N2 + 2 * N2BND, n3e = N3 + 2 * N3BND;
  long shape[4] = {n3e, n2e, n1e, NPR};
  double *buf = (double *)malloc(sizeof(double) * (size_t)n1e * n2e * n3e * NPR);
  char name[128];
  size_t o = 0;
  int i, j, k, pl;
  for (k = -N3BND; k < N3 + N3BND; k++)
    for (j = -N2BND; j < N2 + N2BND; j++)
      for (i = -N1BND; i < N1 + N1BND; i++)
        for (pl = 0; pl < NPR; pl++) buf[o++] = MACP0A1(p, i, j, k, pl);
  snprintf(name, sizeof name, "%s_%s.npy", sub_prefix, what);
  write_npy(sub_dir, name, "<f8", buf, sizeof(double), 4, shape);
  free(buf);
}

static void dump_flags(const char *what)
{
  const int n1e = N1 + 2 * N1BND, n2e = N2 + 2 * N2BND, n3e = N3 + 2 * N3BND;
  long shape[3] = {n3e, n2e, n1e};
  double *buf = (double *)malloc(sizeof(double) * (size_t)n1e * n2e * n3e);
  char name[128];
  size_t o = 0;
  int i, j, k;
  for (k = -N3BND; k < N3 + N3BND; k++)
    for (j = -N2BND; j < N2 + N2BND; j++)
      for (i = -N1BND; i < N1 + N1BND; i++) buf[o++] = GLOBALMACP0A1(pflag, i, j, k, FLAGUTOPRIMFAIL);
  snprintf(name, sizeof name, "%s_%s.npy", sub_prefix, what);
  write_npy(sub_dir, name, "<f8", buf, sizeof(double), 3, shape);
  free(buf);
}

static void dump_scalars(const char *what, const double *v, long n)
{
  char name[128];
  snprintf(name, sizeof name, "%s_%s.npy", sub_prefix, what);
  write_npy(sub_dir, name, "<f8", v, sizeof(double), 1, &n);
}

int __real_advance(int stage, FTYPE (*pi)[NSTORE2][NSTORE3][NPR], FTYPE (*pb)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*pf)[NSTORE2][NSTORE3][NPR], FTYPE (*pstag)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*pl_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                   FTYPE (*pr_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP], FTYPE (*F1)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*F2)[NSTORE2][NSTORE3][NPR], FTYPE (*F3)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*vpot)[NSTORE1 + SHIFTSTORE1][NSTORE2 + SHIFTSTORE2][NSTORE3 + SHIFTSTORE3],
                   FTYPE (*ui)[NSTORE2][NSTORE3][NPR], FTYPE (*uf)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*ucum)[NSTORE2][NSTORE3][NPR], FTYPE *CUf, FTYPE *Cunew, SFTYPE fluxdt,
                   SFTYPE boundtime, int timeorder, int numtimeorders, FTYPE *ndt);

int __wrap_advance(int stage, FTYPE (*pi)[NSTORE2][NSTORE3][NPR], FTYPE (*pb)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*pf)[NSTORE2][NSTORE3][NPR], FTYPE (*pstag)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*pl_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                   FTYPE (*pr_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP], FTYPE (*F1)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*F2)[NSTORE2][NSTORE3][NPR], FTYPE (*F3)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*vpot)[NSTORE1 + SHIFTSTORE1][NSTORE2 + SHIFTSTORE2][NSTORE3 + SHIFTSTORE3],
                   FTYPE (*ui)[NSTORE2][NSTORE3][NPR], FTYPE (*uf)[NSTORE2][NSTORE3][NPR],
                   FTYPE (*ucum)[NSTORE2][NSTORE3][NPR], FTYPE *CUf, FTYPE *Cunew, SFTYPE fluxdt,
                   SFTYPE boundtime, int timeorder, int numtimeorders, FTYPE *ndt)
{
  int r, want = step_wanted(nstep + 1);
  if (want) {
    double v[14];
    int m;
    snprintf(adv_prefix, sizeof adv_prefix, "sub_%ld_%d", nstep + 1, timeorder);
    snprintf(sub_prefix, sizeof sub_prefix, "%s", adv_prefix);
    dump_ext("pi", pi);
    dump_ext("pb", pb);
    v[0] = dt; v[1] = fluxdt; v[2] = timeorder; v[3] = numtimeorders;
    for (m = 0; m < 4; m++) { v[4 + m] = CUf[m]; v[8 + m] = Cunew[m]; }
    v[12] = t; v[13] = boundtime;
    dump_scalars("args", v, 14);
    sub_active = 1;
  }
  r = __real_advance(stage, pi, pb, pf, pstag, pl_ct, pr_ct, F1, F2, F3, vpot, ui, uf, ucum, CUf, Cunew, fluxdt,
                     boundtime, timeorder, numtimeorders, ndt);
  if (want) {
    double v[1];
    sub_active = 0;
    snprintf(sub_prefix, sizeof sub_prefix, "%s", adv_prefix);
    dump_ext("pf", pf);
    dump_flags("pflag");
    v[0] = *ndt;
    dump_scalars("ndt", v, 1);
  }
  return r;
}

int __real_fluxcalc(int stage, FTYPE (*pr)[NSTORE2][NSTORE3][NPR], FTYPE (*pstag)[NSTORE2][NSTORE3][NPR],
                    FTYPE (*pl_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                    FTYPE (*pr_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                    FTYPE (*vpot)[NSTORE1 + SHIFTSTORE1][NSTORE2 + SHIFTSTORE2][NSTORE3 + SHIFTSTORE3],
                    FTYPE (*F1)[NSTORE2][NSTORE3][NPR], FTYPE (*F2)[NSTORE2][NSTORE3][NPR],
                    FTYPE (*F3)[NSTORE2][NSTORE3][NPR], FTYPE CUf, FTYPE fluxdt, FTYPE *ndt1, FTYPE *ndt2,
                    FTYPE *ndt3);

int __wrap_fluxcalc(int stage, FTYPE (*pr)[NSTORE2][NSTORE3][NPR], FTYPE (*pstag)[NSTORE2][NSTORE3][NPR],
                    FTYPE (*pl_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                    FTYPE (*pr_ct)[NSTORE1][NSTORE2][NSTORE3][NPR2INTERP],
                    FTYPE (*vpot)[NSTORE1 + SHIFTSTORE1][NSTORE2 + SHIFTSTORE2][NSTORE3 + SHIFTSTORE3],
                    FTYPE (*F1)[NSTORE2][NSTORE3][NPR], FTYPE (*F2)[NSTORE2][NSTORE3][NPR],
                    FTYPE (*F3)[NSTORE2][NSTORE3][NPR], FTYPE CUf, FTYPE fluxdt, FTYPE *ndt1, FTYPE *ndt2,
                    FTYPE *ndt3)
{
  int r = __real_fluxcalc(stage, pr, pstag, pl_ct, pr_ct, vpot, F1, F2, F3, CUf, fluxdt, ndt1, ndt2, ndt3);
  if (sub_active) {
    double v[3];
    /* a direction of one cell has no flux array (F3 of a 2-D grid) */
    if (N1 > 1) dump_ext("F1", F1);
    if (N2 > 1) dump_ext("F2", F2);
    if (N3 > 1) dump_ext("F3", F3);
    v[0] = *ndt1; v[1] = *ndt2; v[2] = *ndt3;
    dump_scalars("ndtdir", v, 3);
  }
  return r;
}

int __real_post_fixup(int stageit, SFTYPE boundtime, FTYPE (*pv)[NSTORE2][NSTORE3][NPR],
                      FTYPE (*pbackup)[NSTORE2][NSTORE3][NPR], FTYPE (*ucons)[NSTORE2][NSTORE3][NPR],
                      int finalstep);

int __wrap_post_fixup(int stageit, SFTYPE boundtime, FTYPE (*pv)[NSTORE2][NSTORE3][NPR],
                      FTYPE (*pbackup)[NSTORE2][NSTORE3][NPR], FTYPE (*ucons)[NSTORE2][NSTORE3][NPR],
                      int finalstep)
{
  int r, want = step_wanted(nstep + 1);
  if (want) {
    snprintf(sub_prefix, sizeof sub_prefix, "%s", adv_prefix);
    dump_ext("fixin", pv);
    dump_flags("fixflag");
  }
  r = __real_post_fixup(stageit, boundtime, pv, pbackup, ucons, finalstep);
  if (want) {
    snprintf(sub_prefix, sizeof sub_prefix, "%s", adv_prefix);
    dump_ext("fixout", pv);
  }
  return r;
}

/* every bound_prim_user_dir() call (bounds.fishmon.c:15, called per direction from
   bound_anyprim step_ch.c) of a wanted step: its input, output and arguments, numbered in
   call order within the step */
static int bnd_calls = 0;

int __real_bound_prim_user_dir(int boundstage, SFTYPE boundtime, int whichdir, int boundvartype,
                               FTYPE (*prim)[NSTORE2][NSTORE3][NPR]);

int __wrap_bound_prim_user_dir(int boundstage, SFTYPE boundtime, int whichdir, int boundvartype,
                               FTYPE (*prim)[NSTORE2][NSTORE3][NPR])
{
  int r, want = step_wanted(nstep + 1);
  if (want) {
    double v[4];
    snprintf(sub_prefix, sizeof sub_prefix, "bnd_%ld_%d", nstep + 1, bnd_calls);
    v[0] = whichdir; v[1] = boundvartype; v[2] = boundstage; v[3] = BOUNDPRIMTYPE;
    dump_scalars("info", v, 4);
    dump_ext("in", prim);
  }
  r = __real_bound_prim_user_dir(boundstage, boundtime, whichdir, boundvartype, prim);
  if (want) {
    snprintf(sub_prefix, sizeof sub_prefix, "bnd_%ld_%d", nstep + 1, bnd_calls);
    dump_ext("out", prim);
    bnd_calls++;
  }
  return r;
}

/* HREF_PROBE="i,j,k,dir": print the face states and flux of that face at every flux
   computation (flux_compute_general fluxcompute.c:19, called from fluxcalc_standard) */
int __real_flux_compute_general(int i, int j, int k, int dir, struct of_geom *ptrgeom, FTYPE CUf, FTYPE *p_c,
                                FTYPE *p_l, FTYPE *p_r, FTYPE *F, FTYPE *ctopptr);

int __wrap_flux_compute_general(int i, int j, int k, int dir, struct of_geom *ptrgeom, FTYPE CUf, FTYPE *p_c,
                                FTYPE *p_l, FTYPE *p_r, FTYPE *F, FTYPE *ctopptr)
{
  static int pi = -9999, pj, pk, pd;
  int r, pl;
  if (pi == -9999) {
    const char *s = getenv("HREF_PROBE");
    if (!s || sscanf(s, "%d,%d,%d,%d", &pi, &pj, &pk, &pd) != 4) pi = -9998;
  }
  r = __real_flux_compute_general(i, j, k, dir, ptrgeom, CUf, p_c, p_l, p_r, F, ctopptr);
  if (i == pi && j == pj && k == pk && dir == pd) {
    fprintf(stderr, "PROBE nstep=%ld face %d %d %d dir %d\n  p_l", nstep, i, j, k, dir);
    for (pl = 0; pl < NPR; pl++) fprintf(stderr, " %.17g", p_l[pl]);
    fprintf(stderr, "\n  p_r");
    for (pl = 0; pl < NPR; pl++) fprintf(stderr, " %.17g", p_r[pl]);
    fprintf(stderr, "\n  F  ");
    for (pl = 0; pl < NPR; pl++) fprintf(stderr, " %.17g", F[pl]);
    fprintf(stderr, "\n  ctop %.17g\n", *ctopptr);
  }
  return r;
}

/* HREF_WPROBE="dir,j,k[,pl]" (j,k: the transverse indices of the line as the reference's loop
   passes them): print one primitive's line (default the density) of that WENO reconstruction -- input, SMONO indicator,
   pressure-jump indicator and the left/right edge values (pass_1d_line_multipl_weno
   reconstructeno.c:2877, called through a pointer set in interpline.c) */
void __real_pass_1d_line_multipl_weno(int MULTIPLTYPE, int whichquantity, int dir, int do_weight_or_recon,
                                      int recontype, int whichreduce, int preforder, int bs, int ps, int pe, int be,
                                      int *minorder, int *maxorder, int *shift, FTYPE *shockindicator,
                                      FTYPE *stiffindicator, FTYPE *Vline, FTYPE *Pline,
                                      FTYPE (*df)[NUMDFS][NBIGM], FTYPE (*dP)[NBIGM], FTYPE (*etai)[NBIGM],
                                      FTYPE (*monoindicator)[NUMMONOINDICATORS][NBIGM], FTYPE (*yprim)[2][NBIGM],
                                      FTYPE (*ystencilvar)[2][NBIGM], FTYPE (*yin)[2][NBIGM], FTYPE (*yout)[2][NBIGM],
                                      FTYPE (*youtpolycoef)[MAXSPACEORDER][NBIGM], struct of_trueijkp *trueijkp);

void __wrap_pass_1d_line_multipl_weno(int MULTIPLTYPE, int whichquantity, int dir, int do_weight_or_recon,
                                      int recontype, int whichreduce, int preforder, int bs, int ps, int pe, int be,
                                      int *minorder, int *maxorder, int *shift, FTYPE *shockindicator,
                                      FTYPE *stiffindicator, FTYPE *Vline, FTYPE *Pline,
                                      FTYPE (*df)[NUMDFS][NBIGM], FTYPE (*dP)[NBIGM], FTYPE (*etai)[NBIGM],
                                      FTYPE (*monoindicator)[NUMMONOINDICATORS][NBIGM], FTYPE (*yprim)[2][NBIGM],
                                      FTYPE (*ystencilvar)[2][NBIGM], FTYPE (*yin)[2][NBIGM], FTYPE (*yout)[2][NBIGM],
                                      FTYPE (*youtpolycoef)[MAXSPACEORDER][NBIGM], struct of_trueijkp *trueijkp)
{
  static int pd = -9999, pj, pk, ppl = RHO;
  int i;
  __real_pass_1d_line_multipl_weno(MULTIPLTYPE, whichquantity, dir, do_weight_or_recon, recontype, whichreduce,
                                   preforder, bs, ps, pe, be, minorder, maxorder, shift, shockindicator,
                                   stiffindicator, Vline, Pline, df, dP, etai, monoindicator, yprim, ystencilvar, yin,
                                   yout, youtpolycoef, trueijkp);
  if (pd == -9999) {
    const char *s = getenv("HREF_WPROBE");
    if (!s || sscanf(s, "%d,%d,%d,%d", &pd, &pj, &pk, &ppl) < 3) pd = -9998;
  }
  if (dir == pd && trueijkp->j == pj && trueijkp->k == pk && nstep == 0) {
    fprintf(stderr, "WPROBE dir %d j %d k %d bs %d ps %d pe %d be %d preforder %d\n", dir, pj, pk, bs, ps, pe, be,
            preforder);
    for (i = bs; i <= be; i++)
      fprintf(stderr, "  i %3d y %.17g yprim %.17g mono %.17g dP %.17g shock %.17g l %.17g r %.17g\n", i, yin[ppl][0][i], yprim[ppl][0][i],
              monoindicator[ppl][MONOINDTYPE][i], dP[0][i], shockindicator[i], yout[ppl][0][i], yout[ppl][1][i]);
  }
}

static void do_step(void)
{
  bnd_calls = 0;
  nstroke = 0;
  step_ch_full(GLOBALPOINT(pglobal), GLOBALPOINT(pstagglobal), GLOBALPOINT(unewglobal),
               GLOBALPOINT(vpotarrayglobal), GLOBALPOINT(Bhatglobal), GLOBALPOINT(gp_l),
               GLOBALPOINT(gp_r), GLOBALPOINT(F1), GLOBALPOINT(F2), GLOBALPOINT(F3),
               GLOBALPOINT(emf), GLOBALPOINT(ulastglobal));
  nstep++;
}

static double wall(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char *argv[])
{
  const char *mode, *outdir;
  int nthreads, init_argc = 2;
  char *init_argv_store[3], thr[16];
  char **init_argv = init_argv_store;
  if (argc < 4) {
    fprintf(stderr, "usage: %s run|points|time <outdir> <nthreads> ...\n", argv[0]);
    return 2;
  }
  mode = argv[1];
  outdir = argv[2];
  nthreads = atoi(argv[3]);
  mkdir(outdir, 0755);
  /* init() reads the OpenMP thread count from its argv (myargs, mpi_init.c:212); for the
     run and points modes the initial state is set on one thread, so that the perturbation's
     random sequence is assigned to cells in a fixed order */
  snprintf(thr, sizeof thr, "%d", (strcmp(mode, "time") && !getenv("HREF_INIT_ALL_THREADS")) ? 1 : nthreads);
  init_argv_store[0] = argv[0];
  init_argv_store[1] = thr;
  init_argv_store[2] = NULL;
  if (init(&init_argc, &init_argv) >= 1) {
    fprintf(stderr, "ref_driver: init failed\n");
    return 1;
  }
  numopenmpthreads = nthreads;
  omp_set_num_threads(nthreads);
  reallaststep = onemorestep = 0;

  if (!strcmp(mode, "run")) {
    int nsteps, every, s;
    double *rec;
    long shape[2];
    char name[64];
    if (argc < 6) return 2;
    nsteps = atoi(argv[4]);
    every = atoi(argv[5]);
    sub_dir = outdir;
    dump_grid(outdir);
    dump_geometry(outdir);
    if (getenv("HREF_GEOM_ALLK")) dump_geometry_allk(outdir);
    dump_state(outdir, "p0.npy");
    rec = (double *)malloc(sizeof(double) * 4 * (nsteps + 1));
    for (s = 1; s <= nsteps; s++) {
      double dt_used = dt, t0 = t;
      do_step();
      rec[4 * s + 0] = t0;
      rec[4 * s + 1] = dt_used;
      rec[4 * s + 2] = nstroke;
      rec[4 * s + 3] = dt; /* the next step's dt */
      if ((every > 0 && s % every == 0) || s == nsteps) {
        snprintf(name, sizeof name, "p_%d.npy", s);
        dump_state(outdir, name);
      }
    }
    rec[0] = rec[1] = rec[2] = rec[3] = 0.0;
    shape[0] = nsteps + 1;
    shape[1] = 4;
    write_npy(outdir, "steps.npy", "<f8", rec, sizeof(double), 2, shape);
    free(rec);
    return 0;
  }
  if (!strcmp(mode, "points")) {
    FILE *f;
    long n, p, shape[2];
    double *in, *out;
    if (argc < 5) return 2;
    f = fopen(argv[4], "rb");
    if (!f) return 3;
    fseek(f, 0, SEEK_END);
    n = ftell(f) / (long)(sizeof(double) * 18);
    fseek(f, 0, SEEK_SET);
    in = (double *)malloc(sizeof(double) * 18 * n);
    if (fread(in, sizeof(double) * 18, n, f) != (size_t)n) return 3;
    fclose(f);
    out = (double *)malloc(sizeof(double) * 10 * n);
    for (p = 0; p < n; p++) {
      const double *r = in + 18 * p;
      int i = (int)r[0], j = (int)r[1], k = 0, pl;
      struct of_geom geomdontuse, *ptrgeom = &geomdontuse;
      struct of_newtonstats newtonstats;
      FTYPE U[NPR], pr[NPR];
      memset(&newtonstats, 0, sizeof newtonstats);
      for (pl = 0; pl < NPR; pl++) { U[pl] = r[2 + pl]; pr[pl] = r[10 + pl]; }
      get_geometry(i, j, k, CENT, ptrgeom);
      GLOBALMACP0A1(pflag, i, j, k, FLAGUTOPRIMFAIL) = UTOPRIMNOFAIL;
      Utoprimgen(1, EVOLVEUTOPRIM, UEVOLVE, U, ptrgeom, pr, &newtonstats);
      for (pl = 0; pl < NPR; pl++) out[10 * p + pl] = pr[pl];
      out[10 * p + 8] = GLOBALMACP0A1(pflag, i, j, k, FLAGUTOPRIMFAIL);
      out[10 * p + 9] = newtonstats.nstroke;
    }
    shape[0] = n;
    shape[1] = 10;
    write_npy(outdir, "points.npy", "<f8", out, sizeof(double), 2, shape);
    free(in);
    free(out);
    return 0;
  }
  if (!strcmp(mode, "fixup")) {
    const int n1e = N1 + 2 * N1BND, n2e = N2 + 2 * N2BND, n3e = N3 + 2 * N3BND;
    const size_t next = (size_t)n1e * n2e * n3e, nact = (size_t)N1 * N2 * N3;
    FILE *f;
    double *in;
    size_t o = 0;
    int i, j, k, pl;
    if (argc < 5) return 2;
    f = fopen(argv[4], "rb");
    if (!f) return 3;
    in = (double *)malloc(sizeof(double) * (next * NPR + nact));
    if (fread(in, sizeof(double), next * NPR + nact, f) != next * NPR + nact) return 3;
    fclose(f);
    for (k = -N3BND; k < N3 + N3BND; k++)
      for (j = -N2BND; j < N2 + N2BND; j++)
        for (i = -N1BND; i < N1 + N1BND; i++)
          for (pl = 0; pl < NPR; pl++) GLOBALMACP0A1(pglobal, i, j, k, pl) = in[o++];
    for (k = -N3BND; k < N3 + N3BND; k++)
      for (j = -N2BND; j < N2 + N2BND; j++)
        for (i = -N1BND; i < N1 + N1BND; i++) GLOBALMACP0A1(pflag, i, j, k, FLAGUTOPRIMFAIL) = UTOPRIMNOFAIL;
    for (k = 0; k < N3; k++)
      for (j = 0; j < N2; j++)
        for (i = 0; i < N1; i++) GLOBALMACP0A1(pflag, i, j, k, FLAGUTOPRIMFAIL) = (PFTYPE)in[o++];
    sub_dir = outdir;
    snprintf(sub_prefix, sizeof sub_prefix, "post");
    __real_post_fixup(STAGEM1, t, GLOBALPOINT(pglobal), GLOBALPOINT(pglobal), GLOBALPOINT(unewglobal),
                      (argc > 5) ? atoi(argv[5]) : 1);
    dump_ext("fixout", GLOBALPOINT(pglobal));
    dump_flags("fixflag");
    free(in);
    return 0;
  }
  if (!strcmp(mode, "time")) {
    int nsteps, s;
    double t0, t1, rec[4];
    long shape[1] = {4};
    if (argc < 5) return 2;
    nsteps = atoi(argv[4]);
    do_step(); /* first step outside the timed region */
    t0 = wall();
    for (s = 0; s < nsteps; s++) do_step();
    t1 = wall();
    rec[0] = (double)N1 * N2 * N3 * nsteps / (t1 - t0);
    rec[1] = t1 - t0;
    rec[2] = nsteps;
    rec[3] = (double)N1 * N2 * N3;
    write_npy(outdir, "time.npy", "<f8", rec, sizeof(double), 1, shape);
    printf("{\"zone_cycles_per_s\": %.6g, \"seconds\": %.6g, \"steps\": %d, \"threads\": %d}\n",
           rec[0], rec[1], nsteps, nthreads);
    return 0;
  }
  fprintf(stderr, "ref_driver: unknown mode %s\n", mode);
  return 2;
}
