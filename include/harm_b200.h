/*
 * harm_b200.h -- C ABI of the B200 implementation of HARM's per-timestep GRMHD update.
 *
 * Two shared libraries implement this header:
 *   libharm_host.so  host-side producers of the inputs (grid, metric tables, torus
 *                    initial state).  In HARM these are set_grid() (set_grid.c:114),
 *                    set_connection() (set_grid.c:1033) and init() (initbase.c:7).
 *   libharm_b200.so  the device path: reconstruction (MC / PPM / WENO5), HLL fluxes,
 *                    flux-CT, conserved update with connection sources, Utoprimgen
 *                    Newton inversion and floors/fixups, boundary conditions, and the
 *                    learned initial-guess network.  Every numeric routine of the
 *                    step runs on the GPU; there is no CPU fallback in this library.
 *
 * Conventions (shared by every entry point):
 *   - Primitive order RHO,UU,U1,U2,U3,B1,B2,B3 (global.nondepnmemonics.h:883-890);
 *     U1..U3 are the relative 4-velocity \tilde u^i (WHICHVEL=VELREL4), B^i = *F^{it}.
 *   - State arrays are structure-of-arrays FP64: P[pl][k][j][i] with i fastest, over the
 *     extended grid n1e x n2e x n3e (ghost zones included).  Index (i,j,k) of an active
 *     cell maps to (i+ng, j+ng, k+ng3) with ng3 = (n3>1 ? ng : 0).
 *   - Conserved arrays U[pl][k][j][i] are in HARM's UEVOLVE form: sqrt(-g) times
 *     (rho u^t, T^t_t + rho u^t, T^t_i, B^i)  (REMOVERESTMASSFROMUU=2, phys.tools.c:1071).
 *   - Flux arrays F1/F2/F3[pl][k][j][i]: F_d at index i lives on the lower face of cell i
 *     in direction d (flux.c:852 "face" convention; dU = -(F[i+1]-F[i])/dx).
 *   - The Kerr-Schild metric in modified Kerr-Schild coordinates does not depend on x3,
 *     so metric tables are stored per (i,j) only: geom[loc][field][j][i] over n2e x n1e.
 *     FACE3 shares CENT, CORN1 shares FACE2, CORN2 shares FACE1 (HARM stores all eight
 *     locations per (i,j,k): superdefs.h:382).
 *   - Streams: a context enqueues its work on its own non-blocking CUDA stream
 *     (harm_b200_stream).  Calls that return host values (ndt, dt, stats, losses) synchronise
 *     that stream before returning; the others (bound, post_fixup, Utoprimgen over points,
 *     the mlp_* kernels) return once their work is queued.  A caller that writes the
 *     arguments or reads the results on another stream orders that stream against the
 *     context's (events, or a synchronisation).
 *   - Return value: 0 on success, >0 on error (HARM's MYFUN convention,
 *     global.variousmacros.h:43).  Per-cell inversion failures are not return codes;
 *     they are written to an int8 pflag array with HARM's codes
 *     (global.nondepnmemonics.h:824-844).
 */
#ifndef HARM_B200_H
#define HARM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HARM_B200_ABI_VERSION 1

/* primitive / conserved indices */
#define HARM_NPR 8
enum { HARM_RHO = 0, HARM_UU = 1, HARM_U1 = 2, HARM_U2 = 3, HARM_U3 = 4,
       HARM_B1 = 5, HARM_B2 = 6, HARM_B3 = 7 };

/* reconstruction choices (HARM lim[]: MC, PARA, WENO5BND, PARALINE; init.tools.c:128).
   PARALINE is the line PPM of interpline.para.c: extremum-preserving MC slopes and FLASH
   shock flattening from the cell's total pressure and sqrt(-g) rho u^dir; it needs ng >= 4. */
enum { HARM_LIM_MC = 0, HARM_LIM_PARA = 1, HARM_LIM_WENO5 = 2, HARM_LIM_PARALINE = 3 };

/* flux formula at a face (HARM fluxmethod, fluxcompute.c:243): HLL with the LAXF fallback
   where both wave speeds vanish, or LAXF (Rusanov) everywhere */
enum { HARM_FLUX_HLL = 0, HARM_FLUX_LAXF = 1 };

/* arithmetic of the flux path: FP64 everywhere in the IEEE operations of the reference's C
   in its order (HARM_PREC_FP64, no FMA contraction), FP32 reconstruction/HLL/CT with the
   conserved update, inversion and metric kept in FP64 (HARM_PREC_MIXED), or FP64 everywhere
   compiled with FMA contraction and the inversion's shared reciprocals (HARM_PREC_FP64_FMA:
   round-off-level differences from HARM_PREC_FP64; the FP64 path at its best speed) */
enum { HARM_PREC_FP64 = 0, HARM_PREC_MIXED = 1, HARM_PREC_FP64_FMA = 2 };

/* initial guess of the Newton inversion: the previous primitive (set_guess_Wp,
   utoprim_jon.c:890) or the learned network with fallback to the previous primitive */
enum { HARM_GUESS_PREV = 0, HARM_GUESS_MLP = 1 };

/* metric table locations (per (i,j)) */
enum { HARM_LOC_CENT = 0, HARM_LOC_FACE1 = 1, HARM_LOC_FACE2 = 2, HARM_LOC_CORN3 = 3,
       HARM_NLOC = 4 };

/* fields of one metric table location (struct of_compgeom, global.structs.h:20-85).
   Symmetric 4x4 tensors are stored as 10 entries in the order
   00,01,02,03,11,12,13,22,23,33. */
enum {
  HARM_G_GCOV = 0,            /* 10 entries g_{mu nu} */
  HARM_G_GCON = 10,           /* 10 entries g^{mu nu} */
  HARM_G_GCOVPERT_TT = 20,    /* g_tt + 1 (gcovpert[TT]) */
  HARM_G_ALPHA = 21,          /* lapse 1/sqrt(-g^{tt}) (metric.tools.c:1250) */
  HARM_G_BETASQOALPHASQ = 22, /* sum_j g_{tj} g^{tj} (metric.tools.c:1260) */
  HARM_G_BETA = 23,           /* 3 entries beta^j = g^{tj} alpha^2 (metric.tools.c:1275) */
  HARM_G_GDET = 26,           /* sqrt(-g) */
  HARM_G_IGDET = 27,          /* sign(gdet)/(|gdet|+SMALL) (metric.tools.c:1195) */
  HARM_NGF = 28
};

/* per-(i,j) auxiliary table at CENT: Boyer-Lindquist r and the two density floors
   (set_density_floors_default, rescaletype 0: fixup.c:2485-2486) */
enum { HARM_AUX_R = 0, HARM_AUX_RHOFLOOR = 1, HARM_AUX_UFLOOR = 2, HARM_NAUX = 3 };

/* inversion failure codes (global.nondepnmemonics.h:824-844) */
enum {
  HARM_UTOPRIMFAILFIXEDCOLD = -3, HARM_UTOPRIMFAILFIXEDUTOPRIM = -1,
  HARM_UTOPRIMNOFAIL = 0, HARM_UTOPRIMFAILCONV = 1, HARM_UTOPRIMFAILCONVW = 2,
  HARM_UTOPRIMFAILCONVUTSQ = 3, HARM_UTOPRIMFAILCONVGUESSUTSQ = 4,
  HARM_UTOPRIMFAILCONVUTSQVERYBAD = 5, HARM_UTOPRIMFAILNANGUESS = 7,
  HARM_UTOPRIMFAILNANRESULT = 8, HARM_UTOPRIMFAILRHONEG = 9, HARM_UTOPRIMFAILUNEG = 10,
  HARM_UTOPRIMFAILRHOUNEG = 11, HARM_UTOPRIMFAILU2AVG1 = 14, HARM_UTOPRIMFAILU2AVG2 = 15,
  HARM_UTOPRIMFAILCONVRET = 50
};

/* Run-time configuration of one grid (the globals HARM's hot path reads:
   defs.general.h, superdefs.h).  Filled by harm_grid_setup(). */
typedef struct harm_grid {
  int n1, n2, n3;          /* active cells */
  int ng;                  /* ghost cells per side (MAXBND) */
  int n1e, n2e, n3e;       /* extended sizes */
  int ng3;                 /* ghost cells in x3: ng if n3>1 else 0 */
  int lim;                 /* HARM_LIM_* */
  int fluxmethod;          /* HARM_FLUX_*; harm_grid_setup sets HARM_FLUX_HLL */
  double startx[4], dx[4]; /* x^mu of the lower corner of active cell (0,0,0), spacings */
  double a;                /* black-hole spin */
  double hslope, R0, Rin, Rout, Rhor;
  double gam;              /* ideal-gas adiabatic index */
  double cour;             /* Courant factor */
  double defcon, safe;     /* dt = defcon*wavedt, dt <= safe*dt_old (initbase.c:1029-1031) */
  double rho_floor_coef;   /* prfloorcoef[RHO] */
  double u_floor_coef;     /* prfloorcoef[UU] */
  double gammamax;         /* GAMMAMAX (initbase.c:1178) */
  double gammafail;        /* GAMMAFAIL = 100 GAMMAMAX */
} harm_grid;

/* Counters accumulated by the device step (the reference's nstroke and debug counters). */
typedef struct harm_stats {
  double newton_iters;     /* sum over inverted cells of Newton iterations (nstroke) */
  double cells_inverted;   /* number of cell inversions */
  double mlp_fallbacks;    /* cells whose learned guess failed and were re-solved */
  double inversion_failures; /* cells whose final pflag was a failure before fixup */
  double floor_hits;       /* cells where fixup1zone raised rho or u */
  double mlp_cells;        /* cells given the learned start (every cell inverted, except with
                              the gated engine: the cells whose previous state is a poor start) */
} harm_stats;

/* ------------------------------------------------------------------------------------
 * libharm_host.so : input producers (host C)
 * ------------------------------------------------------------------------------------ */

/* Fill a harm_grid for the modified-Kerr-Schild torus grid (LOGRSINTH coordinates,
   coord.c:930 and set_points coord.c:2038; Rin from setRin(setihor()), coord.c:2334-2359).
   Returns 0, or 1 on bad sizes. */
int harm_grid_setup(harm_grid *g, int n1, int n2, int n3, int lim, double a,
                    double hslope, double Rout, double cour);

/* Metric tables at CENT/FACE1/FACE2/CORN3 per (i,j): geom[HARM_NLOC][HARM_NGF][n2e][n1e];
   connection at CENT conn[64][n2e][n1e] with conn[(k*4+l)*4+j] = Gamma^k_{l j}
   (HARM conn[i][j][k][k][l][j], superdefs.h:423); aux[HARM_NAUX][n2e][n1e]. */
int harm_geometry_build(const harm_grid *g, double *geom, double *conn, double *aux);

/* Fishbone-Moncrief torus with a single poloidal loop, normalised to beta_min, internal
   energy perturbed by (1+0.04(U-1/2)) from `seed`; atmosphere at the floors.
   Writes P[8][n3e][n2e][n1e] (active cells; ghost zones are left to harm_b200_bound). */
int harm_torus_init(const harm_grid *g, const double *geom, const double *aux,
                    double beta_min, uint64_t seed, double *P);

/* ------------------------------------------------------------------------------------
 * libharm_b200.so : device path
 * ------------------------------------------------------------------------------------ */

typedef struct harm_ctx harm_ctx;

/* Create a context on CUDA device `device`: uploads the metric tables (once, as
   set_grid does once) and allocates the scratch of the step (fluxes, EMFs, U arrays).
   The caller owns the primitive arrays.  Read at creation, from the environment:
     HARM_B200_FLUX_STAGING=tma   stage the FP32 flux tiles with TMA tensor loads
                                  (default: coalesced loads; same arithmetic)
     HARM_B200_MLP_ENGINE          the learned start (HARM_GUESS_MLP): "gated" (default)
                                  gives it only to the cells whose first Newton step from
                                  the previous state exceeds HARM_B200_MLP_GATE (default
                                  0.02) of the convergence scale, with the mma.sync network
                                  inside the inversion kernel of those cells; every other
                                  cell is the plain inversion.  For every cell: "mma" (the
                                  mma.sync network in a kernel ahead of the inversion),
                                  "mma-fused" (inside the inversion kernel), "tc" (tcgen05
                                  tensor cores, a kernel ahead of it), "tc-fused" (inside
                                  it); the same network, the same results to the BF16
                                  rounding of its activations */
int harm_b200_create(const harm_grid *g, const double *geom_h, const double *conn_h,
                     const double *aux_h, int device, harm_ctx **out);
/* Create a context whose metric (CENT/FACE1/FACE2/CORN3), connection and floor tables are
   computed on the device from the grid (set_grid set_grid.c:114, set_connection
   set_grid.c:1033): Kerr-Schild in MKS coordinates, closed-form inverse metric, connection
   from Ridders-extrapolated central differences of the metric -- the algorithm of the host
   builder harm_geometry_build, whose tables it matches to the last bits of the math library.
   No host tables are needed. */
int harm_b200_create_grid(const harm_grid *g, int device, harm_ctx **out);
/* Copy the context's tables to host arrays in the layout harm_b200_create takes (any
   pointer may be NULL). */
int harm_b200_get_tables(harm_ctx *ctx, double *geom_h, double *conn_h, double *aux_h);
int harm_b200_destroy(harm_ctx *ctx);

/* CUDA stream the context launches on (cudaStream_t as void*). */
void *harm_b200_stream(harm_ctx *ctx);

/* Number of kernels this context has launched so far. */
unsigned long long harm_b200_launch_count(harm_ctx *ctx);

/* bound_prim() (step_ch.c:1332, bounds.fishmon.c): fill the ghost zones of d_P:
   x1 outflow (inner free, outer no-inflow), x2 polar axis, x3 periodic. */
int harm_b200_bound(harm_ctx *ctx, double *d_P);

/* fluxcalc() (flux.c:38): reconstruct d_pb at faces, HLL fluxes, Toth flux-CT.
   Writes d_F1/d_F2/d_F3 (UEVOLVE form) and ndt[3] = cour*dx/ctop minimised per
   direction (host array). */
int harm_b200_fluxcalc(harm_ctx *ctx, int precision, const double *d_pb,
                       double *d_F1, double *d_F2, double *d_F3, double ndt[3]);

/* advance() (advance.c:85 -> advance_standard advance.c:140) for one RK substep:
   fluxes of d_pb, U_i = primtoU(d_pi), source(d_pb), U_f = CUf0 U_i + CUf1 U_f +
   CUf2 dt dU, ucum, then Utoprimgen (utoprimgen.c:32) into d_pf with d_pb as guess,
   then fixup1zone (fixup.c:561).  ndt = defcon*wavedt (prepare_globaldt advance.c:1558).
   d_pflag[k][j][i] (active and ghost layout of P) receives the inversion codes.
   Coefficients: U_f and ucum are formed from U_i and dU of this substep only, which is exact
   for setup_rktimestep's TIMEORDER 1 and RK2 midpoint (CUf[1] = 0; Cunew[0..2] = 0 before
   the final substep); other sets (TVD RK2, RK3, RK4) return 2: they run through
   harm_b200_advance_u, which takes the RK step's conserved arrays. */
int harm_b200_advance(harm_ctx *ctx, int precision, int guess, int timeorder,
                      int numtimeorders, const double *d_pi, const double *d_pb,
                      double *d_pf, int8_t *d_pflag, double dt, const double CUf[4],
                      const double Cunew[4], double *ndt, harm_stats *stats);

/* advance() with the RK step's conserved arrays, as advance.c:85-91 takes ui, uf, ucum:
   d_ui, d_uf, d_ucum are [8][n3e][n2e][n1e] device arrays (UEVOLVE form, active cells used)
   that the caller keeps across the substeps of one step.  Per active cell: ui = primtoU(pi)
   (advance.c:454); on the first substep (timeorder 0) uf and ucum start from zero (:407);
   uf = CUf0 ui + CUf1 uf + CUf2 dt dU and ucum += Cunew0 ui + Cunew1 dt dU + Cunew2 uf
   (dUtoU advance.c:2046, global.stepch.h:1, :10); the inversion takes ucum on the final
   substep and uf before.  Every coefficient set of setup_rktimestep (step_ch.c:1171:
   TIMEORDER 1, 2 midpoint and TVD, 3, 4) runs.  The rest is harm_b200_advance's. */
int harm_b200_advance_u(harm_ctx *ctx, int precision, int guess, int timeorder, int numtimeorders,
                        const double *d_pi, const double *d_pb, double *d_pf, int8_t *d_pflag,
                        double *d_ui, double *d_uf, double *d_ucum, double dt, const double CUf[4],
                        const double Cunew[4], double *ndt, harm_stats *stats);

/* post_fixup() (fixup.c:53 -> bound_pflag, fixup_utoprim fixup.c:1061) of the final substep
   (finalstep 1) or an earlier one (0): every failed active cell (flag > 0) takes the average
   of its unfailed neighbours (for the U2AVG codes the smallest u of neighbour pairs not below
   its own), or where none is usable the average of its 8 in-plane neighbours (zero velocity
   in the reset region of the first 10 radial cells and two cells at either pole), then its
   Lorentz factor is limited to its own before the fix; its flag becomes -1 (the soft
   negative-density/energy and U2AVG codes only when finalstep is set).  d_pf's ghost zones
   must be bounded; the flags' ghost zones are filled here. */
int harm_b200_post_fixup(harm_ctx *ctx, double *d_pf, int8_t *d_pflag, int finalstep);

/* One full RK2 step (step_ch_full step_ch.c:35 with TIMEORDER=2, setup_rktimestep
   step_ch.c:1244-1266): two advance() substeps, each followed by bound, post_fixup,
   bound; then dt <- min(ndt, safe*dt) (post_stepch step_ch.c:213).  d_P is updated in
   place; *dt is the step used on input and the next step on output. */
int harm_b200_step(harm_ctx *ctx, int precision, int guess, double *d_P, double *dt,
                   harm_stats *stats);

/* nsteps full steps back to back with dt kept on the device between steps (one host
   synchronisation at the end).  *dt in: first step; out: the next step. */
int harm_b200_step_n(harm_ctx *ctx, int precision, int guess, double *d_P, int nsteps,
                     double *dt, harm_stats *stats);

/* Same step over a HOST primitive array: copies h_P in (in slabs of k-planes, the first
   substep's flux kernels of each slab starting as soon as it is resident), steps, copies it
   back.  Results are those of harm_b200_step. */
int harm_b200_step_host(harm_ctx *ctx, int precision, int guess, double *h_P, double *dt,
                        harm_stats *stats);

/* nsteps such steps over the host array h_P (each step copies the state in from h_P and back
   out to it, as nsteps calls of harm_b200_step_host would), pipelined across steps: a step's
   copy out runs in k-slabs on a second copy stream and the next step's copy in of each slab
   starts as soon as that slab is back on the host, so the two PCIe directions overlap and the
   next step's first flux tiles start on the slabs already resident.  Results are those of
   harm_b200_step_n; *dt in: first step, out: the next step. */
int harm_b200_step_host_n(harm_ctx *ctx, int precision, int guess, double *h_P, int nsteps,
                          double *dt, harm_stats *stats);

/* ------------------------------------------------------------------------------------
 * HARM's own array layout.  HARM stores primitives, conserved variables and fluxes as
 * FTYPE [N3M][N2M][N1M][NPR] (ORDERSTORAGE 5, global.storage.h:320-340) and its flags as
 * PFTYPE [N3M][N2M][N1M][NUMPFLAGS]; this library's device arrays are [pl][k][j][i] (HARM_NPR
 * planes of one primitive each, i fastest).  Both cover the extended grid with the same ghost
 * width (HARM's MAXBND must equal harm_grid.ng).  The conversions run on the context's stream
 * and return without waiting; HARM-layout arrays must be 16-byte aligned.
 * ------------------------------------------------------------------------------------ */
int harm_b200_from_harm_layout(harm_ctx *ctx, const double *d_harm, double *d_P);
int harm_b200_to_harm_layout(harm_ctx *ctx, const double *d_P, double *d_harm);
/* slot 0 (FLAGUTOPRIMFAIL) of each cell's numpflags ints <-> the int8 flag per cell */
int harm_b200_flags_to_harm(harm_ctx *ctx, const int8_t *d_pflag, int32_t *d_harm_pflag, int numpflags);
int harm_b200_flags_from_harm(harm_ctx *ctx, const int32_t *d_harm_pflag, int8_t *d_pflag, int numpflags);

/* The FP64 reciprocal that HARM_PREC_MIXED's inversion uses in place of IEEE division
   (utoprim_jon.c's divisions in the Newton residual): the hardware approximation
   rcp.approx.ftz.f64 refined by two Newton-Raphson steps, r[i] ~ 1/b[i] for n device
   values, on the context's stream.  Within one ulp of the IEEE quotient where b and 1/b are
   normal; flush-to-zero at the edges: a subnormal or zero b gives NaN, a b whose reciprocal
   is subnormal gives 0. */
int harm_b200_mixed_reciprocal(harm_ctx *ctx, const double *d_b, double *d_r, size_t n);

/* harm_b200_step_host over a host array in HARM's layout (step_ch_full step_ch.c:35 with
   HARM's own p array): one copy per k-slab, each slab converted on the device as it arrives
   (ahead of the first substep's flux tiles that stage it), the state converted back and
   copied out after the step.  Results equal harm_b200_step's on the converted state. */
int harm_b200_step_host_harm(harm_ctx *ctx, int precision, int guess, double *h_P_harm, double *dt,
                             harm_stats *stats);

/* Utoprimgen() (utoprimgen.c:32) over n independent points: d_U[8][n] in UEVOLVE form,
   d_geom[HARM_NGF][n] CENT metric of each point, d_P[8][n] guess in / primitives out,
   d_pflag[n] codes out, d_iters[n] Newton iterations out (may be NULL). */
int harm_b200_utoprimgen_points(harm_ctx *ctx, size_t n, int guess, const double *d_U,
                                const double *d_geom, double *d_P, int8_t *d_pflag,
                                int32_t *d_iters);

/* Stage times of one RK substep on d_P (unchanged), averaged over `reps` runs, measured
   with CUDA events on the context stream: ms[0] flux kernels of all directions and the
   EMF kernel, ms[1] (reserved, 0), ms[2] update+inversion, ms[3] one bound_prim,
   ms[4] post_fixup. */
int harm_b200_time_stages(harm_ctx *ctx, int precision, int guess, const double *d_P,
                          double dt, int reps, double ms[5]);

/* ------------------------------------------------------------------------------------
 * Learned initial guess of the inversion.  No counterpart function in the reference: the
 * network replaces the starting point set_guess_Wp (utoprim_jon.c:890) computes from the
 * previous primitive state; the Newton iteration (general_newton_raphson utoprim_jon.c:3853)
 * and its tolerances are unchanged, and a cell whose learned start does not converge is
 * solved again from the previous-state start.
 *
 * Network: 10 features -> 64 -> 64 -> 64 -> 2 outputs, SiLU.  Features of a cell, from the
 * alpha-scaled setup quantities of U/sqrt(-g) (compute_setup_quantities utoprim_jon.c:716)
 * and the metric, slog(x) = sign(x) log(1+|x|):
 *   log D, slog(B^2/D), slog(Qt^2/D^2), slog((Q.B)^2/D^3), slog(-Q.n'/D),
 *   slog(Qt^2/((Q.n')^2+D^2)), alpha, log sqrt(-g), beta^2/alpha^2, g_tt+1.
 * Outputs: log(W'/D) (the start of the iteration) and log(1+utsq) (v^2 = utsq/(1+utsq)).
 * Parameters: HARM_MLP_NPARAMS floats W1[10][64] b1 W2[64][64] b2 W3[64][64] b3 W4[64][2] b4.
 * Normalisation record: HARM_MLP_NNORM floats: feature means[10], standard deviations[10],
 * target means[2], target standard deviations[2].
 * Arrays of pairs: d_feat[n][10], d_targ[n][2] (FP32, sample-major).
 * ------------------------------------------------------------------------------------ */
#define HARM_MLP_NIN 10
#define HARM_MLP_NOUT 2
#define HARM_MLP_NPARAMS 9154
#define HARM_MLP_NNORM 24

/* Training pairs dumped from the context's most recent inversion: the U that inversion
   inverted and the primitives d_P it produced (active cells t = phase + stride*k, in
   i-fastest order over active cells).  Targets are the converged W' of a plain re-solve;
   cells whose hot inversion fails are skipped.  Writes at most `max` pairs (order not
   fixed; d_cell, if not NULL, receives each pair's active-cell index) and their number. */
int harm_b200_mlp_dump(harm_ctx *ctx, const double *d_P, int stride, int phase, size_t max,
                       float *d_feat, float *d_targ, int32_t *d_cell, size_t *n_out);

/* n synthetic pairs from wide primitive distributions on this context's metric (rho
   log-uniform [1e-6,1], u/rho log-uniform [1e-4,1e2], gamma uniform [1,50], b^2/rho
   log-uniform [1e-3,1e3], isotropic directions, Boyer-Lindquist r uniform [1.2,40]).
   Optional outputs: d_U[8][n] (UEVOLVE), d_P[8][n] and d_cell[n] = the (i,j) offset
   jj*n1e+ii of the metric record used. */
int harm_b200_mlp_synth(harm_ctx *ctx, size_t n, uint64_t seed, float *d_feat, float *d_targ,
                        double *d_U, double *d_P, int32_t *d_cell);

/* Normalisation record of a training set (means and standard deviations, FP64 sums). */
int harm_b200_mlp_norm(harm_ctx *ctx, size_t n, const float *d_feat, const float *d_targ,
                       float *d_norm);

/* Glorot-uniform weights and zero biases from `seed`. */
int harm_b200_mlp_init(harm_ctx *ctx, uint64_t seed, float *d_params);

/* Loss L = 1/(2n) sum (y - t~)^2 over the standardised targets t~ of the n pairs, and its
   gradient d_grad[HARM_MLP_NPARAMS] (FP32 forward and backward kernels). */
int harm_b200_mlp_loss_grad(harm_ctx *ctx, size_t n, const float *d_feat, const float *d_targ,
                            const float *d_params, const float *d_norm, double *loss,
                            float *d_grad);

/* `steps` Adam steps (beta 0.9/0.999, learning rate lr with cosine decay to lr/100) on
   minibatches of `batch` pairs drawn from the n pairs by a hash of `seed`; d_params is
   updated in place.  loss_hist (host, `steps` floats, may be NULL) receives each step's
   minibatch loss. */
int harm_b200_mlp_train(harm_ctx *ctx, size_t n, const float *d_feat, const float *d_targ,
                        const float *d_norm, float *d_params, int steps, int batch, float lr,
                        uint64_t seed, float *loss_hist);

/* Pack the network for inference (BF16 weights, FP32 biases and normalisation) into the
   context; HARM_GUESS_MLP then uses it.  The Newton iteration starts from
   W' = D exp(log(W'/D)_predicted + start_bias): a small positive bias (a few times the
   network's typical error in log(W'/D)) starts it above the root, the side from which it
   converges without verify_Wlast's tenfold raises of W' (utoprim_jon.c:1120). */
int harm_b200_mlp_set(harm_ctx *ctx, const float *d_params, const float *d_norm,
                      double start_bias);

/* Outputs d_out[n][2] (de-standardised) of the packed network for features d_feat[n][10],
   on the tensor cores of the context's engine (HARM_B200_MLP_ENGINE), as in the inversion. */
int harm_b200_mlp_predict(harm_ctx *ctx, size_t n, const float *d_feat, float *d_out);

/* ------------------------------------------------------------------------------------
 * The reference's main dump file (dump() dump.c:256 through dump_gen dumpgen.c:5) written
 * from device state: the header of dump_header_general (dump.c:320) and, for every active
 * cell in the order k, j, i (i fastest), the 52 columns of dump_content (dump.c:449):
 *   ti tj tk  x1 x2 x3  r th ph  rho u v1 v2 v3 B1 B2 B3  p cs2 Sden  U0..U7  divb
 *   uu0..uu3  ud0..ud3  bu0..bu3  bd0..bd3  v1m v1p v2m v2p v3m v3p  gdet
 * TEXT: the header line and one line of "%21.15g " columns per cell (the reference's default
 * output without MPI-IO); BINARY: header fields and columns as raw native values (the
 * header then has no defcoord); MIXED: the text header and raw columns.
 * d_P: primitives with bounded ghost zones; d_U: the conserved state to record (NULL:
 * primtoU of d_P); t, dt, nstep: the header's time, time step and step count.
 * ------------------------------------------------------------------------------------ */
#define HARM_DUMP_TEXT 0
#define HARM_DUMP_BINARY 1
#define HARM_DUMP_MIXED 2
int harm_b200_dump(harm_ctx *ctx, const double *d_P, const double *d_U, double t, double dt,
                   long nstep, int format, const char *path);

/* Largest grid (extended cells n1e*n2e*n3e) harm_b200_fluxcalc_noalloc accepts: its EMF
   scratch is 3 doubles per cell, 48 MiB at this size. */
#define HARM_NOALLOC_MAX_CELLS 2097152

/* No counterpart in the reference.  fluxcalc for callers that cannot allocate device
   memory (a caller working inside a memory pool it does not own, or a host that forbids
   allocation once its time loop runs): same FP64 fluxes and ndt[3] as harm_b200_fluxcalc
   (every reconstruction and flux method of harm_grid), from caller-provided d_geom (the device copy of the geom table), d_pb and d_F1..d_F3, on
   `stream` (cudaStream_t, NULL for the default stream).  It allocates nothing: the EMF and
   CFL scratch is a file-scope device array that every GPU loading the library holds until
   exit.  Grids above HARM_NOALLOC_MAX_CELLS are rejected (return 2).  All calls share the
   scratch, so calls that overlap on the GPU race.  The call is synchronous: it returns ndt on
   the host, so it waits for its own work on `stream` before returning.  The first call on a
   device looks up the scratch address (cudaGetSymbolAddress) with that device current. */
int harm_b200_fluxcalc_noalloc(const harm_grid *g, const double *d_geom, const double *d_pb,
                               double *d_F1, double *d_F2, double *d_F3, double ndt[3],
                               void *stream);

/* Last CUDA error text of this thread's most recent failing call. */
const char *harm_b200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HARM_B200_H */
