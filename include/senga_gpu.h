/*
 * senga_gpu.h — C ABI of the B200 (sm_100a) implementation of SENGA2's
 * per-substage right-hand side and low-storage Runge-Kutta advance.
 *
 * Conventions (match the reference's Fortran call surfaces):
 *   - every entry point returns int: 0 = ok, > 0 = error code (see
 *     senga_status below); nothing aborts, no C++ exception crosses the ABI;
 *   - arrays are Fortran column-major (x fastest); an "interior" array has
 *     nx*ny*nz elements (the reference's FDERIV/STD arrays), a species array
 *     is (nx,ny,nz,nspec) with species slowest (the reference's YRUN layout);
 *   - "_host" entry points take host pointers and copy inside the call; the
 *     others take device pointers and run asynchronously on the context's
 *     stream (synchronise with senga_sync);
 *   - the chemistry/transport tables use the reference's COMMON/CHEMIC and
 *     COMMON/DIFFUS array shapes (src/com_senga2.h:121-214), so a Fortran host
 *     can pass its COMMON blocks field by field.
 */
#ifndef SENGA_GPU_H
#define SENGA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Table dimensions: src/com_senga2.h:80-100,189. NSPCMX and NSTPMX are those
 * of the reference's largest shipped case (src/casefiles/68step/com_senga2.h:74),
 * so every mechanism it ships (1, 4, 21, 25 and 68 steps) fits. */
#define SENGA_NSPCMX 18
#define SENGA_NSTPMX 68
#define SENGA_NTINMX 2
#define SENGA_NCOFMX 7
#define SENGA_NSSMAX 10
#define SENGA_NBDYMX 10
#define SENGA_NLLMAX 10
#define SENGA_NDCFMX 4
#define SENGA_NCFRMX 6

/* ITNDEX, the temperature-interval index of every species at a point:
 * base-4 digits, SENGA_NSPIMX species per 32-bit word (src/com_senga2.h:93-98).
 * Every ITNDEX array below holds (nspec + 14) / 15 interior int32 arrays, one
 * per word, words slowest: one array up to 15 species, two for 16 to 18. */
#define SENGA_NSPIMX 15

/* End conditions per face: src/com_senga2.h (NOBC/NBOUND/NPERI) */
#define SENGA_NOBC 0
#define SENGA_NBOUND 1
#define SENGA_NPERI 2

enum senga_status {
  SENGA_OK = 0,
  SENGA_ERR_ARG = 1,        /* bad argument / size                         */
  SENGA_ERR_CUDA = 2,       /* CUDA runtime error                          */
  SENGA_ERR_IO = 3,         /* cannot read an input file                   */
  SENGA_ERR_TEMPER = 4,     /* Newton T inversion did not converge         */
  SENGA_ERR_UNSUPPORTED = 5,/* option not built                            */
  SENGA_ERR_NONFINITE = 6,  /* NaN/Inf detected in the state               */
  SENGA_ERR_NOMEM = 7       /* device memory exhausted                     */
};

/* COMMON/CHEMIC (src/com_senga2.h:121-178) after CHEMIN's derived-quantity
 * pass (src/chemin.f:822-983). C index order [a][b][c] == Fortran (c,b,a). */
typedef struct senga_chem {
  int nspec, nstep, nbody, ngibb, nlind, ntroe, nsrif;
  int ntint[SENGA_NSPCMX];
  int ncofcp[SENGA_NSPCMX][SENGA_NTINMX], ncpoly[SENGA_NSPCMX][SENGA_NTINMX];
  int ncpom1[SENGA_NSPCMX][SENGA_NTINMX], ncenth[SENGA_NSPCMX][SENGA_NTINMX];
  int ncenpy[SENGA_NSPCMX][SENGA_NTINMX];
  int nsslen[SENGA_NSTPMX], nrslen[SENGA_NSTPMX], npslen[SENGA_NSTPMX];
  int nrclen[SENGA_NSTPMX], npclen[SENGA_NSTPMX];
  int nsspec[SENGA_NSTPMX][SENGA_NSSMAX], nrspec[SENGA_NSTPMX][SENGA_NSSMAX];
  int npspec[SENGA_NSTPMX][SENGA_NSSMAX], nrcpec[SENGA_NSTPMX][SENGA_NSSMAX];
  int npcpec[SENGA_NSTPMX][SENGA_NSSMAX];
  int mblist[SENGA_NSTPMX], mglist[SENGA_NSTPMX], mllist[SENGA_NSTPMX];
  int mtlist[SENGA_NSTPMX], mslist[SENGA_NSTPMX];
  double prefgb, alamda;
  double tintlo[SENGA_NSPCMX][SENGA_NTINMX], tinthi[SENGA_NSPCMX][SENGA_NTINMX];
  double amolcp[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double amolgb[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double amascp[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double amasct[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double amasch[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double amascs[SENGA_NSPCMX][SENGA_NTINMX][SENGA_NCOFMX];
  double rparam[SENGA_NSTPMX][3];
  double rclind[SENGA_NLLMAX][4], rctroe[SENGA_NLLMAX][12], rcsrif[SENGA_NLLMAX][8];
  double diffmu[SENGA_NSTPMX][SENGA_NSSMAX], diffmw[SENGA_NSTPMX][SENGA_NSSMAX];
  double crspec[SENGA_NSTPMX][SENGA_NSSMAX], cpspec[SENGA_NSTPMX][SENGA_NSSMAX];
  double effy3b[SENGA_NBDYMX][SENGA_NSPCMX];
  double wmolar[SENGA_NSPCMX], ovwmol[SENGA_NSPCMX], rgspec[SENGA_NSPCMX];
  double clewis[SENGA_NSPCMX], olewis[SENGA_NSPCMX];
} senga_chem;

/* COMMON/DIFFUS (src/com_senga2.h:189-214) after DIFFIN's derived pass
 * (src/diffin.f:328-405). flmavt = 0 selects constant-Lewis transport. */
typedef struct senga_diff {
  int flmavt, ncodif, ncotdr, ncovis, ncocon;
  double pdifgb, tdifgb;
  double diffco[SENGA_NSPCMX][SENGA_NSPCMX][SENGA_NDCFMX];
  double tdrcco[SENGA_NSPCMX][SENGA_NSPCMX][SENGA_NDCFMX];
  double wilko1[SENGA_NSPCMX][SENGA_NSPCMX], wilko2[SENGA_NSPCMX][SENGA_NSPCMX];
  double viscco[SENGA_NSPCMX][SENGA_NDCFMX], condco[SENGA_NSPCMX][SENGA_NDCFMX];
} senga_diff;

/* Run configuration of one box (cont.dat's grid, domain, BC and dt lines). */
typedef struct senga_config {
  int nx, ny, nz;              /* grid points (NXGLBL..; one rank)          */
  double xgdlen, ygdlen, zgdlen; /* domain lengths [m]; spacing L/(N-1)    */
  int nend[6];                 /* NENDXL,XR,YL,YR,ZL,ZR: SENGA_NPERI/NBOUND */
  double tstep;                /* fixed time step TSTEP [s]                 */
  int adaptive;                /* 1: keep the RK error register (ADAPTT)    */
  int device;                  /* CUDA device ordinal                       */
} senga_config;

typedef struct senga_ctx senga_ctx;

/* ---- tables: host-side CHEMIN / DIFFIN ------------------------------------
 * senga_chem_load restates chem.dat reading (src/chemin.f:146-344) and the
 * derived-table pass (src/chemin.f:822-983).
 * senga_diff_load restates diff.dat reading (src/diffin.f:100-232) and the
 * derived pass (src/diffin.f:328-405); pass path=NULL for constant-Lewis
 * transport (NFMAVT=0, src/diffin.f:65). */
int senga_chem_load(const char* path, senga_chem* out);
int senga_diff_load(const char* path, const senga_chem* chem, senga_diff* out);

/* ---- context: device-resident state for one box ---------------------------
 * Replaces the reference's COMMON-resident registers xRUN/xRHS/xERR, TRUN and
 * ITNDEX (src/com_senga2.h:576-679) with HBM-resident SoA fields. */
int senga_ctx_create(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff,
                     senga_ctx** out);
int senga_ctx_destroy(senga_ctx* ctx);
const char* senga_last_error(void);
int senga_sync(senga_ctx* ctx);
/* device pointer to the context's stream (cudaStream_t) */
void* senga_stream(senga_ctx* ctx);

/* Upload/download the conserved state (rho, rho u, rho v, rho w, rho E,
 * rho Y_1..rho Y_n; nc = 5+nspec interior arrays, field slowest), the
 * temperature seed TRUN and the thermo interval index ITNDEX. Upload sets both
 * RK registers (xRUN = xRHS), as at the end of FINCOM (src/fincom.f:54-168)
 * and after INDATA (src/indata.f:1540-1565). */
int senga_upload_state_host(senga_ctx* ctx, const double* fields, const double* trun, const int32_t* itndex);
int senga_download_state_host(senga_ctx* ctx, double* fields, double* trun, int32_t* itndex);
/* Stream-ordered forms of the two copies: they return at once, queued on the
 * context's stream before/after whatever is launched next (senga_step_graph
 * also returns without waiting). With page-locked host buffers the copies
 * then run on the copy engines while other contexts compute, so a caller
 * with a queue of independent boxes keeps the link and the SMs busy at the
 * same time. The host buffers must stay untouched until senga_sync(ctx). */
int senga_upload_state_async(senga_ctx* ctx, const double* fields, const double* trun, const int32_t* itndex);
int senga_download_state_async(senga_ctx* ctx, double* fields, double* trun, int32_t* itndex);

/* One RK substage (irkstp = 1..5): BOUNDT, PARFER, RHSCAL, RHSVEL, BOUNDS and
 * LINCOM (irkstp < 5) or FINCOM (irkstp = 5): src/senga2.f:113-159. */
int senga_substage(senga_ctx* ctx, int irkstp);
/* nsteps full RK steps (5 substages each, src/senga2.f:96-194; the filter
 * call at src/senga2.f:178 is commented out in the reference and not run). */
int senga_step(senga_ctx* ctx, int nsteps);
/* Capture one full RK step as a CUDA graph and replay it nsteps times. */
int senga_step_graph(senga_ctx* ctx, int nsteps);

/* RHSCAL + RHSVEL on the current U register without the RK update:
 * rhs (nc interior arrays) = R(U); optional trun/prun outputs after TEMPER.
 * Host pointers. */
int senga_rhs_host(senga_ctx* ctx, double* rhs, double* trun, double* prun);

/* One RK step (5 substages) with CUDA events around every kernel launch on
 * the context's stream; ms[4] receives the summed time of the four kernel
 * families (thermo, flow, species_a, species_b+RK), *launches their count.
 * With the species kernels fused (senga_ctx_species_fused) the one species
 * launch is timed as species_a and ms[3] holds only the face kernels, if any.
 * Advances the state like senga_step(ctx, 1). */
int senga_profile_step(senga_ctx* ctx, double* ms, int* launches);
/* *fused_kernels = 1 when the context runs the species kernel and the
 * species+RK kernel as one launch per substage: all-periodic boxes without
 * the transport switches when SENGA_FUSE=1 is set (the rates, correction
 * velocity, VTMP and energy RHS then stay on chip between the two passes;
 * off by default, since the two kernels measure faster). */
int senga_ctx_species_fused(senga_ctx* ctx, int* fused_kernels);
/* *mma = 1 when the context's species kernel takes its x derivatives on the
 * FP64 tensor cores (band-matrix mma): all-periodic boxes of one context
 * whose extents are multiples of 8, when SENGA_SPECIES_MMA=1 is set (read at
 * every launch or graph capture; off by default, since the stencil form
 * measures faster); the other boxes run the stencil form. */
int senga_ctx_species_mma(senga_ctx* ctx, int* mma);

/* Context facts: *mech = thermochemistry kernel in use (0 table-driven, 1 the
 * generated one-step R->P kernel, 2 the generated H2/air kernel), and the
 * device bytes the context holds. */
int senga_ctx_info(senga_ctx* ctx, int* mech, int64_t* device_bytes);

/* Measured FP64 FMA throughput of the device in TFLOP/s (independent FMA
 * chains on every SM): the denominator of the FP64-pipe roofline of the
 * pointwise thermochemistry kernel. No counterpart in the reference. */
int senga_fp64_peak(int device, double* tflops);

/* Status word of the last steps: bit 0 = TEMPER non-convergence; bit 1 =
 * TEMPIN found no sign change of the energy residual in [200, 3000] K (the
 * reference stops there); bit 2 = TEMPIN still unconverged after 200
 * bisections (the reference bisects without limit); bit 3 = a stencil tile's
 * bulk copies did not land within about a second (the tile's results are
 * not written); bit 4 = a wait of the persistent batch kernel ran out (the
 * launch was abandoned). */
int senga_get_status(senga_ctx* ctx, int* status);

/* ---- operator-level entry points (unit parity) -----------------------------
 * DFBYDX/DFBYDY/DFBYDZ(FUNCTN, FDERIV): src/dfbydx.f:36-37,53-238
 * D2FDX2/D2FDY2/D2FDZ2: src/d2fdx2.f:54-270
 * D2FDXY/D2FDXZ/D2FDYZ: src/d2fdxy.f:55-1937
 * kind: 0 dx, 1 dy, 2 dz, 3 dxx, 4 dyy, 5 dzz, 6 dxy, 7 dxz, 8 dyz.
 * f and out are interior arrays (device pointers); periodic directions are
 * wrapped in place of the reference's halo copy. Any direction may be
 * bounded (NBOUND on both faces): one-sided closures, and for the mixed
 * derivatives the end rows of either direction and the corner schemes
 * where both are bounded. A context bounded in y or z runs these operators
 * and the filter only (the RHS entry points return SENGA_ERR_UNSUPPORTED:
 * no y/z face conditions are built). */
int senga_deriv(senga_ctx* ctx, int kind, const double* f, double* out);

/* TEMPIN (src/tempin.f:58-524): start-up temperature of the state in the
 * context (the conserved fields as uploaded, e.g. a restart dump, which
 * carries no temperature). Per point the energy residual
 * sum_k rhoY_k e_k(T) + 1/2 rho|u|^2 - rho E is bracketed from the guess trin
 * (cont.dat's TRIN) in 50 K steps inside [200, 3000] K and bisected until it
 * is below 1e-4; TRUN, ITNDEX and PRUN are set on the device, and copied to
 * trun, itndex and prun (host arrays of the interior, each may be NULL).
 * Failures set status bits 1 and 2 (senga_get_status) instead of stopping. */
int senga_tempin_host(senga_ctx* ctx, double trin, double* trun, int32_t* itndex, double* prun);

/* Initial flame FLAMIN (src/flamin.f:44-322) and INDATA's conversion of the
 * start-up primitives to the conserved state (src/indata.f:1233-1394), on the
 * device: a planar flame across x, progress (1 + erf((x - 5 mm)/0.5 mm))/2,
 * between the reactant (Y_1 = 0.011606960, Y_2 = 0.230295282, T = trin) and
 * the product (Y_2 = 0.139255233, Y_3 = 0.102581446, T = 1417.2 K) states as
 * the reference codes them (the last species the remainder), pressure prin,
 * u = drin urin / rho, v and w from the host arrays (interior, NULL = 0).
 * Sets both registers, TRUN and ITNDEX, as senga_upload_state_host would. */
int senga_flamin(senga_ctx* ctx, double trin, double prin, double drin, double urin, const double* v,
                 const double* w);
int senga_deriv_host(senga_ctx* ctx, int kind, const double* f, double* out);
/* The same nine operators on the reference's own argument shapes
 * (src/dfbydx.f:36-37): f_big is FUNCTN(NXBIGL:NXBIGR, NYBIGL:NYBIGR,
 * NZBIGL:NZBIGR) with NHALO = 5 points on every side, i.e. (nx+10)(ny+10)
 * (nz+10) doubles, x fastest, the interior starting at offset 5 in each
 * direction; out is FDERIV(NXSIZE, NYSIZE, NZSIZE), the nx*ny*nz interior.
 * Periodic directions read their neighbours from the halo as the caller
 * filled it (PARFER's periodic copies, or a neighbour rank's planes), as the
 * reference does; bounded directions use the one-sided closures and never
 * read their halo. senga_deriv_big takes device pointers (asynchronous on
 * the context's stream), senga_deriv_big_host host pointers. */
int senga_deriv_big(senga_ctx* ctx, int kind, const double* f_big, double* out);
int senga_deriv_big_host(senga_ctx* ctx, int kind, const double* f_big, double* out);

/* Mixture-averaged transport switches of cont.dat's transport line
 * (NFMIXW, NFMIXP, NFMSOR, NFMDUF, WMLTDR; src/contin.f:205): molar-mass
 * (src/rhscal.f:1966-2357), pressure (:2361-2757) diffusion, Soret
 * (:2760-3765) and Dufour (:1552-1564) terms; the last two for the species
 * with W_k <= WMLTDR + 1e-3 (src/diffin.f:384-406). Needs a diff.dat
 * (flmavt). All zero turns them off (the default). */
int senga_set_transport(senga_ctx* ctx, int mixw, int mixp, int soret, int dufour, double wmltdr);

/* Optically thin radiation heat loss, RADCAL (src/radcal.f:45-119), run when
 * the cont.dat radiation switch is on (src/rhscal.f:810):
 * ERHS -= 4 STEFBO sum_j a_j(T) rho Y_j R_j T (T^4 - TREFRN^4), with the
 * Planck-mean absorption polynomials a_j of the radiating species read from
 * radn.dat by senga_radn_load (RADCIN, src/radcin.f:57-200; species indices
 * 1-based as in the file) and trefrn the cont.dat reference temperature.
 * senga_set_radiation(ctx, NULL) turns it off (the default). */
typedef struct senga_radn {
  int nsprad;                                   /* radiating species (NSPRAD) */
  int nsprid[SENGA_NSPCMX];                     /* their species indices, 1-based */
  int nkprad[SENGA_NSPCMX];                     /* coefficients per polynomial */
  double akprad[SENGA_NSPCMX][SENGA_NCFRMX];    /* AKPRAD(icoeff, j) as [j][icoeff] */
  double trefrn;                                /* TREFRN [K] */
} senga_radn;
int senga_radn_load(const char* path, const senga_chem* chem, double trefrn, senga_radn* out);
int senga_set_radiation(senga_ctx* ctx, const senga_radn* radn);

/* NSCBC x faces (bounded x, NBOUND on both x faces; y, z periodic). xl and
 * xr each take one of the built kinds; inflow on one face at most.
 * 11: I1 subsonic non-reflecting laminar inflow (NSBCI1), no parameters:
 *   nothing is imposed; the incoming wave amplitude is the chemistry source
 *   term alone (its pressure-relaxation coefficient COBCxx is set by BCINIT
 *   only for an O1 face, so it is zero), the transverse and species waves
 *   are zero, and every conserved right-hand side of the plane is corrected
 *   (BOUNDS src/bounds.f:387-520 left, 1465-1598 right); normal viscous
 *   stress zeroed on the plane (FxxVSN, src/bcinit.f:396-407).
 * 14: I4 inflow after Lodato et al. (NSBCI4), coded in the reference for
 *   the x-left face only (bounds.f:686-845; flags src/bcinit.f:653-658):
 *   nothing imposed; the waves L2..L5 and LY are relaxed towards the targets
 *   u = u_in, v = w = 0, T = t_in, Y = y_in (BCUTXL NXLPRM(1)=1, BCTTXL,
 *   BCYTXL) with the coefficients nrieta[1..5] (NRIETA2..6 = RXLPRC(2..6))
 *   over XGDLEN, plus the transverse terms TT2..TT6 of the face (bounds.f:
 *   185-204); L1 leaves unchanged; normal viscous stress zeroed on the plane.
 *   An I4 face on x-right returns SENGA_ERR_UNSUPPORTED.
 * 12: I2 subsonic reflecting inflow with specified temperature (NSBCI2):
 *   u = u_in (constant, NXxPRM(1)=1; negative through x-right), v = w = 0,
 *   T = t_in (TRIN) and the mass fractions y_in imposed on the inflow plane
 *   from its current density, which alone is integrated there (BOUNDT
 *   src/boundt.f:81-176 left, 495- right; BOUNTT src/bountt.f:84-200 left,
 *   590- right; ranges src/bcinit.f:458-480), its right-hand side corrected
 *   by the wave amplitudes of BOUNDS (src/bounds.f:522-608 left, 1600-1684
 *   right).
 * 13: I3 subsonic inflow with constant velocity (NXxPRM(1)=1): u = u_in
 *   (negative for inflow through x-right), v = w = 0, density rho_in (DRIN),
 *   mass fractions y_in (YRIN) imposed on the inflow plane (BOUNDT
 *   src/boundt.f:177-200 left, 591- right; BOUNTT src/bountt.f:203-252 left,
 *   709- right; RK ranges src/bcinit.f:560-586), energy by the wave
 *   amplitudes of BOUNDS (src/bounds.f:610-675 left, 1688- right).
 * 21: O1 partially non-reflecting outflow: pressure relaxed to p_inf with
 *   COBC = sigma (1 - eta) / (2 XGDLEN) (RXxPRM(1..3)), pio = NXxPRM(1)
 *   (inflow-through-outlet switch), bet_local = NXxPRM(2) (local Mach number
 *   in place of BET = 0.05 on the transverse terms), BOUNDS
 *   src/bounds.f:213-372 left, 1296-1450 right; viscous shear, conduction
 *   and diffusion zeroed on the plane (FxxVST, FxxCON, FxxDIF, FxxADB). Two
 *   O1 faces share these parameters.
 * 31: W1 adiabatic no-slip wall (NSBCW1), on either or both faces, no
 *   parameters: the wall temperature is the zero-gradient extrapolation
 *   (48 T1 - 36 T2 + 16 T3 - 3 T4)/25 of the four planes inward, momentum
 *   is zero and rho E the internal energy at that temperature (BOUNDT
 *   src/boundt.f:243-356 left, 657-768 right; BOUNTT src/bountt.f:290-428,
 *   767-); the density and species right-hand sides take the reflected
 *   wave of BOUNDS (src/bounds.f:917-1056, 1833-1974), momentum and energy
 *   right-hand sides are zero; the wall diffusion flux enters the species
 *   rates (src/rhscal.f:1698-1760); after each RK update every wall mass
 *   fraction is the clipped zero-gradient extrapolation of the updated
 *   state (src/lincom.f:171-210, src/fincom.f:171-210). Conduction and
 *   diffusion are zeroed on the plane (FxxCON, FxxDIF, FxxADB). With the
 *   senga_set_transport switches on, the molar-mass, pressure and Soret
 *   branches add their own wall terms to the wall's species rates
 *   (src/rhscal.f:2116-2175, 2512-2571, 2925-2984); their energy parts and
 *   the Dufour wall terms reach only the wall's energy right-hand side,
 *   which is zero.
 * 32: W2 isothermal no-slip wall (NSBCW2), on either or both faces: the
 *   wall temperature t_wall[side] is imposed with zero momentum and rho E
 *   the internal energy at it, on the U register by BOUNDT and on both
 *   registers by BOUNTT (src/boundt.f:358-470, src/bountt.f:429-560 and
 *   their x-right blocks); neither momentum nor energy is integrated on the
 *   wall (ranges src/bcinit.f:822-855); the density and species take the
 *   reflected wave as for W1 (src/bounds.f:1058-1190, 1975-), the wall
 *   diffusion flux and the zero-gradient mass fractions as for W1; only
 *   diffusion is zeroed on the plane (FxxDIF). The transport switches add
 *   their wall terms as for W1.
 * Face data and wave amplitudes are computed after the thermochemistry
 * kernel and added to the face planes' right-hand side in the RK epilogue.
 * rho_in must be > 0 with an I3 face, p_inf > 0 with an O1 face, t_wall > 0
 * on a W2 face.
 * Other face kinds return SENGA_ERR_UNSUPPORTED. Stepping a box with a
 * bounded x direction needs this call first. */
typedef struct senga_nscbc {
  int xl, xr;
  double u_in, rho_in;
  double y_in[SENGA_NSPCMX];
  double p_inf, sigma, eta;
  int pio, bet_local;
  double t_in;      /* I2: imposed inflow temperature TRIN [K] */
  double t_wall[2]; /* W2: wall temperature of the x-left, x-right face (RXLPRM(1), RXRPRM(1)) [K] */
  double nrieta[6]; /* I4: relaxation coefficients NRIETA1..6 = RXLPRC(1..6) (the first is unused) */
} senga_nscbc;
int senga_set_nscbc(senga_ctx* ctx, const senga_nscbc* bc);

/* Synthetic turbulent inflow velocity on an I3 inflow at x-left: the
 * reference's digital filter (src/inflow.f, M. Klein's method) with the
 * velocity option of BCUTXL NXLPRM(1) = 4 (src/bcutxl.f:476-510). Every RK
 * step first draws three random planes with the reference's RAN1 (host,
 * serial), filters them with Gaussian kernels of length scales lny, lnz (in
 * grid spacings; half-widths nfy, nfz) on the device, correlates them in
 * time over lnx spacings of the mean inflow u_in, and removes their face
 * means; the face then takes u = u_in + u' + coflow, v = v', w = 0 and the
 * matching time derivatives. Velocity only (NXLPRM(2) = 0); the reference's
 * PARAMETERs are lnx = lny = lnz = 30, nfy = nfz = 60. itime is the step
 * number of the next step (ITIME, which seeds RAN1 each step). Set after
 * senga_set_nscbc; the steps then run without graph capture (the random
 * planes are drawn on the host every step). */
typedef struct senga_synth_inflow {
  double urms;   /* RXLPRM(2): fluctuation amplitude [m/s] */
  double coflow; /* RXLPRM(4): added to the inflow velocity [m/s] */
  int lnx, lny, lnz;
  int nfy, nfz;
  int itime;
} senga_synth_inflow;
int senga_set_synthetic_inflow(senga_ctx* ctx, const senga_synth_inflow* p);

/* Adaptive time step (cfg.adaptive = 1, the reference's NSTPSW = 1):
 * ADAPTT (src/adaptt.f:53-330) runs after every step of senga_step /
 * senga_step_graph (the latter then launches kernels per step, since dt
 * changes): per-field maxima of |ERR|/(|RUN|+norm) on the device, the PID
 * controller of DTINIT (src/dtinit.f:99-175) on the host, RK coefficients
 * rescaled, error register zeroed. This returns the current TSTEP, the last
 * ERRMAX and INDERR (-4 rho, -1..-3 momentum, 0 energy, k species). */
int senga_get_tstep(senga_ctx* ctx, double* tstep, double* errmax, int* inderr);

/* Explicit filter FLTREM (src/fltrem.f:43-90) of the U register (xRHS):
 * FILTRX -> FILTRY -> FILTRZ (src/filtrx.f:56-295) on every conserved field,
 * 12th-order interior, 6th..11th-order one-sided rows on bounded faces,
 * coefficients of FLINIT (src/flinit.f:42-…). The reference never calls it
 * (src/senga2.f:178 is commented out); a host calls this after a step, e.g.
 * every 10 steps. mode bit 0: flip the sign of TWFACT (the coded sign
 * amplifies the grid-scale mode; flipped, the filter damps it); bit 1: also
 * filter the S register (xRUN), which the reference leaves unfiltered.
 * Periodic neighbours at +-6 are reached by index wrap. */
int senga_filter(senga_ctx* ctx, int mode);
/* The three-pass filter of one interior field (host pointers). */
int senga_filter_field_host(senga_ctx* ctx, int mode, const double* f, double* out);

/* TEMPER (src/temper.f:58-219) on the current U register; host outputs of
 * T and p (either may be NULL). CHRATE (src/chrate.f:146-741) on the current U
 * register and T: host output of RATE (nspec interior arrays). */
int senga_temper_host(senga_ctx* ctx, double* trun, double* prun);
int senga_chrate_host(senga_ctx* ctx, double* rate);

/* Integrate FUNCTN over [argmin,argmax] by successive Simpson refinement
 * (INTEGF, src/integf.f:57-96): host-side helper used by initial-condition
 * generation (init only, never per substage). */
typedef double (*senga_integrand)(double x, void* user);
int senga_integf(senga_integrand f, void* user, double argmin, double argmax, double* answer);

/* ---- restart dumps ---------------------------------------------------------
 * The reference's dump file of one rank, written by src/output.f:296-322 and
 * read back by src/indata.f:1405-1436: NXNODE, NYNODE, NZNODE, NSPEC, then
 * DRUN, URUN, VRUN, WRUN, ERUN, YRUN (the whole YRUN(..., NSPCMX) array of
 * COMMON, so nspcmx is the reference build's NSPCMX), then ETIME, TSTEP,
 * ERROLD, ERRLDR. formatted = 0: one sequential unformatted record (4-byte
 * length markers, sub-records beyond 2 GB; NDOFMT/NDIFMT = 0); formatted = 1:
 * list-directed text, one line per point (NDOFMT/NDIFMT = 1).
 * fields: (5 + nspec) interior arrays, x fastest, field slowest (the layout
 * of senga_upload_state_host); scalars[4] = ETIME, TSTEP, ERROLD, ERRLDR.
 * senga_dump_read with fields = NULL only returns dims[4] (nx, ny, nz,
 * nspec); capacity is the number of doubles fields can hold. */
int senga_dump_write(const char* path, int formatted, int nx, int ny, int nz, int nspec, int nspcmx,
                     const double* fields, const double* scalars);
int senga_dump_read(const char* path, int formatted, int nspcmx, int* dims, double* fields, int64_t capacity,
                    double* scalars);

/* ---- one box split along z over several contexts --------------------------
 * No counterpart call in the reference, whose MPI decomposition (PARFER halo
 * exchange, src/parfer.f) it replaces: nslabs contexts (devices[r], or
 * cfg->device for all when devices is NULL) each own nz/nslabs planes of one
 * periodic box; the stencil kernels read each tile's z halo directly from the
 * slab that owns those planes (peer loads between GPUs, with peer access
 * enabled at creation), and the slabs' streams wait on one another's events
 * between the phases of every substage. Boxes periodic in y and z (x
 * periodic, or bounded with NSCBC faces: senga_zgroup_set_nscbc) with a fixed
 * time step; fields/trun/itn are the whole box in the senga_upload_state_host
 * layout. */
typedef struct senga_zgroup senga_zgroup;
int senga_zgroup_create(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff, int nslabs,
                        const int* devices, senga_zgroup** out);
/* NSCBC x faces of a z-split box (x bounded on both faces, cfg.nend): the
 * same conditions as senga_set_nscbc, set on every slab (each holds its
 * ny x nz/nslabs part of both x faces); needed before the first step. The
 * transport switches and radiation are not available on a z-split box. */
int senga_zgroup_set_nscbc(senga_zgroup* g, const senga_nscbc* bc);
int senga_zgroup_upload_host(senga_zgroup* g, const double* fields, const double* trun, const int32_t* itndex);
int senga_zgroup_step(senga_zgroup* g, int nsteps);
int senga_zgroup_sync(senga_zgroup* g);
int senga_zgroup_download_host(senga_zgroup* g, double* fields, double* trun, int32_t* itndex);
int senga_zgroup_destroy(senga_zgroup* g);

/* ---- initial turbulence ---------------------------------------------------
 * TURBIN (src/turbin.f:76-362, with TURBFT/FFTSYM and ESPECT/ESPINI) for one
 * box on the current device: a solenoidal velocity field built in
 * wavenumber space (Rogallo) from the RANINI/RANUNI stream seeded with
 * inseed, spectrum E(k) = const0/ck0 (k/ck0)^4 exp(-2 (k/ck0)^2) in integer
 * wavenumbers (SPARAM(1), SPARAM(2) of cont.dat), then transformed to
 * physical space. uvw receives 3 arrays (u, v, w; x fastest) of
 * nx*ny*nz doubles, the field TURBIN leaves in URUN/VRUN/WRUN before INDATA
 * adds the mean velocity (src/indata.f:1111-1141); imag_max (optional) the
 * largest imaginary part left by the transform. Extents 2..1024. */
int senga_turbin_host(int nx, int ny, int nz, int inseed, double const0, double ck0, double* uvw, double* imag_max);

/* ---- post-processing output ------------------------------------------------
 * The record written every NTDUMP steps for post-processing
 * (src/output.f:240-265, file output/out<IDDUMP:5><IPROC:4>.res): DRUN,
 * URUN/DRUN, VRUN/DRUN, WRUN/DRUN, ERUN/DRUN, TRUN, PRUN, YRUN/DRUN (NSPEC
 * fields), RRTE (NSPCMX fields) and ETIME, one unformatted record.
 * senga_keep_rates(ctx, 1) makes every substage keep its CHRATE rates
 * (RRTE, src/rhscal.f:828); senga_post_fields_host then fills post with
 * (7 + 2 nspec) interior arrays (the primitives formed on the device, then
 * RRTE_1..RRTE_nspec); senga_post_write / senga_post_read write and read the
 * file (no size header: the sizes are the caller's). */
int senga_keep_rates(senga_ctx* ctx, int on);
int senga_post_fields_host(senga_ctx* ctx, double* post);
int senga_post_write(const char* path, int nx, int ny, int nz, int nspec, int nspcmx, const double* post,
                     double etime);
int senga_post_read(const char* path, int nx, int ny, int nz, int nspec, int nspcmx, double* post, double* etime);

/* ---- batched ensembles --------------------------------------------------------
 * No counterpart in the reference (it runs one box per MPI job). Many
 * independent periodic boxes of uneven sizes, one mechanism, each with its own
 * dt (cfgs[i].tstep). A substage runs in one of two forms, per table of up to
 * 64 boxes: one persistent launch whose resident CTAs take every box's
 * thermochemistry chunks, flow, species and species+RK tiles from one
 * phase-major device work list (each phase of a box starts when the box's
 * previous phase has completed; bounded waits, status bit 4 on time-out), or
 * four launches (a pointwise kernel striding over 256-point chunks, then one
 * CTA per (box, tile) item for each stencil kernel). The RK step is captured
 * once as a CUDA graph. senga_batch_autotune times one RK step of the
 * uploaded state (saved and restored) for each candidate (the persistent
 * kernel at 1..k resident CTAs per SM, the four launches at several pointwise
 * grid sizes) and keeps the fastest; it reports the number of stencil CTAs
 * per launch of the four-launch form and the pointwise grid; senga_batch_form
 * reports the form in use (persistent = 1) and its grid. SENGA_BATCH=persist
 * or =launches in the environment (read at senga_batch_create) keeps the
 * batch, and its autotuner, to one form; unset, the four launches run until
 * the autotuner picks. */
typedef struct senga_batch senga_batch;
int senga_batch_create(int nbox, const senga_config* cfgs, const senga_chem* chem, const senga_diff* diff,
                       int device, senga_batch** out);
int senga_batch_destroy(senga_batch* b);
int senga_batch_upload_host(senga_batch* b, int ibox, const double* fields, const double* trun,
                            const int32_t* itndex);
int senga_batch_download_host(senga_batch* b, int ibox, double* fields, double* trun, int32_t* itndex);
int senga_batch_step(senga_batch* b, int nsteps);
int senga_batch_autotune(senga_batch* b, int* grid_stencil, int* grid_thermo);
int senga_batch_form(senga_batch* b, int* persistent, int* grid);
int senga_batch_sync(senga_batch* b);
void* senga_batch_stream(senga_batch* b);
int senga_batch_status(senga_batch* b, int* status);

/* ---- serving loop ---------------------------------------------------------------
 * No counterpart in the reference. Continuous batching of DNS requests: a
 * request (one periodic box, its initial state and a number of RK steps) is
 * admitted, first come first served, as soon as the device arena of
 * arena_bytes has room for its fields; all admitted requests advance one RK
 * step per senga_server_tick in one batched launch sequence; finished
 * requests are copied back and their memory freed. A tick queues its step
 * and returns: it waits on the device only while two steps are already in
 * flight. Uploads and results pass through a page-locked staging ring, and
 * a request counts as active (senga_server_result refuses it) until its
 * result has landed in host memory; *finished counts the results that
 * landed during the tick. Times are seconds since creation. */
typedef struct senga_server senga_server;
int senga_server_create(size_t arena_bytes, const senga_chem* chem, const senga_diff* diff, int device,
                        senga_server** out);
int senga_server_destroy(senga_server* s);
int senga_server_submit(senga_server* s, const senga_config* cfg, const double* fields, const double* trun,
                        const int32_t* itndex, int nsteps, int* request_id);
int senga_server_tick(senga_server* s, int* finished);
int senga_server_result(senga_server* s, int request_id, double* fields, double* trun, int32_t* itndex,
                        double* times);
int senga_server_stats(senga_server* s, int* active, int* pending, int64_t* gpsu, int64_t* free_bytes);
/* Caps the grid points advanced per tick (admission stops once the active
 * requests hold that many points; a lone request is always admitted). 0
 * (the default) admits while the arena has room. With a cap, requests run
 * nearly in arrival order instead of all sharing one long tick, which
 * lowers the median time to completion under overload. */
int senga_server_set_max_points(senga_server* s, int64_t max_points);

/* ---- allocation-free right-hand side ----------------------------------------
 * No counterpart in the reference. RHSCAL + RHSVEL of one periodic box, like
 * senga_rhs_host, for callers that cannot allocate device memory when they
 * call (a host that reserves all device memory at start-up, or one that runs
 * inside another framework's memory pool): all arrays are caller-owned
 * device pointers and the intermediate fields live in a fixed file-scope
 * device array of SENGA_NOALLOC_SCRATCH_BYTES, held by every GPU that loads
 * the library until exit. No cudaMalloc/cudaFree is called.
 *   state  : nc = 5+nspec conserved interior arrays (read)
 *   trun   : T seed in, T after TEMPER out;  itndex: interval index in/out
 *   rhs    : nc interior arrays, R(U) out
 *   status : device word (required), bit 0 set on TEMPER non-convergence
 *            (cleared by the call)
 *   stream : cudaStream_t to run on (NULL = default stream); asynchronous.
 * Periodic boxes of any extent (one point in the unused directions of 1D and
 * 2D runs). A box needs (14 + 4*nspec)*8 bytes of scratch per grid point;
 * larger boxes are rejected with SENGA_ERR_ARG. Every call reuses the same
 * array, so calls that overlap on the GPU race. The tables are copied from
 * the host structs at every call, so the call cannot be captured into a CUDA
 * graph: on a capturing stream it returns SENGA_ERR_UNSUPPORTED and queues
 * nothing. The first call on a device (with it current) looks up the
 * array's device address. Under CUDA's lazy module loading (the default) that first
 * call is also when the array and the kernels' code are loaded onto the
 * device: a host that reserves all free device memory at start-up makes one
 * call per device before it does (or sets CUDA_MODULE_LOADING=EAGER). */
#define SENGA_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int senga_rhs_noalloc(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff,
                      const double* state, double* trun, int32_t* itndex, double* rhs,
                      unsigned int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SENGA_GPU_H */
