// Internal declarations shared by the host and device translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "senga_gpu.h"

namespace senga {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Records the message as the thread's last error and returns the code.
int fail(int code, const std::string& msg);

// THRD, TTHD, FTHD of the reference (1/3, 2/3, 4/3 formed as it forms them)
constexpr double kThrd = 1.0 / 3.0, kTthd = 2.0 * kThrd, kFthd = 2.0 * kTthd;

// Field slots of the conserved register (reference: DRHS,URHS,VRHS,WRHS,ERHS,
// YRHS(:,:,:,k)).
enum : int { F_RHO = 0, F_RU = 1, F_RV = 2, F_RW = 3, F_RE = 4, F_Y0 = 5 };

// Box geometry handed to every kernel.
struct Geo {
  int nx, ny, nz;
  int64_t n;            // nx*ny*nz
  int per[3];           // 1 = periodic, 0 = bounded (one-sided closures)
  double ovd[3];        // 1/Delta   (OVDELX..)
  double ovd2[3];       // 1/Delta^2 (OVDLX2..)
  int bxl, bxr;         // x-face treatment bits (BF_*), 0 for periodic x
};

// A box split along z into nr slabs of equal extent, one context each
// (senga_zgroup_*): this slab is `rank`; g.nz is the slab's extent, nzg the
// whole box's. The stencil kernels read the z halo of a tile from whichever
// slab owns those planes: base[r] is the element offset from this slab's
// register pool to slab r's (identical layouts), so a halo plane of slab r
// is addressed as base[r] + its local plane offset. nr = 1: one box.
constexpr int kMaxZRanks = 16;
struct ZDec {
  int nr = 1;
  int rank = 0;
  int nzg = 0;
  int64_t base[kMaxZRanks] = {};
};

// Boundary-plane treatment of a bounded x face (src/bcinit.f:287-600 flags):
// which flux derivatives are zeroed on the face plane inside the RHS, and
// whether the NSCBC correction and the imposed-inflow update apply there.
enum : int {
  BF_VSN = 1,       // FxxVSN: normal viscous stress terms (TAUxx,x)
  BF_VST = 2,       // FxxVST: shear viscous stress terms
  BF_CON = 4,       // FxxCON: heat conduction
  BF_DIF = 8,       // FxxDIF and FxxADB: species diffusion and its enthalpy flux
  BF_NSCBC = 16,    // BOUNDS corrections are added to the plane's RHS
  BF_IMPOSED = 32,  // I3 inflow: D, U, V, W, Y are imposed, not integrated
  BF_IMPOSED_D = 64,  // I2 inflow: U, V, W, E, Y are imposed, only D integrated
  BF_WALL = 128,      // W1/W2 wall: U, V, W, E RHS zero; U, V, W not integrated (W2: nor E)
};
__host__ __device__ __forceinline__ int face_bits(const Geo& g, int gx) {
  return gx == 0 ? g.bxl : (gx == g.nx - 1 ? g.bxr : 0);
}

// Device pointers of one box's registers and per-substage scratch.
// 32-bit words of ITNDEX per grid point: base-4 digits, SENGA_NSPIMX species
// a word (src/com_senga2.h:93-98); the words of a field are stored slowest
constexpr int itn_words(int nspec) { return (nspec + SENGA_NSPIMX - 1) / SENGA_NSPIMX; }

struct Fields {
  double* run;    // S register  [nc][n]   (xRUN)
  double* uin;    // U register read this substage  [nc][n] (xRHS on entry)
  double* uout;   // U register written by the RK update
  double* err;    // error register [nc][n] or nullptr (fixed dt)
  double* t;      // TRUN
  int32_t* itn;   // ITNDEX [itn_words(nspec)][n] (2 bits per species, 15 species a word)
  // scratch
  double* p;      // PRUN
  double* lam;    // thermal conductivity lambda
  double* lcp;    // lambda/cp (constant-Lewis transport; TRANSP)
  double* mu;     // viscosity
  double* rd;     // rho*D_k [nspec][n]
  double* h;      // species enthalpy h_k [nspec][n]
  double* hmix;   // mixture enthalpy
  double* wdot;   // CHRATE rate, then species RHS partial [nspec][n]
  double* vel;    // u,v,w [3][n]
  double* e;      // E = rho E / rho
  double* y;      // Y_k [nspec][n]
  double* rhs;    // R(U) [nc][n]
  double* divm;   // DIVM
  double* vc;     // diffusion correction velocity [3][n] (UCOR,VCOR,WCOR)
  double* vtmp;   // divergence of correction flux (VTMP)
  double* mom;    // rho u, rho v, rho w as the thermochemistry kernel read them [3][n]: the
                  // fused species kernel reads these, since its RK pass rewrites U (or nullptr)
  unsigned int* status;  // device status word
  // NSCBC boxes only (nullptr otherwise)
  double* cp;     // cp_mix after TEMPER (STRGxx source)
  double* rmix;   // rho R_mix after TEMPER (STORE7)
  double* face;   // per-face RHS corrections of BOUNDS [2][nc][ny*nz]
};

struct RK {
  double lhs, rhs, err;  // RKLHS, RKRHS, RKERR of this substage (times dt)
  int last;              // 1 on the final substage (FINCOM)
};

// One box of a batched ensemble, as the batched kernels see it.
struct BoxDesc {
  Geo g;
  Fields f;
  RK rk[5];   // RKLHS/RKRHS/RKERR of the five substages (box's own dt)
  int nspec;
  int pad;
};
// One tile of one box (stencil kernels) or one 256-point chunk (pointwise);
// `box` indexes the BoxTable of the launch.
struct WorkItem {
  int box, x0, y0, z0;
};
// The descriptors of up to kTableBoxes boxes, handed to a batched launch by
// value. Kernel parameters live in a read-only constant bank: a tile function
// reads any descriptor field as an operand (or reloads it) instead of holding
// it in a register, as it does for a single-box launch. Larger batches are
// launched as several tables.
constexpr int kTableBoxes = 64;
struct BoxTable {
  BoxDesc d[kTableBoxes];
};
static_assert(sizeof(BoxTable) + 256 <= 32764, "a kernel's parameters are limited to 32764 bytes");

// One persistent launch per RK substage of a batch (persist.cu): the
// phase-major work list of one table's boxes (thermochemistry chunks, flow
// tiles, species tiles, species+RK tiles), where each phase starts (off[0..3];
// off[4] = total), the items of each (box, phase) pair, and the launch's
// counters ([0] dispenser, [1] abort flag, [2 + 4 box + phase] completed
// items), which the launcher zeroes on the stream before the kernel.
constexpr int kPersistCounters = 2 + 4 * kTableBoxes;
struct PersistArgs {
  const WorkItem* items;
  int off[5];
  const int* need;  // [4 * box + phase]
  int* ctr;         // kPersistCounters ints
  int irk;          // substage, 0-based
};
static_assert(sizeof(BoxTable) + sizeof(PersistArgs) + 64 <= 32764, "persistent launch parameters");
// status bit of a persistent launch whose dependency wait ran out
constexpr unsigned kStatusPersistTimeout = 16u;

// Launchers (kernels.cu).
// Mechanism-specialised thermochemistry: 0 = table-driven (any chem.dat),
// otherwise the id of a generated policy whose constants equal the loaded
// tables bit for bit (select_mech). SENGA_MECH=generic in the environment
// forces the table-driven kernel.
int select_mech(const senga_chem& chem, const senga_diff& diff);
// Returns the number of kernels it launched (the long mechanisms run as two).
int launch_thermo(const Geo& g, const Fields& f, const senga_chem* dchem, const senga_diff* ddiff, int nspec,
                  int flmavt, int mech, cudaStream_t s);
void launch_flow(const Geo& g, const Fields& f, int nspec, cudaStream_t s, const ZDec& zd = ZDec{});
void launch_species_a(const Geo& g, const Fields& f, int nspec, cudaStream_t s, const ZDec& zd = ZDec{});
void launch_species_b_rk(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s,
                         const ZDec& zd = ZDec{});
// the species kernel with its x derivatives on the FP64 tensor cores
// (species_mma.cu): all-periodic boxes of one context with extents that are
// multiples of 8; launch_species_a takes it when species_mma_ok
bool species_mma_ok(const Geo& g, const Fields& f, const ZDec& zd);
void launch_species_mma(const Geo& g, const Fields& f, int nspec, cudaStream_t s);
// the species kernel and the species+RK kernel as one (all-periodic boxes of
// one context, when SENGA_FUSE=1 is set): the caller launches it in place of
// both, after the flow kernel (and RADCAL)
bool species_fusable(const Geo& g, const ZDec& zd = ZDec{});
void launch_species_fused(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s);
// species + RK update marching along z (kernels_zmarch.cu); false when the
// box does not qualify (the caller then launches the tiled form)
bool launch_species_b_rk_z(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s,
                           const ZDec& zd);
void launch_deriv(const Geo& g, int kind, const double* in, double* out, cudaStream_t s);
// the same on a halo-extended input (5 points per side), interior output
void launch_deriv_big(const Geo& g, int kind, const double* in, double* out, cudaStream_t s);
// Batched ensemble (kernels.cu, kernels_tiled.cu): all boxes periodic, one
// mechanism; grid = persistent CTA count.
void tile_shape(int* tx, int* ty, int* tz);
int thermo_block();
void launch_batch_thermo(const BoxTable& boxes, const WorkItem* chunks, int nchunks, int grid, int mech,
                         const senga_chem* dchem, const senga_diff* ddiff, int nspec, int flmavt, cudaStream_t s);
// Flow, species and species+RK phases of substage irk (0-based), one CTA per
// work item; `phase` selects one of them (0, 1, 2) or all three (-1).
// resident CTAs per SM of the persistent kernel for a mechanism (occupancy)
int persist_ctas_per_sm(int mech, int nspec, int flmavt);
void launch_batch_persist(const BoxTable& boxes, const PersistArgs& a, int grid, int mech, const senga_chem* dchem,
                          const senga_diff* ddiff, int nspec, int flmavt, cudaStream_t s);
void launch_batch_stencil(const BoxTable& boxes, const WorkItem* items, int nitems, int irk, int phase,
                          cudaStream_t s);
// NSCBC x faces (nscbc.cu): face kinds 0 (none), 11 (I1 inflow), 12 (I2
// inflow), 13 (I3 inflow), 14 (I4 inflow, x-left), 21 (O1 outflow), 31 (W1
// adiabatic no-slip wall), 32 (W2 isothermal no-slip wall), and their
// parameters.
struct NscbcParams {
  int xl, xr;
  double u_in, rho_in, y_in[SENGA_NSPCMX];  // I3: RXLPRM(1), DRIN, YRIN
  double t_in;                              // I2: TRIN
  double t_wall[2];                         // W2: RXLPRM(1), RXRPRM(1)
  double nrieta[6];                         // I4: NRIETA1..6 = RXLPRC(1..6)
  double p_inf, cobc, bet, xlen;            // O1: PINFXR, COBCXR, BET, XGDLEN
  int pio, betloc;                          // O1: NXRPRM(1), NXRPRM(2)
  // synthetic turbulent inflow velocity on an I3 x-left face (BCUTXL NXLPRM(1)
  // = 4): the INFLOW planes of this and the previous step ([ny*nz] each, y
  // fastest), RXLPRM(4) and the current step; nullptr: constant u_in
  const double *uinf1 = nullptr, *uinf2 = nullptr, *vinf1 = nullptr, *vinf2 = nullptr;
  const double *winf1 = nullptr, *winf2 = nullptr;
  double coflow = 0.0, tstep = 0.0;
};
// BOUNDT (both = false) or BOUNTT (both = true: U and S registers, error zeroed)
void launch_boundt(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, bool both,
                   const senga_chem* dchem, cudaStream_t s);
// face data + BOUNDS corrections into f.face, after the thermochemistry kernel
// (zd: a box split along z reads the transverse z derivatives' neighbours,
// and p(1,1,1), from the slabs that own them)
void launch_face(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, const senga_chem* dchem,
                 cudaStream_t s, const ZDec& zd = ZDec{});
// W1/W2 walls: the wall diffusion-flux terms added to the species rate and VTMP
// (after the species kernel), and the wall temperature plus, when rk, the
// zero-gradient mass fractions of the updated state (after the RK update)
bool has_wall(const NscbcParams& bc);
// the synthetic inflow planes of one context (synth_inflow.cu)
struct SynthInflow;
SynthInflow* synth_create(int ny, int nz, const senga_synth_inflow& p, int device);
void synth_destroy(SynthInflow* s);
// INFLOW for the next step: draws the random planes on the host, filters
// them on the device, and points bc at this step's planes
void synth_step(SynthInflow* s, double xgdlen, int nx, double tstep, NscbcParams& bc, cudaStream_t st);
void launch_wall_flux(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, cudaStream_t s);
void launch_wall_fix(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, bool rk, cudaStream_t s);

// RADCAL (radiation.cu): radiating species (0-based), their polynomials,
// gas constants, 4 STEFBO and TREFRN^4.
struct RadParams {
  int nsprad;
  int id[SENGA_NSPCMX], nk[SENGA_NSPCMX];
  double ak[SENGA_NSPCMX][SENGA_NCFRMX], rg[SENGA_NSPCMX];
  double foursb, trfrth;
};
void launch_radcal(const Geo& g, const Fields& f, const RadParams& r, cudaStream_t s);

// Mixture-averaged transport extras (transport.cu): switches, per-species
// bit masks (FLMSOR, FLMDUF, FLMTDR) and scratch. lng/g1/g2 index 0 molar
// mass, 1 pressure, 2 temperature.
struct MixtParams {
  int w, p, t;
  unsigned sor, duf, tdr;
  double* wmix;      // [n]
  double* lng[3];    // [n] each, nullptr when off
  double* g1[3];     // [3][n] first derivatives
  double* g2[3];     // [n] sum of second derivatives (x part zeroed on diffusion-flux faces)
  double* tdrmix;    // [nspec][n], nullptr without Soret/Dufour
};
int launch_mixt(const Geo& g, const Fields& f, const MixtParams& m, const senga_chem* dchem, const senga_diff* ddiff,
                int nspec, cudaStream_t s);

// Post-processing record fields (post.cu): D, u, v, w, E, T, p, Y_k.
void launch_flamin(const Geo& g, int nspec, double xgdlen, double trin, double prin, double drin, double urin,
                   const senga_chem* dchem, const double* v, const double* w, double* run, double* uin, double* t,
                   int32_t* itn, cudaStream_t s);
void launch_tempin(int64_t n, int nspec, const double* U, const senga_chem* dchem, double trin, double* t,
                   int32_t* itn, double* p, unsigned int* status, cudaStream_t s);
void launch_post(int64_t n, int nspec, const double* run, const double* t, const double* p, double* out,
                 cudaStream_t s);

// ADAPTT error maxima (adapt.cu): out[fl] = max |err|/(|run| + nrm.v[fl])
// as the bit pattern of a non-negative double, per conserved field.
struct ErrNorms {
  double v[5 + SENGA_NSPCMX];
};
void launch_errmax(int64_t n, int nc, const double* err, const double* run, const ErrNorms& nrm,
                   unsigned long long* out, int sms, cudaStream_t s);

// Explicit filter (filter.cu): coefficient table of FLINIT, sign-flipped
// when flip (dissipative), and the three-pass filter of one interior field
// (in -> t1 -> t2 -> out; out may alias in).
struct FilterCoef {
  double in[7];       // c1..c6 of the +-m pairs, then c0
  double bnd[6][12];  // one-sided rows of the first/last six points
};
FilterCoef filter_coef(bool flip);
void launch_filter_field(const Geo& g, const double* in, double* out, double* t1, double* t2, const FilterCoef& c,
                         cudaStream_t s);
void launch_chrate_only(const Geo& g, const Fields& f, const senga_chem* dchem, int nspec, cudaStream_t s);

}  // namespace senga
