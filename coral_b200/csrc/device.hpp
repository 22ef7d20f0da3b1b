// Device-side descriptions (plain structs passed by value to kernels) and the
// launchers of the kernels in kernels.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "fft.cuh"

namespace coral {

constexpr int kMaxGroups = 16;  // monomial groups (i kx)^a (i ky)^b per operator
constexpr int kMaxStages = 4;   // ARS_443 has 4 implicit stages
constexpr int kMaxSets = 8;     // coupled systems of one kind
constexpr int kMaxQuad = 32;    // quadratic variables
constexpr int kMaxFull = 16;    // full variables
constexpr int kMaxStatic = 4;   // full variables whose physical field is given, not transformed
constexpr int kMaxFullTerms = 8;
constexpr int kTabW = 5;        // Galerkin -> Chebyshev entries per Chebyshev row
constexpr int kTileRows = 128;  // rows per tile of the operator-stationary K_std kernel
constexpr int kRhsWin = 5 + kMaxQuad;  // ints per tile of SolveArgs::rhs_win

// Row-list operator: y[r] = sum_k coef[grp(r,k)] * val(r,k) * x[col(r,k)].
// Stored slot-major ([k][r]) so that a warp reading rows r..r+31 of one slot
// touches consecutive words; the group index sits in the top byte of the
// column word; empty slots hold column 0 and value 0.
struct DevEll {
  int rows, width, ngroups;
  int gkx[kMaxGroups], gky[kMaxGroups];
  const int* cg;
  const double* val;
  __device__ __forceinline__ int col(int r, int k) const { return cg[(size_t)k * rows + r] & 0xFFFFFF; }
  __device__ __forceinline__ int grp(int r, int k) const { return cg[(size_t)k * rows + r] >> 24; }
  __device__ __forceinline__ double v(int r, int k) const { return val[(size_t)k * rows + r]; }
};

// An operator row split by monomial group for the tile kernels: the slots of a
// row are grouped (group of slot k = slot_grp[k], the same in every row, groups
// in increasing slot order), so a row is evaluated as sum_g c_g (sum_k v_k x_k)
// with one complex multiply per group.  Groups whose entries coincide in every
// row are merged; the coefficient of a group is the sum of its monomials
// (i kx)^mkx (i ky)^mky.
constexpr int kGSlots = 16;  // slots of a grouped row (register-resident)
constexpr int kGMono = 4;    // monomials of one merged group
struct DevGEll {
  int valid;            // 0: the operator has no grouped form within these limits
  int rows, width, ngroups;
  int slot_grp[kGSlots];
  int nmono[kMaxGroups];
  int mkx[kMaxGroups][kGMono], mky[kMaxGroups][kGMono];
  const int* col;       // [width][rows] window-relative column, 0 in empty slots
  const double* val;    // [width][rows], 0 in empty slots
};

// one term of a full variable build: dsca * (i kx)^dx (i ky)^dy * S_var g
struct FullTermDev {
  int zero_kind;  // 1: mean variable (adds to the (0,0) mode only)
  int set;        // coupled system index
  int dx, dy;
  double dsca;
  const int* tab_t;      // [NZ][kTabW] state index or -1
  const double* tab_v;   // [NZ][kTabW] stencil value
};
struct FullVarDev {
  int nterms;
  FullTermDev term[kMaxFullTerms];
};

struct StateSet {  // pointers of the coupled kxky systems for the full-variable build
  const double2* k[kMaxSets];
  int kT[kMaxSets];
  const double* z[kMaxSets];
};

constexpr int kMaxTs = 16;      // timeseries objects (lines of coral.timeseries)

struct QuadDesc {
  int nq;
  int v1[kMaxQuad], v2[kMaxQuad];
  int ke_q[3];  // quadratic variables whose volume averages form KE (uu, vv, ww), -1 if absent
  // Timeseries objects of output_global_quantities (PL_IMEX_timestepping_output.f90:5-127),
  // evaluated on the first stage's physical fields when ts_partial is non-null:
  // ts_src[o] >= 0: full variable ts_src[o]; < 0: quadratic variable -1 - ts_src[o];
  // ts_z[o] < 0: volume average (Gauss-Chebyshev weights), else the horizontal average at
  // grid level ts_z[o] (0-based z index of phys(NZAA, NXAA, NYAA)).  Per-CTA partial sums
  // go to ts_partial[cta * kMaxTs + o].
  int ts_n;
  int ts_src[kMaxTs], ts_z[kMaxTs];
  double* ts_partial;
  // learned closure: tau[q][y][x][z] added to quadratic variable q after its
  // product (and after its KE contribution) in the unfused forward z pass; null: none
  const double* tau;
  // full variables whose physical values are given instead of transformed:
  // penalisation fields (st_prof 0: st_src[y][x][z], marching.f90:515) and the
  // Smagorinsky viscosity (st_prof 1: one value per z level, st_src[z],
  // marching.f90:516-541); the fused z pass puts them in place of the inverse
  // transform's output
  int st_n;
  int st_var[kMaxStatic], st_prof[kMaxStatic];
  const double* st_src[kMaxStatic];
};

struct Dims {
  int NXH, NYA, NXA, NZ, NZA;
};

// ---- launchers (kernels.cu) -------------------------------------------------
// inverse transform of nf scalars: spectral build (or a plain spec input) + y-FFT
// single = 1: every full variable is mean terms followed by exactly one kxky term
// (the single-term kernel); plain_spec: the transform of one given spectrum
void launch_inv_y(const Dims& d, int nf, const FullVarDev* fv, StateSet st, const double2* plain_spec,
                  const double* kx, const double* ky, double2* Y1, const FftPlan& py, cudaStream_t s,
                  int single = 0);
// pv: FFT plan of the compiled lengths, 1 = two passes (576 = 24 x 24, 288 = 18 x 16), 0 = three passes
// tiles = 1: one CTA per tile; 0: the persistent pipelined kernel (compiled
// lengths with a two-pass plan and pv = 1; others fall back to one CTA per tile)
void launch_inv_x(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, cudaStream_t s, int pv = 1,
                  int tiles = 1);
// z DCT-III; cfl: maxima of |u|, |v|, |w|/wz written (as uint64 bit patterns) to cfl_bits when non-null
void launch_inv_z(const Dims& d, int nf, const double* Y2, double* phys, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, unsigned long long* cfl_bits, cudaStream_t s);
void launch_fwd_z(const Dims& d, int nf, const QuadDesc& q, const double* phys, double* Q2, const FftPlan& pz,
                  const double2* dct_tw, const double* wz, double* ke_partial, cudaStream_t s);
// the z passes of a timestep stage fused: z DCT-III of the nf full variables from
// Y2, CFL maxima (cfl_bits, when non-null), products, KE partial averages (when
// ke_partial is non-null) and z DCT-II of the quadratic variables into Q2;
// wzinv[z] = 1 / wz[z]
void launch_z_fused(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* Q2, const FftPlan& pz,
                    const double2* dct_tw, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                    double* ke_partial, cudaStream_t s, int batch6 = 0, int y0 = 0, int ny = -1);
void launch_fwd_x(const Dims& d, int nq, const double* Q2, double2* Q1, const FftPlan& px, cudaStream_t s, int pv = 1,
                  int y0 = 0, int ny = -1);
// the inverse x pass (one CTA per tile) over the y rows y0 .. y0 + ny - 1 only; with
// launch_z_fused and launch_fwd_x over the same rows, the three passes of a band
// of y rows depend on no other rows (the y-chunked pipeline of a stage)
void launch_inv_x_rows(const Dims& d, int nf, const double2* Y1, double* Y2, const FftPlan& px, int pv, int y0, int ny,
                       cudaStream_t s);
// grid_variant = 1: one CTA per tile instead of the persistent pipelined kernel
void launch_fwd_y(const Dims& d, int nq, const double2* Q1, double2* qspec, double scale, const FftPlan& py,
                  cudaStream_t s, int grid_variant = 0);
void launch_remove_zmean(const Dims& d, double2* qspec_q, cudaStream_t s);
// z operations on one full variable's Chebyshev columns of Y2 (rows y0 .. y0 + ny - 1)
// before its inverse z transform: extract 1 bottom / 2 top surface value, decomp 1
// barotropic / 2 baroclinic (marching.f90:543-575)
void launch_zfilter(const Dims& d, double* Y2_var, int extract, int decomp, int y0, int ny, cudaStream_t s);
// the given physical fields of q.st_* written into phys[var][y][x][z]
void launch_static_phys(const Dims& d, const QuadDesc& q, double* phys, cudaStream_t s);
// Smagorinsky viscosity profile (marching.f90:516-541, 591-617): prof[z] = c sqrt(prof[z]
// + horizontal mean of the squares of phys[vars[k]]), part: NYA x NZA scratch; the
// maximum goes to cfl_max (when non-null) by an atomic maximum of non-negative doubles
void launch_smago(const Dims& d, const double* phys, const int* vars, int nvars, double c, double* part, double* prof,
                  unsigned long long* cfl_max, cudaStream_t s);
// the reference's default penalisation mask (PL_user_penalisation_mask.f90) on the grid,
// mask[y][x][z]; the penalisation field strength (1 + tanh(width mask)) / 2
void launch_penal_default(const Dims& d, double Lx, double Ly, const double* zgrid, double* mask, cudaStream_t s);
void launch_penal_field(size_t n, const double* mask, double strength, double width, double* out, cudaStream_t s);
// ---- split-precision z transforms on the tensor cores (zsplit.cu) ----
// int8 digits of the REDFT01 (fwd = false: NZAA x NZ) or REDFT10 (fwd = true:
// NZ x NZAA) matrix in the kernels' streaming order
std::vector<unsigned char> zsplit_matrix_digits(int K, int NOUT, bool fwd, int NZAA);
bool zsplit_supported(int NZ, int NZAA);
size_t zsplit_ctas(long long ncol, int nvar);
// inverse: Y2 [f][col][NZ] -> phys [f][col][NZAA], CFL maxima (cfl_bits non-null)
// and the full-variable timeseries objects (ts_partial non-null, rows 0..)
void launch_zsplit_inv(const Dims& d, int nf, const QuadDesc& q, const double* Y2, double* phys,
                       const unsigned char* mat, const double* wz, const double* wzinv, unsigned long long* cfl_bits,
                       double* ts_partial, unsigned* flags, cudaStream_t s);
// forward: products of phys -> Q2 [q][col][NZ], KE partials [cta][3] and the
// quadratic-variable timeseries objects (rows ts_row0..)
void launch_zsplit_fwd(const Dims& d, int nf, const QuadDesc& q, const double* phys, double* Q2,
                       const unsigned char* mat, const double* wz, double* ke_partial, double* ts_partial,
                       long long ts_row0, unsigned* flags, cudaStream_t s);

// learned closure (closure.cu): inference on a whole grid, 4 full variables
// [f][y][x][z] -> tau [9][y][x][z]
struct ClosureImpl;
void closure_infer(ClosureImpl* c, const double* fields, int NYA, int NXA, int NZA, double* tau, cudaStream_t s);

// the kx = 0 line (the first NYA x T entries) of a coupled state onto its
// Hermitian part (timeseries.cu)
void launch_hermitian_kx0(double2* field, int NYA, int T, cudaStream_t s);

// CTAs of launch_z_fused (rows of its KE and timeseries partial sums)
size_t z_fused_ctas(const Dims& d);
// total of the n KE partial sums (one CTA, fixed order) into *out
void launch_ke_sum(const double* part, size_t n, double* out, cudaStream_t s);
// timeseries: out[o] = scale * sum over the ncta rows of part[cta * kMaxTs + o]
// (fixed order, deterministic), o < nobj (timeseries.cu)
void launch_ts_reduce(const double* part, size_t ncta, int nobj, double scale, double* out, cudaStream_t s);

struct NLArgs {
  Dims d;
  int T;
  DevEll NL;
  const double2* qspec;
  const double* kx;
  const double* ky;
  const int* act_index;  // [kx*NYA+ky] -> factor slot, -1 for dealiased modes and (0,0)
  double2* Khat;
  int nq;                // quadratic variables in qspec
};
void launch_nl(const NLArgs& a, cudaStream_t s);

struct SolveArgs {
  Dims d;
  int T, kl, ku, ldab;
  DevEll M, L;
  const double2* field;
  double2* out;          // aux (or field itself in the last stage)
  double2* work;         // scratch vectors of the register-window solve (aux)
  double2* Kstd_out;     // null in the last stage
  int nprev;             // stage index i (0-based): Kstd[0..i-1], Khat[0..i]
  const double2* Kstd[kMaxStages];
  const double2* Khat[kMaxStages];
  double ca[kMaxStages];  // dt * a(i, j)
  double ch[kMaxStages];  // dt * ahat(i+1, j)
  const double2* ab;
  const unsigned char* dpiv;
  const int* act_index;
  int last_stage;
  const double* kx;
  const double* ky;
  unsigned int* flags;   // bit 0: non-finite value produced
  // real-scaled factors (see SystemOps::real_scalable): rows flagged in rowflip
  // are multiplied by -i before the solve, columns flagged in colflip by +i after
  const double* abr;
  const unsigned char* rowflip;
  const unsigned char* colflip;
  int ring_cols;         // doubles per column slot of the solve's shared-memory ring
  int nact;              // active systems (factor slots)
  const int* act_list;   // [nact] kx*NYA+ky of each factor slot
  // class split (SystemOps::ncls == 2): factors of both classes interleaved per
  // column (column stride ncls*ldab), kl/ku/ldab those of one class; the
  // right-hand sides and solutions in work are stored class by class
  // (work stride wst >= ncls*Tc) and mapped back through col_pos.
  int ncls, Tc, wst;
  const int* row_pos;    // [T] class position of an equation row (null: unsplit)
  const int* col_pos;    // [T] class position of a variable column (null: unsplit)
  const unsigned char* colflip_cls;  // [ncls*Tc] colflip in class order
  DevEll Lp;             // L with its columns in class positions (= L when unsplit)
  // thread-per-block solve (class split): block b = 2 act + class, lane b % 32 of
  // group b / 32; factors abr[((g Tc + j) ldab + r) 32 + lane], pivots
  // dpiv[(g Tc + j) 32 + lane], right-hand sides / solutions of the active
  // systems work2[(g Tc + j) 32 + lane]; inactive systems stay in work
  double2* work2;        // null: warp-per-system layouts
  int nblk;              // ncls * nact
  const int* cls_col;    // [ncls*Tc] variable column of a class position, -1 = padding: the
                         // thread-per-block solve writes its solution straight into out
  // operator-stationary K_std (null tile_win: k_kstd_out): rows in tiles of
  // kTileRows; tile_win[2 tile + .] = (start, width) of the solution columns the
  // tile's rows of L touch; Lw = L with its columns relative to that window
  const int* tile_win;
  int tile_lwin_max;     // widest window
  DevGEll Lw;            // !valid: k_kstd_out
  // operator-stationary right-hand side (null rhs_win: k_rhs_nl): per tile of
  // kTileRows rows, rhs_win[kRhsWin tile + .] = (start, width) of the state
  // columns its rows of M touch, (start, width) of the Chebyshev range its rows
  // of the NL operator touch, the number of quadratic variables they touch and
  // those variables; Mw = M with columns relative to the state window, NLw = the
  // NL operator with columns slot * width + n - start (slot: position of the
  // variable in the tile's list)
  const int* rhs_win;
  int rhs_win_max;       // widest window (state + all slots), complex entries
  DevEll Mw, NLw;
  DevGEll NLg;           // NLw in grouped form (valid = 0: none)
  int generic_tiles;     // 1: the tile kernels' run-time forms only (no compiled group layouts)
  int subst_rt;          // 1: the run-time-band substitution kernel even for the compiled band
  // band entries that are zero in every block are not loaded (FactorArgs::lmask,
  // umask; null: load all)
  const unsigned* lmask;
  const unsigned* umask;
};
void launch_solve(const SolveArgs& a, cudaStream_t s);
// real-scaled factors (unsplit: kl <= 31, kl+ku <= 63; class split: kl <= 15,
// kl+ku <= 31 per class): right-hand side with the NL assembly fused in,
// substitutions, then K_std and outputs (three kernels)
void launch_solve_real(const SolveArgs& a, const NLArgs& n, cudaStream_t s);
// its three kernels one by one
void launch_rhs_nl(const SolveArgs& a, const NLArgs& n, cudaStream_t s);
void launch_subst(const SolveArgs& a, cudaStream_t s);
void launch_kstd_out(const SolveArgs& a, cudaStream_t s);
// the substitutions of several systems in one persistent launch (ensembles):
// d_args[m] the SolveArgs of member m, d_prefix[m] its first block in the
// concatenated range (d_prefix[nmem] = total); every member must pass
// subst_multi_supported (thread-per-block layout, band (9, 23), ldab 34)
bool subst_multi_supported(const SolveArgs& a);
void launch_subst_multi(const SolveArgs* d_args, const long long* d_prefix, int nmem, long long total,
                        cudaStream_t s);

struct FactorArgs {
  Dims d;
  int T, kl, ku, ldab, nact;
  DevEll M, L;
  double zsca;           // -dt * a(0,0)
  const int* act_list;   // [nact] kx*NYA+ky
  double2* ab;
  unsigned char* dpiv;
  const double* kx;
  const double* ky;
  int* info;             // first zero pivot (1-based column) per system, 0 if none
  double* abr;           // real-scaled factors (when rowflip/colflip are set)
  const unsigned char* rowflip;
  const unsigned char* colflip;
  // class split of the real-scaled factors (see SolveArgs); ncls = 1: unsplit
  int ncls, Tc;
  const int* cls_row;    // [ncls*Tc] equation row of a class position, -1 = identity padding
  const int* col_pos;    // [T] class position of a variable column
  int tpb;               // 1: interleaved thread-per-block factor layout (see SolveArgs::work2)
  int window;            // thread-per-block layout: 1 shared-memory band window, 0 in place in global memory
  // thread-per-block layout: per class column j, the band rows nonzero in any
  // block (cmask, bit r = band row r), and derived from it the L rows
  // (lmask[j], bit i = row kl+ku+1+i of column j) and the U entries of row j
  // (umask[j], bit i = entry (j, j+1+i)) that are nonzero in any block
  unsigned long long* cmask;
  unsigned* lmask;
  unsigned* umask;
};
void launch_factor(const FactorArgs& a, cudaStream_t s);
void launch_factor_real(const FactorArgs& a, cudaStream_t s);

// mean (kx = ky = 0) systems, real arithmetic
struct ZeroSysDev {
  int T, kl, ku, ldab;
  DevEll M, L, NL;
  double* field;
  double* aux;
  double* Kstd[kMaxStages];
  double* Khat[kMaxStages];
  double* ab;
  unsigned char* dpiv;
  const double* src;  // constant source terms of K_hat (marching.f90:398-415), null: none
};
struct ZeroArgs {
  int nsys;
  ZeroSysDev sys[kMaxSets];
  const double2* qspec;  // [q][kx][ky][n]; the (0,0) column is read
  Dims d;
  int stage;
  double ca[kMaxStages], ch[kMaxStages];
  int last_stage;
  double zsca;
  int* info;
};
void launch_zero_step(const ZeroArgs& a, cudaStream_t s);
void launch_zero_factor(const ZeroArgs& a, cudaStream_t s);

// QuickSave helpers
// the z derivatives (order) of dsca x one kxky variable's Chebyshev coefficients
// (its stencil tab_t / tab_v applied to state, T entries per (kx, ky)) into
// out[kx][ky][n]: the full-variable build's dz terms
void launch_full_dz(const Dims& d, const double2* state, int T, const int* tab_t, const double* tab_v, double dsca,
                    int order, double gap, double2* out, cudaStream_t s);
// the same for one mean variable's profile (state: its system's vector)
void launch_zero_dz(int NZ, const double* state, const int* tab_t, const double* tab_v, double dsca, int order,
                    double gap, double* out, cudaStream_t s);
// user outputs: a slice (kind 1 z, 2 y, 3 x at index k) or the weighted z sum
// (kind 4) of phys[y][x][z] in the reference's file order; the horizontal-average
// profile; the product of two fields (b null: a copy)
void launch_usr_slice(const Dims& d, const double* phys, int kind, int k, const double* wz, double* out,
                      cudaStream_t s);
void launch_usr_profile(const Dims& d, const double* phys, double* out, cudaStream_t s);
void launch_phys_product(size_t n, const double* a, const double* b, double* out, cudaStream_t s);
void launch_transpose_xy(const Dims& d, const double* in, double* out, int to_file_order, cudaStream_t s);
// project Chebyshev coefficients spec[kx][ky][n] onto the Galerkin basis of one
// variable (lower-triangular square stencil) and add them into the state
void launch_galerkin_insert(const Dims& d, const double2* spec, int T, const int* var_pos, int nc,
                            const double* sq /*nc x kTabW band, row-major*/, const int* sq_off,
                            double2* field, cudaStream_t s);
void launch_cheb_extract(const Dims& d, const double2* field, int T, const int* tab_t, const double* tab_v,
                         double2* spec, cudaStream_t s);
void launch_check_finite(const double2* x, size_t n, unsigned int* flags, cudaStream_t s);

}  // namespace coral
