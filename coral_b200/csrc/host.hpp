// Host-side description of a plane-layer problem: the parsed equation recipe,
// the geometry and the operator tables the CUDA kernels consume.
//
// Everything here runs once at set-up on the CPU (the reference also assembles
// its operators on the host, src/plane_layer/PL_IMEX_timestepping.f90:488-1635);
// the timestep itself runs only on the GPU.
#pragma once

#include <complex>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace coral {

using cplx = std::complex<double>;

struct CoralError : std::runtime_error {
  int code;
  CoralError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// text returned by coral_last_error(NULL) (calls that have no handle)
void set_global_error(const std::string& msg);

// ---------------------------------------------------------------------------
// coral.parameters.in  (src/plane_layer/PL_geometry.f90:269-305)
// ---------------------------------------------------------------------------
struct Parameters {
  int NX = 0, NY = 0, NZ = 0;
  double Lx = 0, Ly = 0, gap = 1, center = 0.5;
  double dt_max = 0, tolerance = 0, CFL_C = 0;
  std::string scheme;
  bool qsave_restart = false;
  double time_limit = 0;
};
Parameters parse_parameters(const std::string& text);

// ---------------------------------------------------------------------------
// coral.equations  (src/plane_layer/PL_equations.f90:435-593, 1758-2043;
//                   src/plane_layer/PL_string_to_data.f90:53-118, 387-465)
// ---------------------------------------------------------------------------
struct Piece {      // linear_operator_recipe_T entry
  double dsca;
  int kx, ky, Iz, mz, jVar, iEqn;
};
struct NLTerm {     // atom_NL_term_T
  double dsca;
  int dx, dy, Iz, mz, quad, eqn;
};
struct FullTerm {   // a_linear_contribution_T
  bool zero_kind;   // true: a mean ('zero') variable, false: a kxky variable
  int var;          // index in the kxky / mean variable list
  double dsca;
  int dx, dy, dz, mz;
};
struct FullVar {
  std::string name;
  std::vector<FullTerm> terms;
  // z operations on the Chebyshev coefficients before the inverse transform
  // (marching.f90:543-575): extract 0 nowhere, 1 BotSurf, 2 TopSurf (the surface
  // value, PL_equations.f90:497-500); decomp 0 none, 1 barotropic, 2 baroclinic
  // (vertical_decomposition, :502-503, 1052-1067)
  int extract = 0, decomp = 0;
  // enable_penalisation (:508-517): the physical field is strength (1 + tanh(width
  // mask)) / 2 of the user's mask, never transformed
  bool penal = false;
  double penal_strength = 0.0, penal_width = 0.0;
  // nuSmago (--withHorizontalSmagorinsky, :519-526): the horizontal Smagorinsky
  // viscosity, formed in physical space (marching.f90:516-541)
  bool smago = false;
};
struct SourceTerm {  // source_term_T (PL_equations.f90:37-45)
  double dsca;
  int Iz, index;     // Iz^Iz sourceNN (index NN >= 1)
  int set, eqn;      // mean system and equation
};
struct QuadVar {
  std::string name;
  int v1, v2;       // full-variable indices, -1 = 'ONE'
  bool remove_mean; // zFiltered_quadratic_variable
};
struct CoupledSet {
  std::vector<std::string> vars;
  std::vector<int> bcs;
  std::vector<int> orders;
  std::vector<Piece> mass, stif;
  std::vector<NLTerm> nl;
};
struct Recipe {
  std::vector<std::pair<std::string, double>> params;
  std::vector<std::string> kxky_vars, zero_vars;
  std::vector<FullVar> full;
  std::vector<QuadVar> quad;
  std::vector<CoupledSet> kxky, zero;
  std::map<std::string, std::pair<int, int>> kxky_loc, zero_loc;  // (set, position)
  std::vector<std::pair<std::string, double>> source_params;      // sourceParam lines
  std::vector<SourceTerm> sources;                                // add_rhs_source lines
  bool smagorinsky = false;
};
// smagorinsky: the reference's --withHorizontalSmagorinsky switch (the full
// variable nuSmago goes in before the first quadratic variable)
Recipe parse_equations(const std::string& text, bool smagorinsky = false);

// ---------------------------------------------------------------------------
// geometry  (src/plane_layer/PL_geometry.f90:80-236)
// ---------------------------------------------------------------------------
struct Geometry {
  int NX, NY, NZ, NXAA, NYAA, NZAA, NXH;
  double Lx, Ly, gap, center, kx_box, ky_box;
  std::vector<double> kx, ky;
  std::vector<char> deal_x, deal_y;
  explicit Geometry(const Parameters& p);
  bool active(int ix, int iy) const {
    return !(deal_x[ix] || deal_y[iy]) && !(ix == 0 && iy == 0);
  }
  std::vector<double> zweights() const;  // PL_cheby_misc.f90:29-55
};

// ---------------------------------------------------------------------------
// ARS IMEX tableaux  (src/timesteppers/IMEX_schemes.f90:21-402)
// ---------------------------------------------------------------------------
struct Tableau {
  int stages;
  std::vector<double> A;     // stages x stages, row-major
  std::vector<double> Ahat;  // (stages+1) x (stages+1), row-major
  double a(int i, int j) const { return A[i * stages + j]; }
  double ahat(int i, int j) const { return Ahat[i * (stages + 1) + j]; }
};
Tableau ars_tableau(const std::string& name);

// ---------------------------------------------------------------------------
// Chebyshev tools and Galerkin stencils
// ---------------------------------------------------------------------------
using Dense = std::vector<std::vector<double>>;
Dense cheb_IM(int N, double center, double gap, int a, int b, int padding = 15);
Dense stencil(int N, int bc);  // N x ncol

// A sparse row-list ("ELL") operator in the interleaved polynomial ordering.
// y[row] += coef[grp] * val * x[col] for every entry of the row.
struct EllOp {
  int rows = 0, width = 0;           // width = max entries per row
  std::vector<int> col;              // rows*width, -1 = empty slot
  std::vector<double> val;
  std::vector<int> grp;              // monomial group of the entry
  // monomial groups: (kx exponent, ky exponent)
  std::vector<std::pair<int, int>> groups;
};

// one coupled kxky (or mean) system, assembled
struct SystemOps {
  int nV = 0, T = 0;
  std::vector<int> var_size, eq_size, bcs, orders;
  std::vector<std::vector<int>> var_pos, eq_pos;  // interleaving (PL_IMEX_timestepping.f90:1344-1414)
  EllOp M, L;                                     // mass and stiffness operators
  int kl = 0, ku = 0;                             // band of M - dt*a*L
  // NL assembly: for each row t of K_hat, entries (quad var, Chebyshev n, val, group)
  EllOp NLop;                                     // col = quad*NZ + n
  // Galerkin -> Chebyshev: for var v, row n: entries (galerkin coef c, value)
  std::vector<std::vector<std::vector<std::pair<int, double>>>> stencil_rows;
  // Real scaling: when every entry of E = M - dt a L is real or imaginary in a
  // pattern that multiplying some variables by i and some equations by -i turns
  // real, row_flip[t] / col_flip[t] mark the rows (equations) and columns
  // (variables) of that diagonal scaling and real_scalable is true.
  bool real_scalable = false;
  std::vector<unsigned char> row_flip, col_flip;
  // Independent blocks: when the pattern of M and L (equation rows x variable
  // columns) falls apart into blocks that touch only themselves (Chebyshev
  // parity does this for the plane-layer recipes), the components are gathered
  // into ncls = 2 classes of equal size Tc (the smaller padded with identity
  // rows).  Each class is its own band system of band (kl_cls, ku_cls) in the
  // original relative order, and LU with partial pivoting of E factors class by
  // class: the entries of the other class are exact zeros in every pivot
  // column, so pivots and multipliers are those of the whole matrix.
  int ncls = 1, Tc = 0, kl_cls = 0, ku_cls = 0;
  std::vector<int> row_cls_pos;  // [T] class * Tc + index within the class (equation rows)
  std::vector<int> col_cls_pos;  // [T] the same for variable columns
  std::vector<int> cls_row;      // [ncls * Tc] equation row of a class position, -1 = identity padding
  // square stencil (var_size x var_size, lower-banded) for projections of
  // Chebyshev coefficients onto the Galerkin basis (QuickSave import)
  std::vector<Dense> sq_stencil;
};

SystemOps assemble_system(const Geometry& g, const Recipe& r, const CoupledSet& s);

}  // namespace coral
