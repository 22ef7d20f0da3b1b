// Set-up on the host: parameter/equation parsing, geometry, IMEX tableaux,
// Chebyshev matrices, Galerkin stencils and the assembly of the coupled
// systems' operators in the interleaved polynomial ordering.
#include <algorithm>
#include <cctype>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "host.hpp"
#include "../../include/coral_b200.h"

namespace coral {

static double fortran_float(std::string s) {
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw CoralError(CORAL_EPARSE, "cannot read a number from '" + s + "'");
  return v;
}

static std::string first_token(const std::string& line) {
  std::istringstream is(line);
  std::string t;
  is >> t;
  return t;
}

Parameters parse_parameters(const std::string& text) {
  // Fixed line order: the first token of lines 2-4, 6-9, 11-14, 16, 18 holds the values.
  std::vector<std::string> lines;
  std::istringstream is(text);
  std::string l;
  while (std::getline(is, l)) lines.push_back(l);
  if (lines.size() < 18) throw CoralError(CORAL_EPARSE, "coral.parameters.in: expected 18 lines");
  Parameters p;
  p.NX = std::atoi(first_token(lines[1]).c_str());
  p.NY = std::atoi(first_token(lines[2]).c_str());
  p.NZ = std::atoi(first_token(lines[3]).c_str());
  p.Lx = fortran_float(first_token(lines[5]));
  p.Ly = fortran_float(first_token(lines[6]));
  p.gap = fortran_float(first_token(lines[7]));
  p.center = fortran_float(first_token(lines[8]));
  p.dt_max = fortran_float(first_token(lines[10]));
  p.tolerance = fortran_float(first_token(lines[11]));
  p.CFL_C = fortran_float(first_token(lines[12]));
  std::string sch = first_token(lines[13]);
  sch.erase(std::remove(sch.begin(), sch.end(), '\''), sch.end());
  sch.erase(std::remove(sch.begin(), sch.end(), '"'), sch.end());
  p.scheme = sch;
  std::string b = first_token(lines[15]);
  for (auto& ch : b) ch = (char)std::tolower(ch);
  p.qsave_restart = (b.find("true") != std::string::npos) || b == ".t." || b == "t";
  p.time_limit = fortran_float(first_token(lines[17]));
  if (p.NX <= 0 || p.NY <= 0 || p.NZ <= 0) throw CoralError(CORAL_EPARSE, "non-positive resolution");
  return p;
}

// --- equation grammar --------------------------------------------------------

static std::string clean(const std::string& s) {
  std::string o;
  for (char c : s)
    if (c != ' ' && c != '\0' && c != '\t' && c != '\r') o.push_back(c);
  return o;
}

static bool starts(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

static std::string payload(const std::string& line) {
  size_t i = line.find("::"), j = line.find("<<");
  if (i == std::string::npos || j == std::string::npos || j < i + 2)
    throw CoralError(CORAL_EPARSE, "malformed line: " + line.substr(0, 78));
  return line.substr(i + 2, j - i - 2);
}

struct Atom {
  double dsca;
  int dx = 0, dy = 0, Iz = 0, mz = 0;
  std::vector<std::string> unsorted;
};

// break_linear_operators_in_pieces: every '+' piece, then every '-' piece.
static std::vector<Atom> atoms(const std::string& line, const char* dz) {
  std::vector<Atom> out;
  const char signs[2] = {'+', '-'};
  for (int k = 0; k < 2; ++k) {
    std::string aux = line;
    size_t p;
    while ((p = aux.find(signs[k])) != std::string::npos) {
      aux = aux.substr(p + 1);
      size_t end = aux.find_first_of("+-<");
      std::string piece = aux.substr(0, end == std::string::npos ? aux.size() : end);
      Atom a;
      a.dsca = (k == 0) ? 1.0 : -1.0;
      std::string chunk;
      std::istringstream cs(piece);
      while (std::getline(cs, chunk, '.')) {
        std::string c = clean(chunk);
        if (c == "dx") a.dx++;
        else if (c == "dy") a.dy++;
        else if (c == dz) a.Iz++;
        else if (c == "mz") a.mz++;
        else a.unsorted.push_back(c);
      }
      if (a.unsorted.size() > 4)
        throw CoralError(CORAL_EPARSE, "too many unrecognized characters in: " + piece);
      out.push_back(a);
    }
  }
  return out;
}

Recipe parse_equations(const std::string& text, bool smagorinsky) {
  Recipe r;
  r.smagorinsky = smagorinsky;
  bool zero_set = false, smago_pending = smagorinsky;
  auto param_value = [&](const std::string& n, double* v) {
    for (auto& p : r.params)
      if (p.first == n) { *v = p.second; return true; }
    return false;
  };
  std::istringstream is(text);
  std::string line;
  bool eof = false;
  while (!eof && std::getline(is, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (starts(line, ">>=")) continue;
    if (!starts(line, ">>")) continue;
    std::string key = line.substr(2);
    if (starts(key, "EOF")) { eof = true; break; }
    if (starts(key, "Param")) {
      std::string body = payload(line);
      size_t e = body.find(":=");
      if (e == std::string::npos) throw CoralError(CORAL_EPARSE, "Param without ':=': " + line);
      r.params.emplace_back(clean(body.substr(0, e)), fortran_float(clean(body.substr(e + 2))));
    } else if (starts(key, "sourceParam")) {  // add_source_parameter (PL_equations.f90:985-996)
      std::string body = payload(line);
      size_t e = body.find(":=");
      if (e == std::string::npos) throw CoralError(CORAL_EPARSE, "sourceParam without ':=': " + line);
      r.source_params.emplace_back(clean(body.substr(0, e)), fortran_float(clean(body.substr(e + 2))));
    } else if (starts(key, "linear_variable_kxky")) {
      r.kxky_vars.push_back(clean(payload(line)));
    } else if (starts(key, "linear_variable_mean")) {
      r.zero_vars.push_back(clean(payload(line)));
    } else if (starts(key, "linear_variable_full_build")) {
      if (r.full.empty()) throw CoralError(CORAL_EPARSE, "full_build before a full variable");
      for (auto& a : atoms(line, "dz")) {
        FullTerm t{false, -1, a.dsca, a.dx, a.dy, a.Iz, a.mz};
        bool found = false;
        for (auto& s : a.unsorted) {
          auto z = std::find(r.zero_vars.begin(), r.zero_vars.end(), s);
          auto k = std::find(r.kxky_vars.begin(), r.kxky_vars.end(), s);
          double v;
          if (z != r.zero_vars.end()) { t.zero_kind = true; t.var = int(z - r.zero_vars.begin()); found = true; }
          else if (k != r.kxky_vars.end()) { t.zero_kind = false; t.var = int(k - r.kxky_vars.begin()); found = true; }
          else if (param_value(s, &v)) t.dsca = t.dsca * v;
          else throw CoralError(CORAL_EPARSE, "unknown string in equations: " + s);
        }
        if (!found) throw CoralError(CORAL_EPARSE, "invalid full variable def.");
        r.full.back().terms.push_back(t);
      }
    } else if (starts(key, "linear_variable_full")) {
      r.full.push_back(FullVar{clean(payload(line)), {}});
    } else if (starts(key, "linear_variable_bottom_boundary_value") ||
               starts(key, "linear_variable_top_boundary_value")) {
      r.full.push_back(FullVar{clean(payload(line)), {}});
      r.full.back().extract = starts(key, "linear_variable_bottom") ? 1 : 2;
    } else if (starts(key, "vertical_decomposition")) {
      if (r.full.empty()) throw CoralError(CORAL_EPARSE, "vertical_decomposition before a full variable");
      const std::string k = clean(payload(line));
      if (k == "barotropic") r.full.back().decomp = 1;
      else if (k == "baroclinic") r.full.back().decomp = 2;
      else throw CoralError(CORAL_EPARSE, "vertical_decomposition should be baroclinic or barotropic");
    } else if (starts(key, "enable_penalisation")) {
      r.full.push_back(FullVar{clean(payload(line)), {}});
      r.full.back().penal = true;
    } else if (starts(key, "penalisation_strength") || starts(key, "penalisation_width")) {
      if (r.full.empty() || !r.full.back().penal)
        throw CoralError(CORAL_EPARSE, "penalisation parameter without enable_penalisation");
      const double v = fortran_float(clean(payload(line)));
      if (starts(key, "penalisation_strength")) r.full.back().penal_strength = v;
      else r.full.back().penal_width = v;
    } else if (starts(key, "quadratic_variable") || starts(key, "zFiltered_quadratic_variable")) {
      if (smago_pending) {
        r.full.push_back(FullVar{"nuSmago", {}});
        r.full.back().smago = true;
        smago_pending = false;
      }
      std::string body = payload(line);
      size_t e = body.find(":=");
      std::string q = clean(body.substr(0, e)), rhs = clean(body.substr(e + 2));
      size_t d = rhs.find('.');
      std::string a = rhs.substr(0, d), b = rhs.substr(d + 1);
      auto idx = [&](const std::string& n) {
        if (n == "ONE") return -1;
        for (size_t i = 0; i < r.full.size(); ++i)
          if (r.full[i].name == n) return int(i);
        throw CoralError(CORAL_EPARSE, "bad NL var definition (wrong reference to linear var.)");
      };
      QuadVar qv{q, idx(a), idx(b), starts(key, "zFiltered")};
      if (qv.v1 == -1 && qv.v2 == -1) throw CoralError(CORAL_EPARSE, "quad var defined as ONE.ONE");
      r.quad.push_back(qv);
    } else if (starts(key, "add_set_of_coupled_kxky_equations")) {
      r.kxky.emplace_back();
      zero_set = false;
    } else if (starts(key, "add_set_of_coupled_zero_equations")) {
      r.zero.emplace_back();
      zero_set = true;
    } else if (starts(key, "linearly_coupled_var") || starts(key, "add_BC_for_this_var") ||
               starts(key, "new_equation") || starts(key, "add_d/dt_term") ||
               starts(key, "add_rhs_linear") || starts(key, "add_rhs_NL")) {
      auto& sets = zero_set ? r.zero : r.kxky;
      if (sets.empty()) throw CoralError(CORAL_EPARSE, "equation line before a coupled set: " + line);
      CoupledSet& s = sets.back();
      if (starts(key, "linearly_coupled_var")) {
        std::string n = clean(payload(line));
        s.vars.push_back(n);
        s.bcs.push_back(0);
        (zero_set ? r.zero_loc : r.kxky_loc)[n] = {int(sets.size()) - 1, int(s.vars.size()) - 1};
      } else if (starts(key, "add_BC_for_this_var")) {
        s.bcs.back() = std::atoi(clean(payload(line)).c_str());
      } else if (starts(key, "new_equation")) {
        s.orders.push_back(std::atoi(clean(payload(line)).c_str()));
      } else if (starts(key, "add_rhs_NL")) {
        for (auto& a : atoms(line, "Iz")) {
          NLTerm t{a.dsca, a.dx, a.dy, a.Iz, a.mz, -1, int(s.orders.size()) - 1};
          for (auto& st : a.unsorted) {
            double v;
            int q = -1;
            for (size_t i = 0; i < r.quad.size(); ++i)
              if (r.quad[i].name == st) { q = int(i); break; }
            if (q >= 0) t.quad = q;
            else if (param_value(st, &v)) t.dsca = v * t.dsca;
            else throw CoralError(CORAL_EPARSE, "unknown string in equations: " + st);
          }
          if (t.quad < 0) throw CoralError(CORAL_EPARSE, "invalid quad_var_index");
          if (zero_set && (t.dx || t.dy)) throw CoralError(CORAL_EPARSE, "x/y-derivative in a mean-field recipe");
          s.nl.push_back(t);
        }
      } else {
        bool mass = starts(key, "add_d/dt_term");
        for (auto& a : atoms(line, "Iz")) {
          Piece p{a.dsca, a.dx, a.dy, a.Iz, a.mz, -1, int(s.orders.size()) - 1};
          for (auto& st : a.unsorted) {
            double v;
            auto it = std::find(s.vars.begin(), s.vars.end(), st);
            if (it != s.vars.end()) p.jVar = int(it - s.vars.begin());
            else if (param_value(st, &v)) p.dsca = v * p.dsca;
            else throw CoralError(CORAL_EPARSE, "unknown string in equations: " + st);
          }
          if (p.jVar < 0) throw CoralError(CORAL_EPARSE, "invalid stif/mass matrix definition");
          if (p.iEqn < 0) throw CoralError(CORAL_EPARSE, "operator term before new_equation");
          (mass ? s.mass : s.stif).push_back(p);
        }
      }
    } else if (starts(key, "add_rhs_source")) {
      // build_zero_sources_in_full_recipe (PL_equations.f90:1156-1230): mean systems only
      if (!zero_set || r.zero.empty()) throw CoralError(CORAL_EPARSE, "add_rhs_source outside a set of mean equations");
      CoupledSet& s = r.zero.back();
      for (auto& a : atoms(line, "Iz")) {
        if (a.dx || a.dy) throw CoralError(CORAL_EPARSE, "x/y-derivative in a source term");
        SourceTerm t{a.dsca, a.Iz, 0, int(r.zero.size()) - 1, int(s.orders.size()) - 1};
        for (auto& st : a.unsorted) {
          // a string of 8 characters 'sourceNN' names the source and ends the atom's
          // strings; any other is a parameter
          if (st.size() == 8 && starts(st, "source")) {
            if (!std::isdigit((unsigned char)st[6]) || !std::isdigit((unsigned char)st[7]))
              throw CoralError(CORAL_EPARSE, "Source terms must be of the form sourceNN: " + st);
            t.index = std::atoi(st.substr(6).c_str());
            break;
          }
          double v;
          if (param_value(st, &v)) t.dsca = v * t.dsca;
          else throw CoralError(CORAL_EPARSE, "unknown string in equations: " + st);
        }
        if (t.index == 0) throw CoralError(CORAL_EPARSE, "invalid source_index");
        if (t.eqn < 0) throw CoralError(CORAL_EPARSE, "source term before new_equation");
        r.sources.push_back(t);
      }
    } else {
      throw CoralError(CORAL_EPARSE, "the line could not be read: " + line.substr(0, 78));
    }
  }
  if (r.kxky.empty()) throw CoralError(CORAL_EPARSE, "no coupled kxky system");
  return r;
}

// --- geometry -----------------------------------------------------------------

Geometry::Geometry(const Parameters& p) {
  NX = p.NX; NY = p.NY; NZ = p.NZ;
  NXAA = 3 * NX / 2; NYAA = 3 * NY / 2; NZAA = 3 * NZ / 2; NXH = NX / 2;
  Lx = p.Lx; Ly = p.Ly; gap = p.gap; center = p.center;
  const double pi = 4.0 * std::atan(1.0);
  ky_box = 2.0 * pi / Ly;
  kx_box = 2.0 * pi / Lx;
  ky.resize(NYAA); deal_y.resize(NYAA);
  for (int iy = 0; iy < NYAA; ++iy) {
    int k_index = iy + 1;
    if (k_index >= NYAA / 2 + 1) ky[iy] = -double((NYAA + 1 - k_index) * ky_box);
    else ky[iy] = double((k_index - 1) * ky_box);
    deal_y[iy] = std::fabs(ky[iy]) >= ky_box * NY / 2.0;
  }
  kx.resize(NXH); deal_x.resize(NXH);
  for (int ix = 0; ix < NXH; ++ix) {
    kx[ix] = double(ix * kx_box);
    deal_x[ix] = std::fabs(kx[ix]) >= kx_box * NX / 2.0;
  }
}

std::vector<double> Geometry::zweights() const {
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> g(NZAA), mid(NZAA + 1), w(NZAA);
  for (int i = 1; i <= NZAA; ++i) g[i - 1] = std::cos(pi * double(2 * i - 1) / double(2 * NZAA));
  mid[0] = 1.0; mid[NZAA] = -1.0;
  for (int i = 1; i < NZAA; ++i) mid[i] = 0.5 * (g[i] + g[i - 1]);
  for (int i = 0; i < NZAA; ++i) w[i] = (mid[i] - mid[i + 1]) / 2.0 * gap;
  return w;
}

// --- tableaux -----------------------------------------------------------------

Tableau ars_tableau(const std::string& name) {
  Tableau t;
  auto set = [&](int s) { t.stages = s; t.A.assign(s * s, 0.0); t.Ahat.assign((s + 1) * (s + 1), 0.0); };
  auto A = [&](int i, int j) -> double& { return t.A[i * t.stages + j]; };
  auto H = [&](int i, int j) -> double& { return t.Ahat[i * (t.stages + 1) + j]; };
  if (name == "ARS_111") { set(1); A(0, 0) = 1.0; H(1, 0) = 1.0; }
  else if (name == "ARS_122") { set(1); A(0, 0) = 0.5; H(1, 0) = 0.5; }
  else if (name == "ARS_233") {
    set(2); double g = (3.0 + std::sqrt(3.0)) / 6.0;
    A(0, 0) = g; A(1, 1) = g; A(1, 0) = 1.0 - 2.0 * g;
    H(1, 0) = g; H(2, 0) = g - 1.0; H(2, 1) = 2.0 * (1.0 - g);
  } else if (name == "ARS_232") {
    set(2); double d = -2.0 * std::sqrt(2.0) / 3.0, g = 1.0 - 1.0 / std::sqrt(2.0);
    A(0, 0) = g; A(1, 1) = g; A(1, 0) = 1.0 - g;
    H(1, 0) = g; H(2, 0) = d; H(2, 1) = 1.0 - d;
  } else if (name == "ARS_222") {
    set(2); double g = 1.0 - 1.0 / std::sqrt(2.0), d = 1.0 - 1.0 / (2.0 * g);
    A(0, 0) = g; A(1, 1) = g; A(1, 0) = 1.0 - g;
    H(1, 0) = g; H(2, 0) = d; H(2, 1) = 1.0 - d;
  } else if (name == "ARS_343") {
    // default-real literals of the reference are single precision (IMEX_schemes.f90:277-282)
    set(3);
    double g = (double)(float)0.43586652150845895, umg = (double)(float)0.28206673924577053;
    double b1 = (double)(float)1.2084966491760099, b2 = (double)(float)-0.64436317068446880;
    double a42 = 0.5529291479;
    A(0, 0) = g; A(1, 1) = g; A(2, 2) = g; A(1, 0) = umg; A(2, 0) = b1; A(2, 1) = b2;
    H(1, 0) = g;
    H(2, 0) = (15.0 / 4.0 - 15.0 * g + 21.0 / 4.0 * g * g) * a42 - 7.0 / 2.0 + 13.0 * g - 4.5 * g * g;
    H(2, 1) = -(15.0 / 4.0 - 15.0 * g + 21.0 / 4.0 * g * g) * a42 + 4.0 - 12.5 * g + 4.5 * g * g;
    H(3, 0) = 1.0 - a42 - a42; H(3, 1) = a42; H(3, 2) = a42;
  } else if (name == "ARS_443") {
    set(4);
    A(0, 0) = A(1, 1) = A(2, 2) = A(3, 3) = 0.5;
    A(1, 0) = 1.0 / 6.0; A(2, 0) = -0.5; A(2, 1) = 0.5; A(3, 0) = 1.5; A(3, 1) = -1.5; A(3, 2) = 0.5;
    H(1, 0) = 0.5; H(2, 0) = 11.0 / 18.0; H(2, 1) = 1.0 / 18.0;
    H(3, 0) = 5.0 / 6.0; H(3, 1) = -5.0 / 6.0; H(3, 2) = 0.5;
    H(4, 0) = 0.25; H(4, 1) = 7.0 / 4.0; H(4, 2) = 0.75; H(4, 3) = -7.0 / 4.0;
  } else {
    throw CoralError(CORAL_EBADARG, "Invalid time-stepping scheme code: " + name);
  }
  return t;
}

// --- Chebyshev matrices (chebyshev_elementary.f90:28-151) -------------------------

static Dense matmul(const Dense& a, const Dense& b) {
  size_t n = a.size(), m = b[0].size(), k = b.size();
  Dense c(n, std::vector<double>(m, 0.0));
  for (size_t i = 0; i < n; ++i)
    for (size_t l = 0; l < k; ++l) {
      double v = a[i][l];
      if (v == 0.0) continue;
      for (size_t j = 0; j < m; ++j) c[i][j] += v * b[l][j];
    }
  return c;
}

Dense cheb_IM(int N, double center, double gap, int a, int b, int padding) {
  int Np = N + padding;
  Dense I(Np, std::vector<double>(Np, 0.0)), M(Np, std::vector<double>(Np, 0.0));
  M[1][0] = gap / 2.0;
  for (int i = 0; i < Np - 1; ++i) M[i][i + 1] = gap / 4.0;
  for (int i = 1; i < Np - 1; ++i) M[i + 1][i] = gap / 4.0;
  for (int i = 0; i < Np; ++i) M[i][i] = center;
  I[1][0] = 2.0;
  for (int fi = 2; fi < Np; ++fi) I[fi][fi - 1] = 1.0 / double(fi);
  for (int fi = 2; fi < Np; ++fi) I[fi - 1][fi] = -1.0 / double(fi - 1);
  for (auto& row : I)
    for (auto& v : row) v *= gap / 4.0;
  Dense R(Np, std::vector<double>(Np, 0.0));
  for (int i = 0; i < Np; ++i) R[i][i] = 1.0;
  for (int k = 0; k < a; ++k) R = matmul(R, I);
  for (int k = 0; k < b; ++k) R = matmul(R, M);
  Dense out(N, std::vector<double>(N));
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) out[i][j] = R[i][j];
  return out;
}

// --- Galerkin stencils (chebyshev_galerkin_2.f90:7-409) -----------------------------

Dense stencil(int N, int bc) {
  auto make = [&](int nc) { return Dense(N, std::vector<double>(nc, 0.0)); };
  if (bc == 0) {
    Dense S = make(N);
    for (int j = 0; j < N; ++j) S[j][j] = 1.0;
    return S;
  }
  if (bc >= 10 && bc <= 13) {
    Dense S = make(N - 1);
    for (int j = 1; j < N; ++j) {
      double d0, d1;
      if (bc == 10) { d0 = -1.0; d1 = 1.0; }
      else if (bc == 11) { d0 = 1.0; d1 = 1.0; }
      else if (bc == 12) { d0 = -(j + 1.0) * (j + 1.0); d1 = double(j) * double(j); }
      else { d0 = (j + 1.0) * (j + 1.0); d1 = double(j) * double(j); }
      S[j - 1][j - 1] = d0;
      S[j][j - 1] = d1;
    }
    return S;
  }
  if (bc >= 20 && bc <= 24) {
    Dense S = make(N - 2);
    if (bc == 24) {
      S[0][0] = 1.0; S[1][1] = 1.0;
      for (int j = 3; j <= N - 2; ++j) {
        S[j + 1][j - 1] = 1.0;
        double n = double(j + 1);
        S[j - 1][j - 1] = -n * n * (n * n + 1.0) / ((n * n - 3.0 * n + 2.0) * (n * n - 5.0 * n + 6.0));
      }
      return S;
    }
    for (int j = 1; j <= N - 2; ++j) {
      if (bc == 20) { S[j - 1][j - 1] = -1.0; S[j + 1][j - 1] = 1.0; }
      else if (bc == 21) {
        S[j - 1][j - 1] = -1.0;
        double n = double(j + 1);
        S[j + 1][j - 1] = (n - 2.0) * (n - 2.0) / (n * n);
      } else {
        double n = double(j - 1), sg = (bc == 22) ? -1.0 : 1.0;
        S[j - 1][j - 1] = 1.0;
        S[j][j - 1] = sg * (4.0 * n + 4.0) / (2.0 * n * n + 6.0 * n + 5.0);
        S[j + 1][j - 1] = -(n * n + (n + 1.0) * (n + 1.0)) / ((n + 1.0) * (n + 1.0) + (n + 2.0) * (n + 2.0));
      }
    }
    return S;
  }
  if (bc >= 40 && bc <= 43) {
    Dense S = make(N - 4);
    for (int j = 1; j <= N - 4; ++j) {
      if (bc == 40) {
        double n = double(j + 3);
        S[j - 1][j - 1] = -1.0;
        S[j + 1][j - 1] = (2.0 * n - 4.0) / (n - 1.0);
        S[j + 3][j - 1] = -(n - 3.0) / (n - 1.0);
      } else if (bc == 41) {
        double n = double(j + 3);
        double m = 24.0 * n / (2.0 * n * n - 4.0 * n + 3.0);
        m = m - 18.0 / (n - 1.0);
        S[j - 1][j - 1] = -1.0;
        S[j + 1][j - 1] = m + 2.0;
        S[j + 3][j - 1] = -m - 1.0;
      } else {
        double n = double(j - 1), s = (bc == 42) ? -1.0 : 1.0;
        S[j - 1][j - 1] = 1.0;
        S[j][j - 1] = s * (2.0 * n + 2.0) / (n * n + 5.0 * n + 7.0);
        S[j + 1][j - 1] = -(2.0 * n * n * n + 12.0 * n * n + 28.0 * n + 24.0) / (n * n * n + 8.0 * n * n + 22.0 * n + 21.0);
        S[j + 2][j - 1] = -s * (2.0 * n + 2.0) / (n * n + 5.0 * n + 7.0);
        S[j + 3][j - 1] = (n * n * n + 4.0 * n * n + 6.0 * n + 3.0) / (n * n * n + 8.0 * n * n + 22.0 * n + 21.0);
      }
    }
    return S;
  }
  throw CoralError(CORAL_EBADARG, "unknown boundary-condition code " + std::to_string(bc));
}

// --- system assembly ----------------------------------------------------------------

static std::vector<std::vector<int>> interleave(const std::vector<int>& sizes) {
  int nV = int(sizes.size());
  int nmin = *std::min_element(sizes.begin(), sizes.end());
  std::vector<std::vector<int>> pos(nV);
  int rem = 0;
  for (int v = 0; v < nV; ++v) {
    for (int c = 0; c < sizes[v]; ++c)
      pos[v].push_back(c < nmin ? v + c * nV : nmin * nV + rem + (c - nmin));
    rem += sizes[v] - nmin;
  }
  return pos;
}

namespace {
struct Triplet { int row, col, grp; double val; };
}

static void finish_ell(EllOp& op, int rows, std::vector<Triplet>& tr) {
  // sum duplicates (same row, col, group) in insertion order, drop exact zeros
  std::sort(tr.begin(), tr.end(), [](const Triplet& a, const Triplet& b) {
    if (a.row != b.row) return a.row < b.row;
    if (a.col != b.col) return a.col < b.col;
    return a.grp < b.grp;
  });
  std::vector<Triplet> m;
  for (auto& t : tr) {
    if (!m.empty() && m.back().row == t.row && m.back().col == t.col && m.back().grp == t.grp) m.back().val += t.val;
    else m.push_back(t);
  }
  std::vector<std::vector<Triplet>> per(rows);
  for (auto& t : m)
    if (t.val != 0.0) per[t.row].push_back(t);
  int w = 0;
  for (auto& p : per) w = std::max<int>(w, int(p.size()));
  op.rows = rows;
  op.width = std::max(w, 1);
  op.col.assign(size_t(rows) * op.width, -1);
  op.val.assign(size_t(rows) * op.width, 0.0);
  op.grp.assign(size_t(rows) * op.width, 0);
  for (int r = 0; r < rows; ++r)
    for (size_t k = 0; k < per[r].size(); ++k) {
      op.col[size_t(r) * op.width + k] = per[r][k].col;
      op.val[size_t(r) * op.width + k] = per[r][k].val;
      op.grp[size_t(r) * op.width + k] = per[r][k].grp;
    }
}

static int group_of(EllOp& op, int a, int b) {
  for (size_t i = 0; i < op.groups.size(); ++i)
    if (op.groups[i].first == a && op.groups[i].second == b) return int(i);
  op.groups.emplace_back(a, b);
  return int(op.groups.size()) - 1;
}

// Connected components of the bipartite graph (equation rows, variable columns)
// of every stored entry of M and L, gathered into two classes of equal size.
// Leaves ncls = 1 when the pattern is one block or a block is not square.
static void split_classes(SystemOps& o) {
  const int T = o.T;
  std::vector<int> par(2 * T);
  for (int u = 0; u < 2 * T; ++u) par[u] = u;
  auto find = [&](int u) {
    while (par[u] != u) u = par[u] = par[par[u]];
    return u;
  };
  for (const EllOp* op : {&o.M, &o.L})
    for (int rr = 0; rr < op->rows; ++rr)
      for (int k = 0; k < op->width; ++k) {
        const int c = op->col[size_t(rr) * op->width + k];
        if (c < 0) continue;
        const int a = find(rr), b = find(T + c);
        if (a != b) par[a] = b;
      }
  std::map<int, std::pair<int, int>> count;  // root -> (rows, columns)
  for (int t = 0; t < T; ++t) {
    ++count[find(t)].first;
    ++count[find(T + t)].second;
  }
  if (count.size() < 2) return;
  for (const auto& kv : count)
    if (kv.second.first != kv.second.second) return;
  // largest components first, each into the smaller class
  std::vector<std::pair<int, int>> comps;  // (size, root)
  for (const auto& kv : count) comps.emplace_back(kv.second.first, kv.first);
  std::stable_sort(comps.begin(), comps.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
    return a.first > b.first;
  });
  std::map<int, int> cls_of_root;
  int size[2] = {0, 0};
  for (const auto& cp : comps) {
    const int cl = (size[0] <= size[1]) ? 0 : 1;
    cls_of_root[cp.second] = cl;
    size[cl] += cp.first;
  }
  const int Tc = std::max(size[0], size[1]);
  o.ncls = 2;
  o.Tc = Tc;
  o.row_cls_pos.assign(T, -1);
  o.col_cls_pos.assign(T, -1);
  o.cls_row.assign(2 * (size_t)Tc, -1);
  int nr[2] = {0, 0}, nc[2] = {0, 0};
  for (int t = 0; t < T; ++t) {
    const int cr = cls_of_root[find(t)];
    o.row_cls_pos[t] = cr * Tc + nr[cr];
    o.cls_row[cr * Tc + nr[cr]] = t;
    ++nr[cr];
    const int cc = cls_of_root[find(T + t)];
    o.col_cls_pos[t] = cc * Tc + nc[cc]++;
  }
  o.kl_cls = o.ku_cls = 0;
  for (const EllOp* op : {&o.M, &o.L})
    for (int rr = 0; rr < op->rows; ++rr)
      for (int k = 0; k < op->width; ++k) {
        const int c = op->col[size_t(rr) * op->width + k];
        if (c < 0) continue;
        const int i = o.row_cls_pos[rr] % Tc, j = o.col_cls_pos[c] % Tc;
        o.kl_cls = std::max(o.kl_cls, i - j);
        o.ku_cls = std::max(o.ku_cls, j - i);
      }
}

SystemOps assemble_system(const Geometry& g, const Recipe& r, const CoupledSet& s) {
  (void)r;
  SystemOps o;
  const int NZ = g.NZ;
  o.nV = int(s.vars.size());
  if (int(s.orders.size()) != o.nV)
    throw CoralError(CORAL_EPARSE, "Incompatible number of coupled equations and variables");
  o.bcs = s.bcs;
  o.orders = s.orders;
  int T1 = 0, T2 = 0;
  for (int v = 0; v < o.nV; ++v) {
    o.var_size.push_back(NZ - s.bcs[v] / 10);
    o.eq_size.push_back(NZ - s.orders[v]);
    T1 += o.eq_size.back();
    T2 += o.var_size.back();
  }
  if (T1 != T2) throw CoralError(CORAL_EPARSE, "Incompatible number of boundary conditions");
  o.T = T1;
  o.var_pos = interleave(o.var_size);
  o.eq_pos = interleave(o.eq_size);

  std::vector<Dense> S(o.nV);
  for (int v = 0; v < o.nV; ++v) S[v] = stencil(NZ, s.bcs[v]);
  std::map<std::pair<int, int>, Dense> im;
  auto IM = [&](int a, int b) -> const Dense& {
    auto k = std::make_pair(a, b);
    auto it = im.find(k);
    if (it == im.end()) it = im.emplace(k, cheb_IM(NZ, g.center, g.gap, a, b)).first;
    return it->second;
  };

  auto build = [&](const std::vector<Piece>& pieces, EllOp& op) {
    std::vector<Triplet> tr;
    for (const Piece& p : pieces) {
      int grp = group_of(op, p.kx, p.ky);
      const Dense& C = IM(p.Iz, p.mz);
      const Dense& Sv = S[p.jVar];
      int o_e = s.orders[p.iEqn];
      int nc = int(Sv[0].size());
      for (int rr = 0; rr < o.eq_size[p.iEqn]; ++rr) {
        const auto& crow = C[o_e + rr];
        for (int c = 0; c < nc; ++c) {
          double acc = 0.0;
          for (int n = 0; n < NZ; ++n)
            if (crow[n] != 0.0 && Sv[n][c] != 0.0) acc += crow[n] * Sv[n][c];
          if (acc != 0.0) tr.push_back({o.eq_pos[p.iEqn][rr], o.var_pos[p.jVar][c], grp, p.dsca * acc});
        }
      }
    }
    finish_ell(op, o.T, tr);
  };
  build(s.mass, o.M);
  build(s.stif, o.L);
  if (o.M.groups.empty()) o.M.groups.emplace_back(0, 0);
  if (o.L.groups.empty()) o.L.groups.emplace_back(0, 0);
  // band of E = M - dt a L
  o.kl = o.ku = 0;
  for (const EllOp* op : {&o.M, &o.L})
    for (int rr = 0; rr < op->rows; ++rr)
      for (int k = 0; k < op->width; ++k) {
        int c = op->col[size_t(rr) * op->width + k];
        if (c < 0) continue;
        o.kl = std::max(o.kl, rr - c);
        o.ku = std::max(o.ku, c - rr);
      }
  // NL assembly rows
  {
    std::vector<Triplet> tr;
    for (const NLTerm& t : s.nl) {
      int grp = group_of(o.NLop, t.dx, t.dy);
      const Dense& C = IM(t.Iz, t.mz);
      int o_e = s.orders[t.eqn];
      for (int rr = 0; rr < o.eq_size[t.eqn]; ++rr)
        for (int n = 0; n < NZ; ++n) {
          double v = C[o_e + rr][n];
          if (v != 0.0) tr.push_back({o.eq_pos[t.eqn][rr], t.quad * NZ + n, grp, t.dsca * v});
        }
    }
    finish_ell(o.NLop, o.T, tr);
    if (o.NLop.groups.empty()) o.NLop.groups.emplace_back(0, 0);
  }
  // real scaling: parity of (i kx)^a (i ky)^b is a+b; an entry of equation e and
  // variable v becomes real under the scaling iff r_e = (a+b+s_v) mod 2
  {
    const int nV = o.nV;
    std::vector<int> r_e(nV, -1), s_v(nV, -1);
    std::vector<std::array<int, 3>> edges;  // (e, v, parity)
    for (const auto* pieces : {&s.mass, &s.stif})
      for (const Piece& p : *pieces) edges.push_back({p.iEqn, p.jVar, (p.kx + p.ky) & 1});
    bool ok = true;
    // propagate from each unlabelled equation
    for (int start = 0; start < nV && ok; ++start) {
      if (r_e[start] >= 0) continue;
      r_e[start] = 0;
      bool changed = true;
      while (changed && ok) {
        changed = false;
        for (auto& ed : edges) {
          int e = ed[0], v = ed[1], par = ed[2];
          if (r_e[e] >= 0 && s_v[v] < 0) { s_v[v] = (r_e[e] + par) & 1; changed = true; }
          else if (s_v[v] >= 0 && r_e[e] < 0) { r_e[e] = (s_v[v] + par) & 1; changed = true; }
          else if (s_v[v] >= 0 && r_e[e] >= 0 && r_e[e] != ((s_v[v] + par) & 1)) ok = false;
        }
      }
    }
    for (int v = 0; v < nV; ++v)
      if (s_v[v] < 0) s_v[v] = 0;
    o.real_scalable = ok;
    o.row_flip.assign(o.T, 0);
    o.col_flip.assign(o.T, 0);
    if (ok) {
      for (int e = 0; e < nV; ++e)
        for (int rr : o.eq_pos[e]) o.row_flip[rr] = (unsigned char)r_e[e];
      for (int v = 0; v < nV; ++v)
        for (int c : o.var_pos[v]) o.col_flip[c] = (unsigned char)s_v[v];
    }
  }
  // stencil rows and square stencils
  o.stencil_rows.resize(o.nV);
  o.sq_stencil.resize(o.nV);
  for (int v = 0; v < o.nV; ++v) {
    o.stencil_rows[v].resize(NZ);
    int nc = int(S[v][0].size());
    for (int n = 0; n < NZ; ++n)
      for (int c = 0; c < nc; ++c)
        if (S[v][n][c] != 0.0) o.stencil_rows[v][n].emplace_back(c, S[v][n][c]);
    Dense sq(nc, std::vector<double>(nc));
    for (int i = 0; i < nc; ++i)
      for (int j = 0; j < nc; ++j) sq[i][j] = S[v][i][j];
    o.sq_stencil[v] = sq;
  }
  split_classes(o);
  return o;
}

}  // namespace coral
